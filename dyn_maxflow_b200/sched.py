"""Learned schedule picker: trace recording, training and evaluation.

The picker (dmf_sched, kernels in csrc/dmf_sched.cu) is an MLP 12 -> 64 -> 64 -> 4
with bf16 weights and fp32 accumulation.  Per update batch it predicts, for each
of four schedules (ACTIONS), log2 of the time the batch would take, and the
solver runs the cheapest.  Every schedule computes the same exact maximum flow,
so a wrong pick costs time, never correctness; the plain schedule (action 0)
is the fallback when no model is given and the yardstick of the time regret.

Traces.  For every batch of a training run the solver measures the batch's
features on the device against the live residual state (dmf_solver_features),
then the batch is solved under each action from that same state
(dmf_solver_copy_state into a scratch solver, dmf_apply_updates_action); the
four times are the targets.  The trunk state then advances.

  python -m dyn_maxflow_b200.sched record --out traces.npz [--scales 16,17,18 --seeds 40 --batches 10]
  python -m dyn_maxflow_b200.sched train --traces traces.npz --out weights.npz [--steps 4000]
  python -m dyn_maxflow_b200.sched eval --weights weights.npz [--scale 20 --seeds 1000,1001 --batches 20]
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

import dyn_maxflow_b200 as D

FEATURE_NAMES = (
    "batch_fraction",          # k / m
    "log_batch_size",          # log2(1 + k) / 24
    "frac_decreases",
    "frac_saturating_decreases",  # new capacity below the arc's current flow
    "excess_created_over_flow",   # sum(flow - new cap) over those / current flow value
    "frac_increases_on_saturated",
    "frac_inserts",             # capacity 0 -> positive
    "frac_deletes",             # positive -> 0
    "log_mean_tail_degree",
    "log_max_tail_degree",
    "log_last_bfs_depth",       # BFS levels per global relabel of the previous solve
    "log_vertices",
)

# defaults of the mixed update batches (the R-MAT batch parameters of the
# benchmark configurations): 40% increases, 40% decreases, 10% inserts, 10% deletes
MIX = dict(p_inc=0.4, p_dec=0.4, p_ins=0.1, delta_hi=500, ins_lo=1, ins_hi=1000)


def rmat_instance(scale: int, seed: int, reserve_frac: float = 0.02):
    """R-MAT graph (a=0.57, b=0.19, c=0.19, 16 * 2^scale samples, caps U[1,1000]) with
    reserved insert slots; s = max out-degree vertex, t = max in-degree other vertex."""
    narcs = 16 << scale
    g, s, t = D.gen_rmat(scale, narcs, 0.57, 0.19, 0.19, seed=seed, cap_lo=1, cap_hi=1000,
                         reserve=int(reserve_frac * narcs) + 16)
    return g, s, t


def batch_sizes(rng, count: int, lo: float, hi: float):
    """Batch fractions log-uniform in [lo, hi]."""
    return np.exp(rng.uniform(math.log(lo), math.log(hi), size=count))


def next_batch(g, frac: float, seed: int):
    (b,) = D.gen_batches(g, 1, frac=float(frac), seed=seed, **MIX)
    return b


def record(specs, batches: int, frac_lo: float, frac_hi: float, verbose=True, out=None, save_every=8):
    """Traces of (features, per-action log2 ms) over R-MAT instances `specs` =
    [(scale, seed), ...].  Returns X[n,12], T[n,4] (ms), meta list.  With `out`,
    the traces so far are saved there every `save_every` instances."""
    X, T, meta = [], [], []
    for done, (scale, seed) in enumerate(specs, 1):
        t0 = time.time()
        g, s, t = rmat_instance(scale, seed)
        trunk = D.Solver(g, s, t)
        scratch = D.Solver(g, s, t)
        trunk.static_maxflow()
        scratch.copy_state_from(trunk)
        rng = np.random.default_rng(seed)
        fracs = batch_sizes(rng, batches, frac_lo, frac_hi)
        # one untimed pass of every action so that no timing holds first-launch costs
        bs, bd, bw = next_batch(g, 1e-3, seed * 7919 + 99991)
        for a in range(D.N_ACTIONS):
            scratch.copy_state_from(trunk)
            scratch.apply_updates_action(a, bs, bd, bw)
        for b, frac in enumerate(fracs):
            bs, bd, bw = next_batch(g, frac, seed * 7919 + b)
            x = trunk.features(bs, bd, bw)
            times, flows = [], []
            for a in range(D.N_ACTIONS):
                scratch.copy_state_from(trunk)
                flows.append(scratch.apply_updates_action(a, bs, bd, bw))
                times.append(scratch.stats()["last_ms"])
            if len(set(flows)) != 1:
                raise RuntimeError(f"actions disagree on the flow: {flows} (scale {scale} seed {seed} batch {b})")
            trunk.copy_state_from(scratch)  # advance (state of the last action)
            g.set_caps(bs, bd, bw)          # keep the host capacities in step for the generator
            X.append(x)
            T.append(times)
            meta.append({"scale": scale, "seed": seed, "batch": b, "k": int(len(bs)), "flow": int(flows[0])})
        trunk.close()
        scratch.close()
        if verbose:
            print(f"recorded scale {scale} seed {seed}: {batches} batches in {time.time() - t0:.1f}s", flush=True)
        if out and (done % save_every == 0 or done == len(specs)):
            np.savez(out, X=np.array(X, np.float32), T=np.array(T, np.float32), meta=json.dumps(meta))
    return np.array(X, np.float32), np.array(T, np.float32), meta


MARGIN = 0.1  # log2 units a non-plain action must be predicted to win by (the model's default)


def targets(T) -> np.ndarray:
    """log2 of each action's time over the plain schedule's (column 0 is 0): the
    differences that decide the pick are the whole target, not a small part of
    an absolute time that varies 100x across graph sizes."""
    L = np.log2(np.maximum(np.asarray(T, np.float64), 1e-3))
    return (L - L[:, :1]).astype(np.float32)


def balance(X, T, groups):
    """Repeats samples so that every group (graph scale) weighs the same."""
    groups = np.asarray(groups)
    keys, counts = np.unique(groups, return_counts=True)
    mx = counts.max()
    idx = np.concatenate([np.repeat(np.where(groups == k)[0], int(math.ceil(mx / c))) for k, c in zip(keys, counts)])
    return X[idx], T[idx]


def pick_actions(pred, margin=MARGIN) -> np.ndarray:
    """The decision rule of the device kernel (k_decide) on predictions."""
    pred = np.asarray(pred)
    best = np.zeros(len(pred), int)
    bestv = pred[:, 0] - margin
    for a in range(1, pred.shape[1]):
        better = pred[:, a] < bestv
        best[better] = a
        bestv = np.where(better, pred[:, a], bestv)
    return best


def train(X, T, groups=None, steps=4000, lr=3e-3, seed=0, device=-1):
    """Trains a Scheduler on traces (balanced over `groups` when given); returns
    (scheduler, loss curve)."""
    if groups is not None:
        X, T = balance(np.asarray(X), np.asarray(T), groups)
    sched = D.Scheduler(device, seed)
    loss = sched.train(X, targets(T), steps=steps, batch=64, lr=lr, seed=seed)
    return sched, loss


def choice_quality(sched, X, T) -> dict:
    """Offline quality on traces: time of the picked action vs plain and vs the best."""
    pred = sched.predict(X)
    pick = pick_actions(pred)
    T = np.asarray(T, np.float64)
    rows = np.arange(len(T))
    return {
        "n": int(len(T)),
        "plain_ms": float(T[:, 0].sum()),
        "learned_ms": float(T[rows, pick].sum()),
        "best_ms": float(T.min(1).sum()),
        "pick_hist": np.bincount(pick, minlength=D.N_ACTIONS).tolist(),
        "best_hist": np.bincount(T.argmin(1), minlength=D.N_ACTIONS).tolist(),
    }


def evaluate(sched, specs, batches: int, frac_lo: float, frac_hi: float, oracle=True, verbose=True, warmup=1):
    """The learned schedule against the plain one on held-out instances
    (`warmup` untimed batches of 0.1% first).

    Paired timing (oracle=True): before the learned solver applies a batch, the
    batch is solved under every action from a copy of the learned solver's
    state; the learned time of the batch is the time of the action it picks,
    the plain time that of action 0, both from the same state.  (Two solvers
    that apply the same batches independently hold different residual flows --
    push-relabel's atomics make the flow decomposition vary -- so their times
    differ by several per cent even under the same schedule.)  A plain solver
    also runs its own trajectory; every flow of every action and of both
    solvers must be identical.  With oracle=False only the two live solvers
    are timed."""
    plain_ms, learned_ms, best_ms, picks, exact = [], [], [], [], True
    live_plain, live_learned = [], []
    for scale, seed in specs:
        g, s, t = rmat_instance(scale, seed)
        P = D.Solver(g, s, t)
        L = D.Solver(g, s, t)
        O = D.Solver(g, s, t) if oracle else None
        P.static_maxflow()
        L.static_maxflow()
        rng = np.random.default_rng(seed)
        fracs = batch_sizes(rng, batches, frac_lo, frac_hi)
        for wi in range(warmup):  # untimed
            bs, bd, bw = next_batch(g, 1e-3, seed * 7919 + 99991 + wi)
            P.apply_updates_scheduled(None, bs, bd, bw)
            L.apply_updates_scheduled(sched, bs, bd, bw)
            if O is not None:
                for a in range(D.N_ACTIONS):
                    O.copy_state_from(L)
                    O.apply_updates_action(a, bs, bd, bw)
            g.set_caps(bs, bd, bw)
        for b, frac in enumerate(fracs):
            bs, bd, bw = next_batch(g, frac, seed * 7919 + b)
            t_all, f_all = [], []
            if O is not None:
                for a in range(D.N_ACTIONS):
                    O.copy_state_from(L)
                    f_all.append(O.apply_updates_action(a, bs, bd, bw))
                    t_all.append(O.stats()["last_ms"])
            fp, _ = P.apply_updates_scheduled(None, bs, bd, bw)
            live_plain.append(P.stats()["last_ms"])
            fl, a = L.apply_updates_scheduled(sched, bs, bd, bw)
            live_learned.append(L.stats()["last_ms"])
            picks.append(a)
            exact &= fp == fl and all(f == fl for f in f_all)
            if t_all:
                plain_ms.append(t_all[0])
                learned_ms.append(t_all[a])
                best_ms.append(min(t_all))
            else:
                plain_ms.append(live_plain[-1])
                learned_ms.append(live_learned[-1])
            g.set_caps(bs, bd, bw)
        for x in (P, L, O):
            if x is not None:
                x.close()
        if verbose:
            print(f"evaluated scale {scale} seed {seed}", flush=True)

    def pct(v, q):
        return float(np.percentile(np.asarray(v), q)) if v else None

    def summary(v):
        return {"total_ms": float(np.sum(v)), "p50_ms": pct(v, 50), "p99_ms": pct(v, 99)}

    out = {
        "batches": len(plain_ms), "exact_equal_flows": bool(exact), "timing": "paired" if best_ms else "live",
        "plain": summary(plain_ms), "learned": summary(learned_ms),
        "live_solvers": {"plain": summary(live_plain), "learned": summary(live_learned)},
        "pick_hist": np.bincount(np.asarray(picks, int), minlength=D.N_ACTIONS).tolist(),
        "per_batch": {"plain_ms": [round(x, 4) for x in plain_ms], "learned_ms": [round(x, 4) for x in learned_ms],
                      "best_ms": [round(x, 4) for x in best_ms], "picks": [int(a) for a in picks]},
    }
    out["speedup_vs_plain"] = out["plain"]["total_ms"] / max(out["learned"]["total_ms"], 1e-9)
    if best_ms:
        out["best_total_ms"] = float(np.sum(best_ms))
        out["regret_vs_best"] = out["learned"]["total_ms"] / max(out["best_total_ms"], 1e-9) - 1.0
        out["plain_regret_vs_best"] = out["plain"]["total_ms"] / max(out["best_total_ms"], 1e-9) - 1.0
    return out


# ---- numpy restatement of the forward pass (for tests) -------------------------
def bf16_to_f32(bits: np.ndarray) -> np.ndarray:
    return (np.asarray(bits, np.uint32) << 16).view(np.float32)


def forward_reference(weights: np.ndarray, biases: np.ndarray, X: np.ndarray) -> np.ndarray:
    """fp32 forward of the same bf16 weights (checks the CUDA inference)."""
    W = bf16_to_f32(weights)
    W1 = W[:768].reshape(64, 12)
    W2 = W[768:768 + 4096].reshape(64, 64)
    W3 = W[4864:].reshape(4, 64)
    b1, b2, b3 = biases[:64], biases[64:128], biases[128:]
    h1 = np.maximum(np.asarray(X, np.float32) @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    return h2 @ W3.T + b3


def _specs(scales, seeds, spread=False):
    """Every seed at every scale, or (spread) seed i at scales[i % len(scales)]."""
    if spread:
        return [(scales[i % len(scales)], sd) for i, sd in enumerate(seeds)]
    return [(sc, sd) for sd in seeds for sc in scales]


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m dyn_maxflow_b200.sched")
    sub = ap.add_subparsers(dest="cmd", required=True)
    r = sub.add_parser("record")
    r.add_argument("--out", required=True)
    r.add_argument("--scales", default="16,17,18")
    r.add_argument("--seeds", type=int, default=40)
    r.add_argument("--seed-base", type=int, default=0)
    r.add_argument("--batches", type=int, default=10)
    r.add_argument("--frac-lo", type=float, default=5e-4)
    r.add_argument("--frac-hi", type=float, default=0.1)
    r.add_argument("--spread", action="store_true",
                   help="one graph per seed, the scales taken in turn (200 seeds over 7 scales = 200 graphs)")
    t = sub.add_parser("train")
    t.add_argument("--traces", required=True, nargs="+")
    t.add_argument("--out", required=True)
    t.add_argument("--steps", type=int, default=4000)
    t.add_argument("--lr", type=float, default=3e-3)
    e = sub.add_parser("eval")
    e.add_argument("--weights", required=True)
    e.add_argument("--scale", type=int, default=20)
    e.add_argument("--seeds", default="1000,1001")
    e.add_argument("--batches", type=int, default=20)
    e.add_argument("--frac-lo", type=float, default=5e-4)
    e.add_argument("--frac-hi", type=float, default=0.1)
    a = ap.parse_args(argv)
    if a.cmd == "record":
        scales = [int(x) for x in a.scales.split(",")]
        specs = _specs(scales, range(a.seed_base, a.seed_base + a.seeds), spread=a.spread)
        X, T, meta = record(specs, a.batches, a.frac_lo, a.frac_hi, out=a.out)
        np.savez(a.out, X=X, T=T, meta=json.dumps(meta))
        print(f"{len(X)} records -> {a.out}")
    elif a.cmd == "train":
        Xs, Ts, G = [], [], []
        for p in a.traces:
            d = np.load(p)
            Xs.append(d["X"])
            Ts.append(d["T"])
            G += [m["scale"] for m in json.loads(str(d["meta"]))]
        X, T = np.concatenate(Xs), np.concatenate(Ts)
        sched, loss = train(X, T, groups=G, steps=a.steps, lr=a.lr)
        sched.save(a.out)
        q = choice_quality(sched, X, T)
        print(json.dumps({"loss_first": float(loss[:50].mean()), "loss_last": float(loss[-50:].mean()),
                          "train_quality": q}))
    else:
        sched = D.Scheduler.load(a.weights)
        specs = _specs([a.scale], [int(x) for x in a.seeds.split(",")])
        print(json.dumps(evaluate(sched, specs, a.batches, a.frac_lo, a.frac_hi)))


if __name__ == "__main__":
    main()
