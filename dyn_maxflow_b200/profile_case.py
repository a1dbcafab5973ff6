"""A small, fixed launch sequence for profiling the solve kernel:

    python -m dyn_maxflow_b200.profile_case SCALE BATCHES

One solver on the R-MAT graph of the given scale (the benchmark's generator
and parameters: a=0.57 b=0.19 c=0.19, 16 * 2^scale samples, caps U[1,1000],
reserved insert slots), a static solve (k_solve launch 0), then BATCHES
successive 1% mixed batches already on the device (launches 1..BATCHES).
Prints one JSON line: per launch the flow, device ms and counters.
"""
from __future__ import annotations

import json
import sys


def main(argv=None) -> None:
    import torch
    import dyn_maxflow_b200 as D
    argv = sys.argv[1:] if argv is None else argv
    scale, nb = int(argv[0]), int(argv[1])
    narcs = 16 << scale
    g, s, t = D.gen_rmat(scale, narcs, 0.57, 0.19, 0.19, seed=0, cap_lo=1, cap_hi=1000,
                         reserve=int(0.1 * 0.01 * narcs * 10) + 16)
    batches = D.gen_batches(g, nb, frac=0.01, p_inc=0.4, p_dec=0.4, p_ins=0.1, delta_hi=500, ins_lo=1,
                            ins_hi=1000, seed=1)
    torch.cuda.set_device(0)
    dbat = [[torch.as_tensor(x, dtype=torch.int32).cuda() for x in b] for b in batches]
    with D.Solver(g, s, t) as sv:
        out = [{"launch": "static", "flow": sv.static_maxflow(), "ms": sv.stats()["last_ms"]}]
        for b in dbat:
            f = sv.apply_updates_device(b[0].data_ptr(), b[1].data_ptr(), b[2].data_ptr(), int(b[0].numel()))
            st = sv.stats()
            out.append({"launch": "batch", "flow": f, "ms": st["last_ms"], "arcs_scanned": st["arcs_scanned"],
                        "bfs_arcs": st["bfs_arcs"], "dead_kept": st["dead_kept"]})
    print(json.dumps(out))


if __name__ == "__main__":
    main()
