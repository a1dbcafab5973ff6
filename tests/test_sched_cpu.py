"""Host-side checks of the learned schedule picker (no GPU needed): constants
agree between include/dmf.h and the package, the numpy restatement of the
forward pass used to check the CUDA inference is itself right, and a model
cannot be created without a device (no CPU fallback)."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_defines():
    hdr = open(os.path.join(ROOT, "include", "dmf.h")).read()
    return {k: int(v) for k, v in re.findall(r"#define (DMF_SCHED_[A-Z]+|DMF_ACTION_[A-Z]+) (\d+)", hdr)}


def test_constants_match_header(dmf):
    d = header_defines()
    assert d["DMF_SCHED_FEATURES"] == dmf.N_FEATURES == 12
    assert d["DMF_SCHED_HIDDEN"] == dmf.N_HIDDEN == 64
    assert d["DMF_SCHED_ACTIONS"] == dmf.N_ACTIONS == len(dmf.ACTIONS) == 4
    assert d["DMF_SCHED_WEIGHTS"] == dmf.N_WEIGHTS == 64 * 12 + 64 * 64 + 4 * 64
    assert d["DMF_SCHED_BIASES"] == dmf.N_BIASES == 64 + 64 + 4
    assert [d["DMF_ACTION_PLAIN"], d["DMF_ACTION_SHORT"], d["DMF_ACTION_REVIVE"], d["DMF_ACTION_RECOMPUTE"]] == [0, 1, 2, 3]
    from dyn_maxflow_b200 import sched
    assert len(sched.FEATURE_NAMES) == dmf.N_FEATURES


def test_bf16_decoding():
    from dyn_maxflow_b200 import sched
    bits = np.array([0x3F80, 0xBF80, 0x4000, 0x0000, 0x3E80], np.uint16)
    np.testing.assert_array_equal(sched.bf16_to_f32(bits), np.array([1.0, -1.0, 2.0, 0.0, 0.25], np.float32))


def test_forward_reference_layout():
    """A hand-made net whose output is known: unit 0 of each hidden layer copies
    feature 0 (through ReLU), action a's output = (a + 1) * that unit + bias a."""
    from dyn_maxflow_b200 import sched
    one = 0x3F80
    w = np.zeros(5120, np.uint16)
    w[0 * 12 + 0] = one             # W1[0][0]
    w[768 + 0 * 64 + 0] = one       # W2[0][0]
    two, three, four = 0x4000, 0x4040, 0x4080
    for a, bits in enumerate([one, two, three, four]):
        w[4864 + a * 64 + 0] = bits  # W3[a][0]
    b = np.zeros(132, np.float32)
    b[128:] = [0.5, -1.0, 0.0, 2.0]
    X = np.zeros((3, 12), np.float32)
    X[:, 0] = [0.0, 1.5, -2.0]
    out = sched.forward_reference(w, b, X)
    x0 = np.maximum(X[:, 0], 0)
    want = np.stack([x0 * (a + 1) + b[128 + a] for a in range(4)], 1)
    np.testing.assert_allclose(out, want, rtol=0, atol=1e-6)


def test_scheduler_needs_a_device(dmf):
    if dmf.device_count() > 0:
        pytest.skip("a GPU is visible")
    with pytest.raises(dmf.DmfError):
        dmf.Scheduler()


def test_committed_model_on_its_traces():
    """The shipped weights, run through the numpy forward pass and the kernel's
    decision rule on the recorded traces: never slower than the plain schedule
    by more than 1% per scale, and faster overall."""
    import glob
    import json
    from dyn_maxflow_b200 import sched
    d = np.load(os.path.join(ROOT, "dyn_maxflow_b200", "sched_weights.npz"))
    w, b = d["weights"], d["biases"]
    assert w.dtype == np.uint16 and w.shape == (5120,) and b.dtype == np.float32 and b.shape == (132,)
    assert np.isfinite(sched.bf16_to_f32(w)).all() and np.isfinite(b).all()
    plain_all = learned_all = 0.0
    for p in sorted(glob.glob(os.path.join(ROOT, "dyn_maxflow_b200", "sched_data", "traces_*.npz"))):
        t = np.load(p)
        X, T = t["X"], t["T"].astype(np.float64)
        scale = np.array([m["scale"] for m in json.loads(str(t["meta"]))])
        pick = sched.pick_actions(sched.forward_reference(w, b, X))
        for s in np.unique(scale):
            i = scale == s
            plain = T[i, 0].sum()
            learned = T[i][np.arange(i.sum()), pick[i]].sum()
            assert learned <= 1.01 * plain, (p, s, plain, learned)
            plain_all += plain
            learned_all += learned
    assert plain_all > 0 and learned_all < 0.97 * plain_all
