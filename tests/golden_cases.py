"""Golden fixtures (reference outputs) and the cases that produced them.

The case definitions live in tests/golden/make_golden.py; the .npz files hold the reference's
per-step outputs for them.
"""

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def load_cases():
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = []
    for name, case, prim, nsteps, keep in mod.golden_cases():
        data = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
        out.append((name, case, prim, data))
    return out


def golden_steps(data):
    return sorted({int(k.split("_")[1]) for k in data if k.startswith("time_")})


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale), float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))
