"""Batched ensemble (many uneven cases in one persistent kernel) against the same cases run one by
one through the single-case path: identical states, step counts and times, case by case."""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["c1", "c2", "vx", "vy", "p", "rho", "E"]


@pytest.fixture(scope="module")
def fv():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from schemi_b200 import fv as fvmod

    fvmod.load()
    return fvmod


@pytest.mark.parametrize("precision", ["f64", "f32flux"])
def test_batch_equals_plain_runs(fv, precision):
    from schemi_b200 import cases

    sizes = [32, 40, 48, 56, 64, 72]
    built = [cases.richtmyer_meshkov(i, n=n, precision=precision) for i, n in enumerate(sizes)]
    # end times of a handful of steps each, different per case
    t_end = [t * 0.002 * (1 + i % 3) for i, (_, _, t) in enumerate(built)]
    plain, batched = [], []
    for case, prim, _ in built:
        a = fv.FVCase(case)
        a.upload(prim)
        plain.append(a)
        b = fv.FVCase(case)
        b.upload(prim)
        batched.append(b)
    steps_plain = [a.run(te).steps for a, te in zip(plain, t_end)]
    batch = fv.FVBatch(batched)
    stats = batch.run(t_end)
    assert stats.steps_max == max(steps_plain)
    assert stats.cell_updates == sum(s * c.n_cells for s, (c, _, _) in zip(steps_plain, built))
    for a, b in zip(plain, batched):
        ta, tb = a.time()[0], b.time()[0]
        assert ta == tb
        oa, ob = a.download(), b.download()
        for f in FIELDS:
            assert np.array_equal(oa[f], ob[f]), f
    # a second run continues every case from where it stopped
    t2 = [te * 1.5 for te in t_end]
    for a, te in zip(plain, t2):
        a.run(te)
    batch.run(t2)
    for a, b in zip(plain, batched):
        oa, ob = a.download(), b.download()
        for f in FIELDS:
            assert np.array_equal(oa[f], ob[f]), f
