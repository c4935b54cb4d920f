"""The FP64 CPU tangent oracle (oracle/fv_tangent.py) that the CUDA adjoint is checked against:
its forward step against the C restatement (fv_oracle.cpp, itself pinned to the reference binary),
its tangent against central finite differences of its own forward, and the differentiable
Rayleigh-Taylor initial condition against the numpy one."""

import numpy as np
import pytest
import torch


def _state(tc, prim):
    return tc.conserved_from_primitive([torch.from_numpy(np.asarray(p).reshape(tc.shape)) for p in prim])


@pytest.mark.parametrize("name", ["rt", "kh", "rt_hll"])
def test_tangent_forward_matches_c_oracle(oracle_mod, name):
    import fv_tangent
    from schemi_b200 import cases

    if name == "kh":
        case, prim = cases.kelvin_helmholtz_2d(32)
    else:
        case, prim = cases.rayleigh_taylor_2d(16, 48)
        if name == "rt_hll":
            case.flux = "HLL"
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    tc = fv_tangent.TangentCase(case)
    U = _state(tc, prim)
    for _ in range(25):
        t0, _ = oc.time()
        oc.step()
        t1, dt_next = oc.time()
        U = tc.step(U, t1 - t0)
        cons = oc.conserved()
        # rounding-level agreement (different operation order): 1e-13 of the state's scale
        scale = max(float(np.abs(np.asarray(c)).max()) for c in cons)
        for i in range(case.n_conserved):
            ref = np.asarray(cons[i]).reshape(tc.shape)
            assert float(np.abs(U[i].numpy() - ref).max()) <= 1e-13 * scale, (name, i)
        assert tc.cfl(U) == pytest.approx(dt_next, rel=1e-13)


def test_tangent_matches_finite_differences():
    import fv_tangent
    from schemi_b200 import adjoint, cases

    case, _ = cases.rayleigh_taylor_2d(16, 48)
    tc = fv_tangent.TangentCase(case)
    a0 = torch.from_numpy(np.random.default_rng(7).normal(0.0, 1e-3, size=64))

    def U0(a):
        prim = adjoint.rayleigh_taylor_primitive(a, 16, 48).reshape(6, 48, 16)
        return tc.conserved_from_primitive(list(prim))

    dts = tc.schedule(U0(a0), 0.5)
    f = lambda a: tc.objective(U0(a), dts, 0)
    d = torch.from_numpy(np.random.default_rng(8).normal(size=64))
    J, dJ = fv_tangent.tangent(f, a0, d)
    h = 1e-6
    fd = (float(f(a0 + h * d)) - float(f(a0 - h * d))) / (2 * h)
    assert float(dJ) == pytest.approx(fd, rel=1e-6)


def test_rt_primitive_matches_numpy():
    from schemi_b200 import adjoint, cases

    for nx, ny in ((16, 48), (64, 192)):
        case, prim = cases.rayleigh_taylor_2d(nx, ny)
        a = torch.from_numpy(np.random.default_rng(2029).normal(0.0, 1e-3, size=64))
        pt = adjoint.rayleigh_taylor_primitive(a, nx, ny)
        for i in range(6):
            assert np.array_equal(pt[i].numpy(), np.asarray(prim[i]))


def test_a_b_2c_oracle_conserves_mass_and_releases_heat(oracle_mod):
    """A uniform mixture at rest: the advection leaves it alone, so one step is the chemistry
    alone.  The mixture density is unchanged, the species densities still sum to it, C grows at
    the expense of A and B, and the energy rises by q/2 per mole of C formed (equal heat
    capacities: no dCv term)."""
    from schemi_b200 import cases

    case, prim = cases.reacting_shear_3d(n=4, precision="f64", periodic=True)
    case.chem_forward = (1e14, 0.0, case.chem_forward[2])
    n = case.n_cells
    c = float(prim[0].max())
    prim = [np.full(n, 0.4 * c), np.full(n, 0.4 * c), np.full(n, 0.2 * c), np.zeros(n), np.zeros(n), np.zeros(n),
            np.full(n, 101325.0)]
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    oc.set_time(0.0, 1e-5)  # a step long enough for the heat release to stand far above rounding
    before = oc.download()
    oc.step()
    after = oc.download()
    assert np.allclose(after["rho"], before["rho"], rtol=0, atol=1e-15 * before["rho"].max())
    s = after["rho1"] + after["rho2"] + after["rho3"]
    assert np.allclose(s, after["rho"], rtol=1e-14)
    dC = after["c3"] - before["c3"]
    assert (dC > 0).all() and (after["c1"] < before["c1"]).all()
    dE = after["E"] - before["E"]
    assert np.allclose(dE / dC, 0.5 * case.chem_q, rtol=1e-9)
