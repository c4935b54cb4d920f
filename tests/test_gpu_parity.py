"""Parity of the CUDA path (through the C-ABI) against the reference's outputs and the oracle.

FP64 mode is compiled without FMA contraction and follows the reference's operation order, so
it is expected to reproduce the reference bit for bit; the bar written in the tests is the
stated FP64 tolerance, 1e-12 relative (L-inf over the field, relative to its max magnitude).
"""

import numpy as np
import pytest

from golden_cases import golden_steps, load_cases, rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
# Redlich-Kwong and Kataoka mixtures: the device solves the cubic in FP64 where the reference uses
# long double, and its pow / exp / acos ... round their last bit differently from the host's
REAL_GAS_TOL = 1e-11
COMPARE = ["c1", "c2", "c3", "vx", "vy", "p", "rho", "E", "mx", "my"]
# the fixtures with chemistry are checked by test_gpu_chemistry.py (exp/pow round differently on
# the GPU, and velocities that start from rest are compared on the flow's speed scale there)
CASES = [c for c in load_cases() if c[1].chemistry == "no"]


@pytest.fixture(scope="module")
def fv():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from schemi_b200 import fv as fvmod

    fvmod.load()
    return fvmod


def _advance(g, n, t_end):
    for _ in range(n):
        g.step()
        t, dt = g.time()
        if t + dt > t_end:
            g.set_time(t, t_end - t)


@pytest.mark.parametrize("name,case,prim,data", CASES, ids=[c[0] for c in CASES])
def test_gpu_fp64_matches_reference(fv, name, case, prim, data):
    tol = REAL_GAS_TOL if case.eos in ("RedlichKwong", "Kataoka") else FP64_TOL
    g = fv.FVCase(case)
    g.upload(prim)
    t_end = float(data["t_end"])
    done = 0
    worst = 0.0
    for target in golden_steps(data):
        _advance(g, target - done, t_end)
        done = target
        t, _ = g.time()
        assert abs(t - float(data[f"time_{target}"])) <= 1e-14 * max(1.0, abs(t))
        out = g.download()
        for f in COMPARE:
            key = f"{f}_{target}"
            if key in data and f in out:
                linf, l1 = rel_err(out[f], data[key])
                worst = max(worst, linf)
                assert linf <= tol, f"{name} step {target} {f}: rel Linf {linf:.3e} L1 {l1:.3e}"
    print(f"{name}: max rel Linf vs reference = {worst:.3e}")


def test_gpu_run_config1_full(fv):
    """Config 1 through fv_run (device time loop in CUDA graphs): 955 steps to t = 0.2."""
    name, case, prim, data = [c for c in CASES if c[0] == "shock_tube_1d_full"][0]
    g = fv.FVCase(case)
    g.upload(prim)
    st = g.run(case.t_end)
    n = int(data["n_steps"])
    assert st.steps == n
    assert st.time == pytest.approx(0.2, abs=1e-15)
    out = g.download()
    for f in COMPARE:
        key = f"{f}_{n}"
        if key in data:
            linf, _ = rel_err(out[f], data[key])
            assert linf <= FP64_TOL, f"{f}: {linf:.3e}"


def _oracle_compare(fv, oracle_mod, case, prim, steps, tol, fields=COMPARE, l1=False):
    g = fv.FVCase(case)
    g.upload(prim)
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    worst = 0.0
    for _ in range(steps):
        g.step()
        oc.step()
    a, b = g.download(), oc.download()
    for f in fields:
        if f in a and f in b:
            linf, rl1 = rel_err(a[f], b[f])
            e = rl1 if l1 else linf
            worst = max(worst, e)
            assert e <= tol, f"{case.name} {f}: rel {'L1' if l1 else 'Linf'} {e:.3e}"
    return g, worst


def test_gpu_periodic_kh_march_matches_oracle(fv, oracle_mod):
    from schemi_b200 import cases

    case, prim = cases.kelvin_helmholtz_2d(n=64)
    g, worst = _oracle_compare(fv, oracle_mod, case, prim, 20, FP64_TOL)
    assert g.path == fv.PATH_MARCH


def test_gpu_march_equals_generic(fv):
    """The fused march (zero slopes proven by the limiter) equals the full MUSCL-Hancock."""
    from schemi_b200 import cases

    case, prim = cases.kelvin_helmholtz_2d(n=48)
    a = fv.FVCase(case)
    b = fv.FVCase(case)
    b.force_generic()
    a.upload(prim)
    b.upload(prim)
    for _ in range(10):
        a.step()
        b.step()
    oa, ob = a.download(), b.download()
    for f in COMPARE:
        if f in oa:
            assert np.array_equal(oa[f], ob[f]), f


def test_gpu_3d_vdw_periodic_matches_oracle(fv, oracle_mod):
    from schemi_b200 import cases

    case, prim = cases.reacting_shear_3d(n=16, precision="f64")
    case.chemistry = "no"
    _oracle_compare(fv, oracle_mod, case, prim, 5, FP64_TOL)


def test_gpu_3d_generic_linear_matches_oracle(fv, oracle_mod):
    from schemi_b200 import cases

    case, prim = cases.reacting_shear_3d(n=10, precision="f64")
    case.chemistry = "no"
    case.limiter = "linear"
    g, _ = _oracle_compare(fv, oracle_mod, case, prim, 3, FP64_TOL)
    assert g.path == fv.PATH_GENERIC


def test_gpu_fp32_flux_within_tolerance(fv, oracle_mod):
    """FP32 flux arithmetic with FP64 accumulation: relative L1 error <= 1e-5 after 20 steps."""
    from schemi_b200 import cases

    case, prim = cases.kelvin_helmholtz_2d(n=64, precision="f32flux")
    _oracle_compare(fv, oracle_mod, case, prim, 20, 1e-5, l1=True)


def _f32_march_cases():
    """2D FP32-flux cases for the warp-strip march: strip and tile edges (odd widths, fewer
    columns than a strip, fewer rows than a tile), every patch type, gravity and both fluxes."""
    from schemi_b200 import cases
    from schemi_b200.case import BC, PatchBC

    out = []
    c, p = cases.rayleigh_taylor_2d(nx=37, ny=70, modes=3, precision="f32flux")
    c.g_delta = (0.0, -0.05, 0.0)
    out.append(("rt_gravity_37x70", c, p))
    c, p, _ = cases.richtmyer_meshkov(1, n=61, precision="f32flux")
    out.append(("rm_free_slip_61", c, p))
    c, p = cases.kelvin_helmholtz_2d(n=45, precision="f32flux", periodic=False)
    c.bc["tail"] = PatchBC([BC("fixedValueCell", 0.05), BC("fixedValueCell", 0.05)],
                           BC("fixedValueCell", (0.6, 0.01, 0.0)), BC("fixedValueCell", 2.6))
    c.bc["point"] = PatchBC.uniform("freeBoundary", 2)
    c.bc["right"] = PatchBC.uniform("periodic", 2)
    c.bc["left"] = PatchBC.uniform("periodic", 2)
    out.append(("kh_inflow_periodic_y_45", c, p))
    c, p = cases.kelvin_helmholtz_2d(n=20, precision="f32flux")
    c.flux = "HLL"
    out.append(("kh_hll_20", c, p))
    c, p = cases.rayleigh_taylor_2d(nx=94, ny=5, modes=2, precision="f32flux")
    out.append(("rt_short_94x5", c, p))
    return out


@pytest.mark.parametrize("name,case,prim", _f32_march_cases(), ids=[c[0] for c in _f32_march_cases()])
def test_gpu_fp32_flux_march_cases(fv, oracle_mod, name, case, prim):
    """FP32-flux 2D march on strip / tile edges and every patch type: relative L1 <= 1e-5.
    A velocity component that starts at zero (the x velocity of Rayleigh-Taylor, the y velocity
    of Richtmyer-Meshkov) stays at 1e-7 .. 1e-10 for these few steps, far below FP32 rounding of
    the flow, so velocities are measured on the flow's speed scale sqrt(max p / min rho) and
    momenta on that scale times the largest density."""
    g = fv.FVCase(case)
    g.upload(prim)
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    for _ in range(15):
        g.step()
        oc.step()
    a, b = g.download(), oc.download()
    assert g.path == fv.PATH_MARCH
    speed = float(np.sqrt(b["p"].max() / b["rho"].min()))
    floors = {"vx": speed, "vy": speed, "mx": speed * b["rho"].max(), "my": speed * b["rho"].max()}
    worst = 0.0
    for f in COMPARE:
        if f in a and f in b:
            ref = np.maximum(np.abs(b[f]), floors.get(f, 0.0))
            e = float(np.sum(np.abs(a[f] - b[f])) / max(np.sum(ref), 1e-300))
            worst = max(worst, e)
            assert e <= 1e-5, f"{name} {f}: rel L1 {e:.3e}"
    print(f"{name}: max rel L1 vs oracle = {worst:.3e}")


@pytest.mark.parametrize("limiter,fails_at", [("UTCDFS", 2), ("linear", 4)])
def test_gpu_riemann_failure_status(fv, limiter, fails_at):
    """The reference's Riemann failures on the 200-cell tube (UTCDFS at step 2, the unlimited
    linear reconstruction at step 4) end the same step on the GPU with RiemannSolverError."""
    from schemi_b200 import cases

    c, p = cases.shock_tube_1d(n=200)
    c.limiter = limiter
    g = fv.FVCase(c)
    g.upload(p)
    for _ in range(fails_at - 1):
        g.step()
    with pytest.raises(fv.FVError) as ei:
        g.step()
    assert ei.value.status == 1


def test_gpu_download_into_pinned_buffers(fv):
    """fv_download into caller-owned page-locked arrays returns the same values as into new
    arrays, and a buffer of the wrong size is refused before the call."""
    import torch

    from schemi_b200 import cases

    case, prim = cases.kelvin_helmholtz_2d(n=48)
    g = fv.FVCase(case)
    g.upload(prim)
    for _ in range(3):
        g.step()
    ref = g.download()
    outs = {name: torch.zeros(g.n_cells, dtype=torch.float64, pin_memory=True).numpy()
            for name in g.download_fields()}
    got = g.download(outs)
    assert set(got) == set(ref)
    for name in ref:
        assert got[name] is outs[name]
        assert np.array_equal(got[name], ref[name]), name
    outs["p"] = np.zeros(g.n_cells - 1)
    with pytest.raises(ValueError):
        g.download(outs)


def test_step_kernel_finalizes_itself(fv, oracle_mod):
    """Without chemistry the step kernel's last CTA runs the CFL finalize: one launch per step on
    the fused march (four on the generic path), and a run of steps through fv_run still matches
    the oracle step for step (the clock, the step sizes and the state)."""
    from schemi_b200 import cases

    case, prim = cases.kelvin_helmholtz_2d(n=64)
    g = fv.FVCase(case)
    assert g.path == fv.PATH_MARCH and g.kernels_per_step == 1
    g.upload(prim)
    st = g.run(1.0, max_steps=25)
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    for _ in range(25):
        oc.step()
    assert st.steps == 25
    assert g.time() == oc.time()
    a, b = g.download(), oc.download()
    for f in COMPARE:
        if f in a and f in b:
            linf, _ = rel_err(a[f], b[f])
            assert linf <= FP64_TOL, f
    t, _ = cases.shock_tube_1d(n=100)
    assert fv.FVCase(t).kernels_per_step == 4


@pytest.mark.parametrize("eos", ["stiffened", "RedlichKwong", "Kataoka"])
def test_gpu_real_gas_2d_and_f32flux_against_oracle(fv, oracle_mod, eos):
    """The real-gas mixtures on a 2D mesh (generic path, periodic in x) against the FP64 oracle,
    in FP64 and in FP32-flux arithmetic (their EOS stays FP64 in both)."""
    import numpy as np

    from schemi_b200 import cases
    from schemi_b200.case import PatchBC

    tube, tprim = cases.real_gas_tube(eos, n=24)
    for prec, tol, l1 in (("f64", REAL_GAS_TOL if eos != "stiffened" else FP64_TOL, False), ("f32flux", 1e-5, True)):
        case = tube.__class__(**{**tube.__dict__})
        case.dims, case.n, case.precision = 2, (24, 24, 1), prec
        case.bc = {"tail": PatchBC.uniform("periodic", 2), "point": PatchBC.uniform("periodic", 2),
                   "right": PatchBC.uniform("slip", 2), "left": PatchBC.uniform("slip", 2)}
        # the tube's jump along y, a small shear along x
        prim = [np.repeat(a, 24) for a in tprim]
        prim[2] = 0.3 * np.sqrt(np.abs(prim[5]) / np.maximum(prim[0] + prim[1], 1e-30)) * np.tile(
            np.sin(np.linspace(0, 2 * np.pi, 24, endpoint=False)), 24)
        g, worst = _oracle_compare(fv, oracle_mod, case, prim, 8, tol, l1=l1)
        assert g.path == fv.PATH_GENERIC


def test_fp64_primitive_cache_follows_the_state(fv, oracle_mod):
    """The FP64 warp strip reuses the primitives its previous step recovered; a new state (upload)
    must not see the old ones, and mixing single steps, runs and time changes keeps the result the
    oracle's bit for bit."""
    from schemi_b200 import cases

    case, prim = cases.kelvin_helmholtz_2d(n=40)
    _, other = cases.kelvin_helmholtz_2d(n=40, seed=7)
    g = fv.FVCase(case)
    g.upload(prim)
    g.run(1.0, max_steps=6)        # primitives cached for the state of step 6
    g.upload(other)                # a different state: the cache must be dropped
    g.step()
    g.run(1.0, max_steps=4)
    t, dt = g.time()
    g.set_time(t, dt)
    g.step()
    oc = oracle_mod.OracleCase(case)
    oc.upload(other)
    for _ in range(6):
        oc.step()
    assert g.time() == oc.time()
    a, b = g.download(), oc.download()
    for f in COMPARE:
        if f in a and f in b:
            linf, _ = rel_err(a[f], b[f])
            assert linf <= FP64_TOL, f
