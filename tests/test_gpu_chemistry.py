"""Chemistry pass on the GPU (FP64) against the oracle restatement, itself pinned bit for bit to
the reference binary on the Cl2 fixtures: the Cl2 mechanism with every per-cell solver of the
reference, after the SecondOrderRK and ThirdOrder averages as well, the A+B->2C mechanism in 3D
(van der Waals mixture, periodic and slip patches) in FP64 and FP32-flux arithmetic, and the
reference's failure (sub-cycling below the minimal time step)."""

import numpy as np
import pytest

from golden_cases import golden_steps, load_cases, rel_err

pytestmark = pytest.mark.gpu

FIELDS = ["c1", "c2", "c3", "vx", "vy", "vz", "p", "rho", "E", "T"]
# GPU and CPU differ only through the last bit of exp() and pow() inside the rate constants
TOL = 1e-12


@pytest.fixture(scope="module")
def fv():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from schemi_b200 import fv as fvmod

    fvmod.load()
    return fvmod


def _compare(out, ref, fields, tol, what):
    # velocities are measured against the flow's speed scale sqrt(p / rho) (a mixture at rest
    # starts to move at 1e-10 m/s, where a rounding-level difference would look large)
    vscale = float(np.sqrt(np.max(ref["p"]) / np.min(ref["rho"]))) if "p" in ref and "rho" in ref else 0.0
    for f in fields:
        if f in out and f in ref:
            a, b = np.asarray(out[f], dtype=np.float64), np.asarray(ref[f], dtype=np.float64)
            scale = max(float(np.abs(b).max()), vscale if f in ("vx", "vy", "vz") else 0.0, 1e-300)
            linf = float(np.abs(a - b).max()) / scale
            assert linf <= tol, f"{what} field {f}: rel Linf {linf:.3e}"


@pytest.mark.parametrize("name", ["cl2_4x4_vdw_gs", "cl2_4x4_ideal_gs", "cl2_4x4_vdw_jacobi", "cl2_4x4_vdw_ge",
                                  "cl2_4x4_vdw_const_dt", "cl2_4x4_vdw_gs_rk2", "cl2_4x4_ideal_gs_rk3"])
def test_cl2_matches_reference_fixture(fv, name):
    cases = {c[0]: c for c in load_cases()}
    _, case, prim, data = cases[name]
    g = fv.FVCase(case)
    g.upload(prim)
    done = 0
    for target in golden_steps(data):
        while done < target:
            g.step()
            done += 1
        t, _ = g.time()
        assert t == pytest.approx(float(data[f"time_{target}"]), rel=1e-13)
        out = g.download()
        ref = {f: data[f"{f}_{target}"] for f in FIELDS if f"{f}_{target}" in data}
        _compare(out, ref, FIELDS, TOL, f"{name} step {target}")


def test_cl2_matches_oracle_longer_run(fv, oracle_mod):
    from schemi_b200 import cases

    case, prim = cases.chlorine_dissociation_2d(8, seed=11)
    g = fv.FVCase(case)
    g.upload(prim)
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    for s in range(25):
        g.step()
        oc.step()
    assert g.time()[0] == pytest.approx(oc.time()[0], rel=1e-12)
    _compare(g.download(), oc.download(), FIELDS, 1e-11, "cl2 8x8 step 25")


def test_cl2_conjugate_gradient_matches_oracle_per_cell(fv, oracle_mod):
    """With the reference's conjugate-gradient solver (absolute residual tolerance 1e-10 on a system
    whose free term is ~1e5) some cells reach the iteration limit and are sub-cycled.  The
    reference's serial loop keeps the finer sub-step for every later cell; the CUDA path sub-cycles
    the failing cell alone.  The oracle in its per-cell mode reproduces the CUDA path's choice."""
    cases = {c[0]: c for c in load_cases()}
    _, case, prim, data = cases["cl2_4x4_vdw_cg"]
    g = fv.FVCase(case)
    g.upload(prim)
    oc = oracle_mod.OracleCase(case)
    oc.set_chem_carry(False)
    oc.upload(prim)
    for _ in range(6):
        g.step()
        oc.step()
    assert g.time()[0] == pytest.approx(oc.time()[0], rel=1e-13)
    _compare(g.download(), oc.download(), FIELDS, TOL, "cl2 CG per-cell sub-cycling")


def test_cl2_solver_failure_is_reported(fv):
    from schemi_b200 import cases

    case, prim = cases.chlorine_dissociation_2d(4, solver="JacobiConjugateGradient")
    g = fv.FVCase(case)
    g.upload(prim)
    with pytest.raises(fv.FVError) as e:
        g.step()
    assert e.value.status == 4  # systemError, as the reference ("Timestep become too small.")


def _reacting(n, precision, periodic, rate=1e14):
    from schemi_b200 import cases

    case, prim = cases.reacting_shear_3d(n=n, precision=precision, periodic=periodic)
    # a faster reaction than the benchmark's so that a few steps move the composition visibly
    case.chem_forward = (rate, case.chem_forward[1], case.chem_forward[2])
    return case, prim


@pytest.mark.parametrize("periodic", [False, True])
def test_a_b_2c_3d_matches_oracle_f64(fv, oracle_mod, periodic):
    case, prim = _reacting(12, "f64", periodic)
    g = fv.FVCase(case)
    g.upload(prim)
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    c3_0 = np.asarray(prim[2]).copy()
    for _ in range(6):
        g.step()
        oc.step()
    out, ref = g.download(), oc.download()
    assert float(np.abs(ref["c3"] - c3_0).max()) > 1e-3  # the reaction ran
    _compare(out, ref, FIELDS, 1e-11, f"A+B->2C periodic={periodic}")


def test_a_b_2c_3d_f32flux_close_to_oracle(fv, oracle_mod):
    case, prim = _reacting(16, "f32flux", True)
    g = fv.FVCase(case)
    g.upload(prim)
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    for _ in range(5):
        g.step()
        oc.step()
        # the same step sizes, so that the comparison is of the step and not of the CFL rounding
        t, dt = oc.time()
        g.set_time(t, dt)
    out, ref = g.download(), oc.download()
    for f in ("c1", "c2", "c3", "rho", "E", "p"):
        _, l1 = rel_err(out[f], ref[f])
        assert l1 <= 1e-5, f"FP32-flux {f}: rel L1 {l1:.3e}"


def test_chemistry_kernel_counted(fv):
    case, prim = _reacting(8, "f64", True)
    g = fv.FVCase(case)
    assert g.kernels_per_step == 3  # march + chemistry + CFL finalize


@pytest.mark.parametrize("order", ["SecondOrderRK", "ThirdOrderCada"])
def test_a_b_2c_multistage_matches_oracle(fv, oracle_mod, order):
    """A+B->2C after the multi-stage average (the pass reads and averages the stored
    concentrations) in 3D: FP64 within 1e-11 of the oracle after 4 steps, the oracle in per-cell
    sub-cycling (a cell of the fourth ThirdOrderCada step sub-cycles; the reference's serial
    loop would keep the finer sub-step for the cells after it).  ThirdOrder's xi-free limiter
    fails this sharp shear layer in the oracle as in the reference; the Cada switch leaves its
    smooth parts unlimited."""
    case, prim = _reacting(8, "f64", True)
    case.order = order
    g = fv.FVCase(case)
    g.upload(prim)
    oc = oracle_mod.OracleCase(case)
    oc.set_chem_carry(False)
    oc.upload(prim)
    for _ in range(4):
        g.step()
        oc.step()
    assert g.time()[0] == pytest.approx(oc.time()[0], rel=1e-12)
    a, b = g.download(), oc.download()
    _compare(a, b, FIELDS + ["c0"], 1e-11, f"A+B->2C {order}")
    stages = 2 if order == "SecondOrderRK" else 3
    per_stage = 1 if g.path == fv.PATH_MARCH else 4
    # the stages, the averages, the chemistry pass and the CFL finalize
    assert g.kernels_per_step == stages * per_stage + (stages - 1) + 1 + 1
