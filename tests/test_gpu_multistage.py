"""Multi-stage step solvers on the GPU: SecondOrderRK (two stages without the Hancock predictor,
then the 0.5 average that keeps the averaged concentrations as state; secondOrderStepSolverRK.cpp,
Advection2dOrder.cpp), ThirdOrder (SSP-RK3 of the directional reconstruction;
thirdOrderStepSolver.cpp, Advection3dOrder.cpp, thirdOrderLimiter.hpp) and ThirdOrderCada (the
same stages with the smoothness switch of thirdOrderLimiterCada.hpp).

The reference fixtures of these step solvers (tests/golden/*_rk2*.npz, *_rk3*.npz, *_cada*.npz)
are checked step by step by test_gpu_parity.py; these tests cover the device time loop, periodic
meshes (which the reference cannot express) and 3D against the oracle, the FP32-flux arithmetic
and the kernel counts.
"""

import numpy as np
import pytest

from golden_cases import rel_err

pytestmark = pytest.mark.gpu

FIELDS = ["c1", "c2", "c0", "vx", "vy", "p", "rho", "E", "T"]


@pytest.fixture(scope="module")
def fv():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from schemi_b200 import fv as fvmod

    fvmod.load()
    return fvmod


def _rk2(case):
    case.order = "SecondOrderRK"
    return case


def _rk3(case):
    case.order = "ThirdOrder"
    return case


@pytest.mark.parametrize("limiter,path", [("vanLeer", "march"), ("linear", "generic")])
def test_rk2_periodic_run_matches_oracle(fv, oracle_mod, limiter, path):
    """Periodic KH through fv_run (CUDA graphs): FP64 within 1e-12 of the oracle."""
    from schemi_b200 import cases

    case, prim = cases.kelvin_helmholtz_2d(n=40, limiter=limiter)
    _rk2(case)
    case.t_end = 0.05
    g = fv.FVCase(case)
    g.upload(prim)
    st = g.run(case.t_end)
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    _, steps = oc.run(case.t_end)
    assert st.steps == steps
    assert g.time()[0] == oc.time()[0]
    assert g.path == (fv.PATH_MARCH if path == "march" else fv.PATH_GENERIC)
    a, b = g.download(), oc.download()
    for f in FIELDS:
        linf, _ = rel_err(a[f], b[f])
        assert linf <= 1e-12, f"{f}: {linf:.3e}"


def test_rk2_f32flux_within_tolerance(fv, oracle_mod):
    """FP32-flux stages (warp-strip march) with the FP64 average: relative L1 <= 1e-5."""
    from schemi_b200 import cases

    case, prim = cases.kelvin_helmholtz_2d(n=64, precision="f32flux")
    _rk2(case)
    g = fv.FVCase(case)
    g.upload(prim)
    ref_case, _ = cases.kelvin_helmholtz_2d(n=64)
    _rk2(ref_case)
    oc = oracle_mod.OracleCase(ref_case)
    oc.upload(prim)
    for _ in range(15):
        g.step()
        oc.step()
    a, b = g.download(), oc.download()
    for f in ["c1", "c2", "vx", "p", "rho", "E"]:
        _, l1 = rel_err(a[f], b[f])
        assert l1 <= 1e-5, f"{f}: {l1:.3e}"


def test_rk2_kernels_per_step(fv):
    from schemi_b200 import cases

    case, prim = cases.kelvin_helmholtz_2d(n=32)
    g = fv.FVCase(_rk2(case))
    assert g.kernels_per_step == 4  # two march stages, the average, the CFL finalize
    case, prim = cases.shock_tube_1d(n=50)
    g = fv.FVCase(_rk2(case))
    assert g.kernels_per_step == 10  # two generic stages of four kernels, average, finalize


def test_rk2_rejected_where_unsupported(fv):
    from schemi_b200 import cases

    case, prim, _ = cases.richtmyer_meshkov(0, n=32, precision="f32flux")
    g = fv.FVCase(_rk2(case))
    g.upload(prim)
    with pytest.raises(fv.FVError):
        fv.FVBatch([g])


@pytest.mark.parametrize("limiter", ["vanLeer", "minmod2"])
def test_rk3_periodic_run_matches_oracle(fv, oracle_mod, limiter):
    """Periodic KH (wrap faces in the directional limiter) through fv_run: FP64 within 1e-12."""
    from schemi_b200 import cases

    case, prim = cases.kelvin_helmholtz_2d(n=32, limiter=limiter)
    _rk3(case)
    case.t_end = 0.04
    g = fv.FVCase(case)
    g.upload(prim)
    st = g.run(case.t_end)
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    _, steps = oc.run(case.t_end)
    assert st.steps == steps
    assert g.time()[0] == oc.time()[0]
    assert g.path == fv.PATH_GENERIC
    a, b = g.download(), oc.download()
    for f in FIELDS:
        linf, _ = rel_err(a[f], b[f])
        assert linf <= 1e-12, f"{f}: {linf:.3e}"


def test_rk3_f32flux_within_tolerance(fv, oracle_mod):
    from schemi_b200 import cases

    case, prim = cases.kelvin_helmholtz_2d(n=48, precision="f32flux")
    _rk3(case)
    g = fv.FVCase(case)
    g.upload(prim)
    ref_case, _ = cases.kelvin_helmholtz_2d(n=48)
    _rk3(ref_case)
    oc = oracle_mod.OracleCase(ref_case)
    oc.upload(prim)
    for _ in range(10):
        g.step()
        oc.step()
    a, b = g.download(), oc.download()
    for f in ["c1", "c2", "vx", "p", "rho", "E"]:
        _, l1 = rel_err(a[f], b[f])
        assert l1 <= 1e-5, f"{f}: {l1:.3e}"


def test_rk3_kernels_per_step(fv):
    from schemi_b200 import cases

    case, prim = cases.kelvin_helmholtz_2d(n=32)
    g = fv.FVCase(_rk3(case))
    assert g.path == fv.PATH_GENERIC
    assert g.kernels_per_step == 15  # three generic stages of four kernels, two averages, finalize


def _cada(case):
    case.order = "ThirdOrderCada"
    return case


@pytest.mark.parametrize("limiter", ["vanLeer", "superbee"])
def test_cada_periodic_run_matches_oracle(fv, oracle_mod, limiter):
    """Periodic KH with ThirdOrderCada through fv_run: FP64 within 1e-12 of the oracle."""
    from schemi_b200 import cases

    case, prim = cases.kelvin_helmholtz_2d(n=32, limiter=limiter)
    _cada(case)
    case.t_end = 0.04
    g = fv.FVCase(case)
    g.upload(prim)
    st = g.run(case.t_end)
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    _, steps = oc.run(case.t_end)
    assert st.steps == steps
    assert g.time()[0] == oc.time()[0]
    assert g.path == fv.PATH_GENERIC
    assert g.kernels_per_step == 15
    a, b = g.download(), oc.download()
    for f in FIELDS:
        linf, _ = rel_err(a[f], b[f])
        assert linf <= 1e-12, f"{f}: {linf:.3e}"


def test_cada_3d_matches_oracle(fv, oracle_mod):
    """3D periodic shear layer (van der Waals mixture, 9-component velocity gradients in the
    switch) with ThirdOrderCada: FP64 within 1e-12 of the oracle after 3 steps."""
    from schemi_b200 import cases

    case, prim = cases.reacting_shear_3d(n=10, precision="f64")
    case.chemistry = "no"
    _cada(case)
    g = fv.FVCase(case)
    g.upload(prim)
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    for _ in range(3):
        g.step()
        oc.step()
    a, b = g.download(), oc.download()
    for f in ["c1", "c2", "c3", "vx", "vy", "p", "rho", "E"]:
        if f in a and f in b:
            linf, _ = rel_err(a[f], b[f])
            assert linf <= 1e-12, f"{f}: {linf:.3e}"


def test_cada_f32flux_within_tolerance(fv, oracle_mod):
    """ThirdOrderCada in FP32-flux arithmetic: relative L1 <= 1e-5 against the FP64 oracle."""
    from schemi_b200 import cases

    case, prim = cases.kelvin_helmholtz_2d(n=48, precision="f32flux")
    _cada(case)
    g = fv.FVCase(case)
    g.upload(prim)
    ref_case, _ = cases.kelvin_helmholtz_2d(n=48)
    _cada(ref_case)
    oc = oracle_mod.OracleCase(ref_case)
    oc.upload(prim)
    for _ in range(10):
        g.step()
        oc.step()
    a, b = g.download(), oc.download()
    for f in ["c1", "c2", "vx", "p", "rho", "E"]:
        _, l1 = rel_err(a[f], b[f])
        assert l1 <= 1e-5, f"{f}: {l1:.3e}"
