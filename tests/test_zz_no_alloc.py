"""fv_step_noalloc: the step entry point for hosts that cannot allocate device memory on the
step's path (pooling allocators that forbid driver allocations, loops that cannot take the
synchronisation of cudaMalloc).  Its results must equal the handle-based fv_step's, to the FP64
tolerance of the parity tests, on two calls in a row.  This file is collected last."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12
F32_TOL = 1e-5  # relative L1, the FP32-flux tolerance of the parity tests


@pytest.fixture(scope="module")
def env():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from schemi_b200 import fv

    lib = fv.load()
    lib.fv_step_noalloc.restype = ctypes.c_int
    lib.fv_step_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                    ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    return torch, fv, lib


def _conserved(g):
    """Conserved state of a handle in the library layout, read through fv_download."""
    out = g.download()
    N = g.case.n_species
    fields = [out[f"rho{k + 1}"] for k in range(N)] + [out["rho"], out["mx"], out["my"], out["mz"], out["E"]]
    return np.concatenate(fields)


def _compare(a, b, n_cells, n_fields, f32=False):
    for f in range(n_fields):
        x = a[f * n_cells:(f + 1) * n_cells]
        y = b[f * n_cells:(f + 1) * n_cells]
        if f32:
            err = np.abs(x - y).sum() / max(np.abs(y).sum(), 1e-300)
            assert err <= F32_TOL, f"field {f}: rel L1 {err:.3e}"
        else:
            scale = max(np.abs(y).max(), 1e-300)
            assert np.abs(x - y).max() / scale <= TOL, f"field {f}"


def _case(which):
    from schemi_b200 import cases

    if which == "tube_1000":
        return cases.shock_tube_1d(n=1000)
    if which == "kh_slip_24":
        return cases.kelvin_helmholtz_2d(n=24, periodic=False)
    if which == "kh_periodic_24_f32flux":
        return cases.kelvin_helmholtz_2d(n=24, precision="f32flux")
    # 3D, periodic in x and z, three van der Waals species, 512 cells
    case, prim = cases.reacting_shear_3d(n=8, precision="f64")
    case.chemistry = "no"
    return case, prim


@pytest.mark.parametrize("which", ["tube_1000", "kh_slip_24", "kh_periodic_24_f32flux", "shear3d_8_vdw_periodic"])
def test_noalloc_matches_handle_step_twice(env, which):
    torch, fv, lib = env
    case, prim = _case(which)
    f32 = case.precision == "f32flux"
    g = fv.FVCase(case)
    if f32:
        g.force_generic()  # the FP32-flux march computes faces in another order; compare like with like
    g.upload(prim)
    g.step()  # step 1 (uses the restart primitives); both paths continue from its state
    cfg = case.fv_config()
    n, nf = case.n_cells, case.n_conserved
    src = torch.tensor(_conserved(g), dtype=torch.float64, device="cuda")
    dst = torch.empty_like(src)
    torch.cuda.synchronize()
    for call in range(2):
        dt_used, dt_next = g.step()
        ref = _conserved(g)
        got_dt = ctypes.c_double()
        st = lib.fv_step_noalloc(ctypes.byref(cfg), ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()),
                                 dt_used, ctypes.byref(got_dt), ctypes.c_void_p(0))
        assert st == 0, f"call {call}: status {st}"
        _compare(dst.cpu().numpy(), ref, n, nf, f32)
        assert abs(got_dt.value - dt_next) <= (F32_TOL if f32 else TOL) * dt_next
        src, dst = dst, src


def test_noalloc_rejects_oversized_mesh(env):
    torch, fv, lib = env
    from schemi_b200 import cases

    case, _ = cases.kelvin_helmholtz_2d(n=64, periodic=False)  # 4096 cells > 1024
    cfg = case.fv_config()
    buf = torch.zeros(case.n_conserved * case.n_cells, dtype=torch.float64, device="cuda")
    dt = ctypes.c_double()
    st = lib.fv_step_noalloc(ctypes.byref(cfg), ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(buf.data_ptr()),
                             1e-6, ctypes.byref(dt), ctypes.c_void_p(0))
    assert st == 11  # initialisationError


@pytest.mark.parametrize("order", ["SecondOrderRK", "ThirdOrder", "ThirdOrderCada"])
def test_noalloc_rejects_multistage_solvers(env, order):
    torch, fv, lib = env
    from schemi_b200 import cases

    case, _ = cases.kelvin_helmholtz_2d(n=16, periodic=False)
    case.order = order
    cfg = case.fv_config()
    a = torch.zeros(case.n_conserved * case.n_cells, dtype=torch.float64, device="cuda")
    b = torch.zeros_like(a)
    dt = ctypes.c_double()
    st = lib.fv_step_noalloc(ctypes.byref(cfg), ctypes.c_void_p(a.data_ptr()), ctypes.c_void_p(b.data_ptr()),
                             1e-6, ctypes.byref(dt), ctypes.c_void_p(0))
    assert st == 11


def test_noalloc_rejects_overlapping_state(env):
    """The step reads state_in while writing state_out: the same or overlapping arrays are refused."""
    torch, fv, lib = env
    from schemi_b200 import cases

    case, _ = cases.kelvin_helmholtz_2d(n=16, periodic=False)
    cfg = case.fv_config()
    n = case.n_conserved * case.n_cells
    buf = torch.zeros(n + 64, dtype=torch.float64, device="cuda")
    dt = ctypes.c_double()
    for off in (0, 64):
        st = lib.fv_step_noalloc(ctypes.byref(cfg), ctypes.c_void_p(buf.data_ptr()),
                                 ctypes.c_void_p(buf.data_ptr() + 8 * off), 1e-6, ctypes.byref(dt), ctypes.c_void_p(0))
        assert st == 11
