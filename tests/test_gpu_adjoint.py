"""Hand-written adjoint (fv_record / fv_adjoint through adjoint.TimeLoop) against
  * the FP64 CPU tangent oracle (oracle/fv_tangent.py, forward mode through an independent torch
    restatement of the same zero-slope step, itself pinned to the C restatement), and
  * central finite differences (h = 1e-6) of the GPU forward replayed with the recorded steps,
on reduced Rayleigh-Taylor grids (the objective is the time-integrated mixing width), a 3D
periodic/slip case with gravity, the HLL flux and the FP32-flux arithmetic."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, NY, T_END = 16, 48, 0.5


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from schemi_b200 import fv

    fv.load()
    return torch


def _rt(precision="f64", flux="HLLC", nx=NX, ny=NY):
    from schemi_b200 import cases

    case, _ = cases.rayleigh_taylor_2d(nx, ny, precision=precision, t_end=T_END)
    case.flux = flux
    return case


def _amplitudes(torch, seed=2029):
    return torch.from_numpy(np.random.default_rng(seed).normal(0.0, 1e-3, size=64))


def _gpu_gradient(torch, case, a, checkpoint_every=10, w=None):
    """dJ/da (and J) through the GPU adjoint; w: optional weight of <w, U_T> added to J."""
    from schemi_b200 import adjoint, fv

    g = fv.FVCase(case)
    ad = a.clone().cuda().requires_grad_(True)
    prim = adjoint.rayleigh_taylor_primitive(ad, case.n[0], case.n[1])
    J, UT = adjoint.TimeLoop.apply(prim, g, T_END, checkpoint_every, 0)
    loss = J if w is None else J + (w.cuda() * UT).sum()
    loss.backward()
    return ad.grad.detach().cpu(), float(loss.detach()), g


def _oracle(torch, case, nx=NX, ny=NY):
    import fv_tangent
    from schemi_b200 import adjoint

    tc = fv_tangent.TangentCase(case)

    def U0(a):
        prim = adjoint.rayleigh_taylor_primitive(a, nx, ny).reshape(6, ny, nx)
        return tc.conserved_from_primitive(list(prim))

    return tc, U0


def test_record_objective_matches_oracle(torch_cuda):
    torch = torch_cuda
    case = _rt()
    a = _amplitudes(torch)
    tc, U0 = _oracle(torch, case)
    dts = tc.schedule(U0(a), T_END)
    J_ref = float(tc.objective(U0(a), dts, 0))
    _, J, g = _gpu_gradient(torch, case, a)
    assert J == pytest.approx(J_ref, rel=1e-12)
    assert g.record(T_END).steps == 0  # already at t_end: nothing to record


def test_replay_reproduces_record(torch_cuda):
    torch = torch_cuda
    from schemi_b200 import adjoint, fv

    case = _rt()
    g = fv.FVCase(case)
    prim = adjoint.rayleigh_taylor_primitive(_amplitudes(torch).cuda(), NX, NY).contiguous()
    torch.cuda.synchronize()
    g.upload_device([prim[i].data_ptr() for i in range(6)])
    rec = g.record(T_END, 9)
    U1 = torch.empty((7, NX * NY), dtype=torch.float64, device="cuda")
    g.state_copy(U1.data_ptr())
    g.upload_device([prim[i].data_ptr() for i in range(6)])
    rep = g.replay()
    U2 = torch.empty_like(U1)
    g.state_copy(U2.data_ptr())
    assert rep.steps == rec.steps > 10
    assert rep.objective == rec.objective
    assert torch.equal(U1, U2)


@pytest.mark.parametrize("flux", ["HLLC", "HLL"])
def test_gradient_matches_tangent_oracle(torch_cuda, flux):
    torch = torch_cuda
    import fv_tangent

    case = _rt(flux=flux)
    a = _amplitudes(torch)
    grad, _, _ = _gpu_gradient(torch, case, a)
    tc, U0 = _oracle(torch, case)
    dts = tc.schedule(U0(a), T_END)
    f = lambda x: tc.objective(U0(x), dts, 0)
    rng = np.random.default_rng(11)
    dirs = [torch.from_numpy(rng.normal(size=64)) for _ in range(3)]
    for m in (0, 4, 31):
        e = torch.zeros(64, dtype=torch.float64)
        e[m] = 1.0
        dirs.append(e)
    scale = float(grad.norm())
    assert scale > 0
    for d in dirs:
        _, dJ = fv_tangent.tangent(f, a, d)
        # FP64 rounding of two independent implementations of the same derivative
        assert float(grad @ d) == pytest.approx(float(dJ), abs=1e-9 * scale * float(d.norm()))


def test_gradient_matches_finite_differences(torch_cuda):
    torch = torch_cuda
    from schemi_b200 import adjoint

    case = _rt()
    a = _amplitudes(torch)
    grad, _, g = _gpu_gradient(torch, case, a)
    h = 1e-6

    def J_at(x):
        prim = adjoint.rayleigh_taylor_primitive(x.cuda(), NX, NY).contiguous()
        torch.cuda.synchronize()
        g.upload_device([prim[i].data_ptr() for i in range(6)])
        return g.replay().objective

    scale = float(grad.abs().max())
    for m in (0, 1, 2, 7, 40):
        e = torch.zeros(64, dtype=torch.float64)
        e[m] = h
        fd = (J_at(a + e) - J_at(a - e)) / (2 * h)
        assert float(grad[m]) == pytest.approx(fd, abs=1e-5 * scale), m


def test_terminal_state_gradient(torch_cuda):
    torch = torch_cuda
    import fv_tangent

    case = _rt()
    a = _amplitudes(torch)
    w = torch.from_numpy(np.random.default_rng(5).normal(size=(7, NX * NY)))
    w[5] = 0.0  # m_z is not carried in 2D
    grad, _, _ = _gpu_gradient(torch, case, a, w=w)
    tc, U0 = _oracle(torch, case)
    dts = tc.schedule(U0(a), T_END)

    def f(x):
        u = U0(x)
        J = torch.zeros((), dtype=torch.float64)
        for dt in dts:
            u = tc.step(u, dt)
            J = J + dt * tc.width(u, 0)
        return J + (w.reshape(7, NY, NX) * u).sum()

    d = torch.from_numpy(np.random.default_rng(6).normal(size=64))
    _, dJ = fv_tangent.tangent(f, a, d)
    assert float(grad @ d) == pytest.approx(float(dJ), rel=1e-9)


def test_checkpoint_interval_does_not_change_gradient(torch_cuda):
    torch = torch_cuda
    case = _rt()
    a = _amplitudes(torch)
    g1, J1, _ = _gpu_gradient(torch, case, a, checkpoint_every=1)
    g7, J7, _ = _gpu_gradient(torch, case, a, checkpoint_every=7)
    g50, J50, _ = _gpu_gradient(torch, case, a, checkpoint_every=50)
    assert J1 == J7 == J50
    assert torch.equal(g7, g50)
    assert torch.equal(g1, g50)


def test_3d_gradient_matches_tangent_oracle(torch_cuda):
    torch = torch_cuda
    import fv_tangent
    from schemi_b200 import adjoint, fv
    from schemi_b200.case import BC, Case, PatchBC, Species

    nx, ny, nz = 12, 10, 8
    sp = [Species(M=3.0, Cv=1.0 / 0.4), Species(M=1.0, Cv=1.0 / 0.6)]
    bc = {"tail": PatchBC.uniform("periodic", 2), "point": PatchBC.uniform("periodic", 2),
          "bottom": PatchBC.uniform("periodic", 2), "top": PatchBC.uniform("periodic", 2),
          "right": PatchBC.uniform("slip", 2), "left": PatchBC.uniform("slip", 2)}
    case = Case(dims=3, n=(nx, ny, nz), L=(1.0, 1.0, 0.8), species=sp, t_end=0.2, limiter="minmod", flux="HLLC",
                courant=0.5, gravity=(0.0, -0.1, 0.0), bc=bc, name="box3d")
    rng = np.random.default_rng(3)
    z, y, x = np.meshgrid((np.arange(nz) + 0.5) / nz * 0.8, (np.arange(ny) + 0.5) / ny, (np.arange(nx) + 0.5) / nx,
                          indexing="ij")
    frac = 0.5 + 0.4 * np.tanh((y - 0.5 - 0.05 * np.sin(2 * np.pi * x)) / 0.1)
    prim = np.stack([frac, 1 - frac, 0.3 * np.sin(2 * np.pi * z / 0.8) + 0.02 * rng.normal(size=frac.shape),
                     0.02 * rng.normal(size=frac.shape), 0.1 * np.cos(2 * np.pi * x), 2.5 + 0.1 * y])
    prim = torch.from_numpy(prim.reshape(6, -1))
    g = fv.FVCase(case)
    p = prim.clone().cuda().requires_grad_(True)
    J, UT = adjoint.TimeLoop.apply(p, g, 0.2, 6, 0)
    J.backward()
    grad = p.grad.detach().cpu()

    tc = fv_tangent.TangentCase(case)
    tc.nmom = 3
    U0 = lambda q: tc.conserved_from_primitive(list(q.reshape(6, nz, ny, nx)))
    dts = tc.schedule(U0(prim), 0.2)
    f = lambda q: tc.objective(U0(q), dts, 0)
    assert float(J) == pytest.approx(float(f(prim)), rel=1e-12)
    for s in range(3):
        d = torch.from_numpy(np.random.default_rng(20 + s).normal(size=prim.shape))
        _, dJ = fv_tangent.tangent(f, prim, d)
        assert float((grad * d).sum()) == pytest.approx(float(dJ), rel=1e-9)


def test_f32flux_gradient_close_to_f64(torch_cuda):
    torch = torch_cuda
    a = _amplitudes(torch)
    g64, J64, _ = _gpu_gradient(torch, _rt("f64"), a)
    g32, J32, _ = _gpu_gradient(torch, _rt("f32flux"), a)
    assert J32 == pytest.approx(J64, rel=1e-5)
    # FP32 face arithmetic in forward and reverse, FP64 accumulation: relative L2 error
    assert float((g32 - g64).norm() / g64.norm()) < 1e-3


def test_adjoint_rejects_unsupported_cases(torch_cuda):
    from schemi_b200 import cases, fv

    case, prim = cases.shock_tube_1d(64)  # 1D: generic path
    g = fv.FVCase(case)
    g.upload(prim)
    with pytest.raises(fv.FVError) as e:
        g.record(0.01)
    assert e.value.status == 11
    g2 = fv.FVCase(_rt())
    with pytest.raises(fv.FVError):
        g2.replay()  # nothing recorded


def test_second_forward_on_the_handle_invalidates_the_first_backward(torch_cuda):
    """A handle keeps one recorded trajectory: after a second forward on the same FVCase, the
    first forward's backward raises instead of returning the gradient of the second."""
    torch = torch_cuda
    from schemi_b200 import adjoint, fv

    case = _rt()
    g = fv.FVCase(case)
    a = _amplitudes(torch).cuda()
    a1 = a.clone().requires_grad_(True)
    J1, _ = adjoint.TimeLoop.apply(adjoint.rayleigh_taylor_primitive(a1, NX, NY), g, T_END, 10, 0)
    a2 = (2 * a).clone().requires_grad_(True)
    J2, _ = adjoint.TimeLoop.apply(adjoint.rayleigh_taylor_primitive(a2, NX, NY), g, T_END, 10, 0)
    with pytest.raises(RuntimeError, match="recorded again"):
        J1.backward()
    J2.backward()  # the latest forward still differentiates
    assert a2.grad is not None and torch.isfinite(a2.grad).all()
