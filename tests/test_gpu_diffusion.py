"""The diffusion stage on the GPU (Diffusion.cpp through fv_step / fv_run), with the explicit and
the Gauss-Seidel solvers and the constant, hard-sphere and Lennard-Jones transport models,
against the FP64 oracle.

Both follow the reference's operation order in FP64 without contraction, so the device state,
its temperature (the stage's own, not TFromUv of the energy), the CFL step and the source time
step the stage sets must agree bit for bit.  The Lennard-Jones collision integrals and the Cl2
rate constants call pow and exp, whose last bit the device library may round otherwise than the
host's: those cases are compared to a relative tolerance.  The oracle itself is byte-identical to the
reference on the diffusion deck fixtures (tests/test_reference_adapter.py, test_fvrun_deck.py);
tests/test_gpu_fvrun.py and test_gpu_adapter.py replay those decks on the GPU.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["c1", "c2", "c3", "vx", "vy", "vz", "p", "rho", "rho1", "rho2", "mx", "my", "E", "Uv", "T", "sonic"]


@pytest.fixture(scope="module")
def fv():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from schemi_b200 import fv as fvmod

    fvmod.load()
    return fvmod


def _tube(**kw):
    from schemi_b200 import cases

    c, p = cases.shock_tube_1d(n=60)
    c.diffusion, c.mu, c.D, c.kappa = True, 1e-4, 1e-3, 1e-4
    c.enthalpy_flow, c.molmass_diffusion, c.diffusion_timestep = "explicit", True, True
    for k, v in kw.items():
        setattr(c, k, v)
    return c, p


def _vdw_box(dims):
    from schemi_b200 import cases
    from schemi_b200.case import Case, PatchBC

    c3, p3 = cases.reacting_shear_3d(n=6, periodic=False, precision="f64")
    if dims == 3:
        c, p = c3, p3
        c.chemistry = "no"
        for k in list(c.bc):
            c.bc[k] = PatchBC.uniform("slip", 3)
    else:
        c = Case(dims=2, n=(6, 6, 1), L=(1.0, 1.0, 1.0), species=c3.species, t_end=1.0, R_units="SI",
                 eos="vanDerWaals", limiter="vanLeer", name="vdw2d")
        for k in ("tail", "point", "right", "left"):
            c.bc[k] = PatchBC.uniform("slip", 3)
        p = [a.reshape(6, 6, 6)[0].ravel() for a in p3]
    c.diffusion, c.mu, c.D, c.kappa = True, 1e-5, 1e-5, 1e-3
    c.enthalpy_flow, c.molmass_diffusion, c.diffusion_timestep = "explicit", False, True
    return c, p


def _rt_gravity():
    from schemi_b200 import cases

    c, p = cases.rayleigh_taylor_2d(nx=8, ny=16, modes=2)
    c.g_delta = (0.0, -0.05, 0.0)
    c.diffusion, c.mu, c.D, c.kappa = True, 1e-3, 1e-3, 1e-3
    c.enthalpy_flow, c.molmass_diffusion = "explicit", True
    return c, p


def _kh_periodic():
    """A periodic axis (no reference counterpart; the oracle's periodic faces) with diffusion."""
    from schemi_b200 import cases

    c, p = cases.kelvin_helmholtz_2d(n=24)
    c.diffusion, c.mu, c.D, c.kappa = True, 1e-4, 1e-4, 1e-4
    c.enthalpy_flow, c.molmass_diffusion, c.diffusion_timestep = "explicit", True, True
    c.reconstruction = "linear"
    return c, p


def _hard_spheres(make, molmass=None):
    """The same case with the hard-sphere model (kinetic diameters; the constants added)."""
    def f():
        c, p = make()
        c.transport = "hardSpheres"
        for sp, d in zip(c.species, (1.0, 1.3, 0.9, 1.1)):
            sp.diameter = d * (3.6 if c.R_units == "SI" else 1.0)
        if molmass is not None:
            c.molmass_diffusion = molmass
        return c, p
    return f


def _lennard_jones(make, molmass=None):
    def f():
        c, p = make()
        c.transport = "LennardJones"
        si = c.R_units == "SI"
        for sp, e, sg in zip(c.species, (0.8, 1.1, 0.95), (1.0, 1.2, 1.1)):
            sp.tr_eps, sp.tr_sigma = e * (100.0 if si else 1.0), sg * (3.6 if si else 1.0)
        if molmass is not None:
            c.molmass_diffusion = molmass
        return c, p
    return f


def _cl2_diffusion():
    """Cl2 dissociation after a Gauss-Seidel hard-sphere diffusion stage (the ClorumTest deck's
    transport data) on a hot, non-uniform mixture."""
    from schemi_b200 import cases

    c, p = cases.chlorine_dissociation_2d(n=4)
    c.diffusion, c.transport, c.sle_solver = True, "hardSpheres", "GaussSeidel"
    c.mu, c.D, c.kappa = 2e-8, 2e-8, 2e-5
    c.species[0].diameter, c.species[1].diameter = 3.2, 1.6
    c.enthalpy_flow, c.molmass_diffusion = "explicit", True
    return c, p


def _kh_periodic_plain():
    c, p = _kh_periodic()
    c.enthalpy_flow = "no"
    return c, p


def _gs(make, solver="GaussSeidel"):
    """The same case with an implicit solver (Gauss-Seidel unless named)."""
    def f():
        c, p = make()
        c.sle_solver = solver
        return c, p
    return f


CASES = [
    ("tube_enthalpy_molmass", lambda: _tube(), 25),
    ("tube_gs", _gs(lambda: _tube()), 25),
    ("tube_gs_plain", _gs(lambda: _tube(enthalpy_flow="no", molmass_diffusion=False, reconstruction="linear",
                                        diffusion_timestep=False)), 25),
    ("vdw3_2d_gs", _gs(lambda: _vdw_box(2)), 10),
    ("vdw3_3d_gs", _gs(lambda: _vdw_box(3)), 6),
    ("rt_gravity_gs", _gs(_rt_gravity), 12),
    ("tube_linear_plain", lambda: _tube(enthalpy_flow="no", molmass_diffusion=False, reconstruction="linear",
                                        diffusion_timestep=False), 25),
    ("vdw3_2d", lambda: _vdw_box(2), 10),
    ("vdw3_3d", lambda: _vdw_box(3), 8),
    ("rt_gravity", _rt_gravity, 14),
    ("kh_periodic", _kh_periodic, 12),
    # hard spheres: bitwise (sqrt and division only); the explicit solver without the molar-mass
    # correction (with it the reference's explicit enthalpy source cools a pure-species interface
    # cell within one 1e-15 s step)
    ("tube_hs", _hard_spheres(lambda: _tube(), molmass=False), 25),
    ("tube_hs_gs", _gs(_hard_spheres(lambda: _tube())), 25),
    ("vdw3_2d_hs_gs", _gs(_hard_spheres(lambda: _vdw_box(2), molmass=True)), 10),
    ("vdw3_3d_hs", _hard_spheres(lambda: _vdw_box(3)), 6),
    ("rt_gravity_hs_gs", _gs(_hard_spheres(_rt_gravity)), 10),
    ("kh_periodic_hs", _hard_spheres(lambda: _kh_periodic_plain(), molmass=False), 8),
    ("vdw3_3d_hs_gs_molmass", _gs(_hard_spheres(lambda: _vdw_box(3), molmass=True)), 6),
    # the other solvers of the stage's matrices: Jacobi, Thomas (1D), noSolver
    ("tube_jacobi", _gs(lambda: _tube(), "Jacobi"), 25),
    ("vdw3_2d_jacobi", _gs(lambda: _vdw_box(2), "Jacobi"), 10),
    ("vdw3_3d_jacobi", _gs(lambda: _vdw_box(3), "Jacobi"), 6),
    ("rt_gravity_jacobi", _gs(_rt_gravity, "Jacobi"), 10),
    ("tube_thomas", _gs(lambda: _tube(), "Thomas"), 25),
    ("tube_thomas_plain", _gs(lambda: _tube(enthalpy_flow="no", molmass_diffusion=False, reconstruction="linear",
                                            diffusion_timestep=False), "Thomas"), 25),
    ("tube_nosolver", _gs(lambda: _tube(), "noSolver"), 25),
    ("vdw3_2d_nosolver", _gs(lambda: _vdw_box(2), "noSolver"), 10),
    # the implicit enthalpy flow: the upwind term in the temperature matrix (explicit solver: the
    # temperature stays)
    ("tube_enth_implicit_gs", _gs(lambda: _tube(enthalpy_flow="implicit")), 25),
    ("tube_enth_implicit_jacobi", _gs(lambda: _tube(enthalpy_flow="implicit"), "Jacobi"), 25),
    ("tube_enth_implicit_thomas", _gs(lambda: _tube(enthalpy_flow="implicit"), "Thomas"), 25),
    ("tube_enth_implicit_explicit", lambda: _tube(enthalpy_flow="implicit"), 25),
    ("vdw3_2d_enth_implicit_gs", _gs(lambda: (lambda cp: (setattr(cp[0], "enthalpy_flow", "implicit"), cp)[1])(
        _vdw_box(2))), 10),
    ("vdw3_3d_enth_implicit_gs", _gs(lambda: (lambda cp: (setattr(cp[0], "enthalpy_flow", "implicit"), cp)[1])(
        _vdw_box(3))), 6),
]

# cases whose arithmetic calls pow / exp: (name, make, steps, relative tolerance).  Each is
# well conditioned: a one-ulp change of its input pressure moves its state by about 1e-15 after six
# steps.  The Gauss-Seidel stage with the molar-mass correction on the tube and boxes above is
# not: the same one-ulp change moves T by 1e-2 within three steps (the Maxwell-Stefan system's
# pivot and replaced row are chosen by comparisons of nearly equal values), so a last-bit
# difference of the collision integrals would grow to that size; those configurations are
# compared bit for bit with the hard-sphere model instead.
TOLERANT = [
    ("tube_lj_gs", _gs(_lennard_jones(lambda: _tube(), molmass=False)), 25, 1e-11),
    ("vdw3_2d_lj", _lennard_jones(lambda: _vdw_box(2)), 10, 1e-11),
    ("vdw3_3d_lj_gs", _gs(_lennard_jones(lambda: _vdw_box(3), molmass=False)), 6, 1e-11),
    ("cl2_4x4_diffusion_gs", _cl2_diffusion, 12, 1e-11),
    # the conjugate-gradient solvers: block sums for the reference's serial dot products
    ("tube_cg", _gs(lambda: _tube(molmass_diffusion=False), "conjugateGradient"), 20, 1e-10),
    ("tube_bicg", _gs(lambda: _tube(molmass_diffusion=False), "biConjugateGradient"), 20, 1e-10),
    ("vdw3_2d_jcg", _gs(lambda: _vdw_box(2), "JacobiConjugateGradient"), 8, 1e-10),
    ("vdw3_2d_bicg", _gs(lambda: _vdw_box(2), "biConjugateGradient"), 8, 1e-10),
    ("vdw3_3d_cg", _gs(lambda: _vdw_box(3), "conjugateGradient"), 5, 1e-10),
]


@pytest.mark.parametrize("name,make,steps", CASES, ids=[c[0] for c in CASES])
def test_gpu_diffusion_step_matches_oracle_bitwise(fv, oracle_mod, name, make, steps):
    case, prim = make()
    g = fv.FVCase(case)
    g.upload(prim)
    assert g.path == fv.PATH_GENERIC
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    for s in range(steps):
        g.step()
        oc.step()
        assert g.time() == oc.time(), f"{name} step {s + 1}: clock {g.time()} vs {oc.time()}"
        assert g.source_timestep() == oc.source_timestep(), f"{name} step {s + 1}: source time step"
    a, b = g.download(), oc.download()
    for f in FIELDS:
        if f in a and f in b:
            bad = np.flatnonzero(a[f] != b[f])
            assert bad.size == 0, f"{name} {f}: {bad.size} cells differ, first {bad[0]}: {a[f][bad[0]]!r} vs {b[f][bad[0]]!r}"


@pytest.mark.parametrize("name,make,steps,tol", TOLERANT, ids=[c[0] for c in TOLERANT])
def test_gpu_diffusion_step_matches_oracle_within_tolerance(fv, oracle_mod, name, make, steps, tol):
    """Per field, the largest difference over the field's largest magnitude (velocities over the
    flow's speed scale sqrt(p / rho), as a mixture at rest starts to move at rounding level)."""
    case, prim = make()
    g = fv.FVCase(case)
    g.upload(prim)
    assert g.path == fv.PATH_GENERIC
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    for s in range(steps):
        g.step()
        oc.step()
        tg, dg = g.time()
        to, do = oc.time()
        assert tg == pytest.approx(to, rel=tol) and dg == pytest.approx(do, rel=tol), f"{name} step {s + 1}"
    a, b = g.download(), oc.download()
    vscale = float(np.sqrt(np.max(b["p"]) / np.min(b["rho"])))
    for f in FIELDS:
        if f in a and f in b:
            scale = max(float(np.abs(b[f]).max()), vscale if f in ("vx", "vy", "vz") else 0.0, 1e-300)
            err = float(np.abs(np.asarray(a[f]) - np.asarray(b[f])).max()) / scale
            assert err <= tol, f"{name} {f}: relative difference {err:.3e}"


def test_gpu_diffusion_run_matches_oracle(fv, oracle_mod):
    """fv_run (CUDA graphs of step chunks) with the stage: the same state and step count."""
    case, prim = _tube()
    g = fv.FVCase(case)
    g.upload(prim)
    st = g.run(0.02)
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    t, n = oc.run(0.02, 10**6)
    assert st.steps == n and st.time == t
    a, b = g.download(), oc.download()
    for f in FIELDS:
        if f in a and f in b:
            assert np.array_equal(a[f], b[f]), f


def test_gpu_diffusion_kernel_count(fv):
    case, prim = _tube()
    g = fv.FVCase(case)
    assert g.kernels_per_step == 4 + 5  # the generic step's 4, the stage's 4, the finalize
    case.sle_solver = "GaussSeidel"
    g = fv.FVCase(case)
    # step 4; prim, faces, matrices, 2 solves, concentrations, averaged enthalpy flow, matrices,
    # 1 + 1 solves (1D: one momentum component), phase, source, finalize
    assert g.kernels_per_step == 4 + 2 + 1 + 2 + 1 + 1 + 1 + 2 + 1 + 1 + 1
    # a chemical mechanism after the stage: one more kernel before the finalize
    case, _ = _cl2_diffusion()
    g = fv.FVCase(case)
    assert g.kernels_per_step == 4 + 2 + 1 + 2 + 1 + 1 + 1 + 3 + 1 + 1 + 1 + 1
    # noSolver: the implicit branch without its 1 + 1 + 1 solves
    case, _ = _gs(lambda: _tube(), "noSolver")()
    assert fv.FVCase(case).kernels_per_step == 4 + 2 + 1 + 1 + 1 + 1 + 1 + 1 + 1


def test_gpu_diffusion_refusals(fv):
    """Configurations outside the stage are refused at fv_create with initialisationError."""
    for kw in ({"precision": "f32flux"}, {"order": "SecondOrderRK"}, {"flux": "HLL"}):
        case, _ = _tube(**kw)
        with pytest.raises(fv.FVError) as e:
            fv.FVCase(case)
        assert e.value.status == 11, kw
    case, _ = _hard_spheres(lambda: _tube())()
    case.species[1].diameter = 0.0  # a hard sphere without a diameter
    with pytest.raises(fv.FVError) as e:
        fv.FVCase(case)
    assert e.value.status == 11
    for solver in ("GaussSeidel", "Jacobi", "noSolver"):  # the implicit branch without wrap-around
        case, _ = _kh_periodic()
        case.sle_solver = solver
        with pytest.raises(fv.FVError) as e:
            fv.FVCase(case)
        assert e.value.status == 11, solver
    case, _ = _vdw_box(2)
    case.sle_solver = "Thomas"  # 1D only
    with pytest.raises(fv.FVError) as e:
        fv.FVCase(case)
    assert e.value.status == 11
