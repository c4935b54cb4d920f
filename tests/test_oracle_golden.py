"""The FP64 oracle against the reference solver's own outputs (golden fixtures).

Pins the CPU restatement: it must reproduce the reference bit for bit (the fixtures were
written with 20 significant digits, which round-trip doubles exactly).
"""

import numpy as np
import pytest

from golden_cases import golden_steps, load_cases, rel_err

CASES = load_cases()
COMPARE = ["c1", "c2", "c3", "vx", "vy", "p", "rho", "E", "mx", "my", "T"]


@pytest.mark.parametrize("name,case,prim,data", CASES, ids=[c[0] for c in CASES])
def test_oracle_matches_reference(oracle_mod, name, case, prim, data):
    steps = golden_steps(data)
    oc = oracle_mod.OracleCase(case)
    oc.upload(prim)
    t_end = float(data["t_end"])
    done = 0
    for target in steps:
        while done < target:
            oc.step()
            done += 1
            t, dt = oc.time()
            if t + dt > t_end:
                oc.set_time(t, t_end - t)
        t, _ = oc.time()
        assert t == float(data[f"time_{target}"])
        out = oc.download()
        for f in COMPARE:
            key = f"{f}_{target}"
            if key in data and f in out:
                linf, l1 = rel_err(out[f], data[key])
                assert linf == 0.0, f"{name} step {target} field {f}: rel Linf {linf:.3e}"
    assert done == int(data["n_steps"]) or "full" not in name


@pytest.mark.parametrize("limiter,fails_at", [("UTCDFS", 2), ("linear", 4)])
def test_oracle_riemann_failure_matches_reference(oracle_mod, limiter, fails_at):
    """On the 200-cell tube UTCDFS makes the HLLC wave speeds NaN at step 2 in the reference, and
    the unlimited linear reconstruction at step 4 (it prints "Fatal error in Riemann solver." and
    exits); the oracle reports RiemannSolverError at the same step."""
    from schemi_b200 import cases

    c, p = cases.shock_tube_1d(n=200)
    c.limiter = limiter
    oc = oracle_mod.OracleCase(c)
    oc.upload(p)
    for _ in range(fails_at - 1):
        oc.step()
    with pytest.raises(RuntimeError, match="status 1"):
        oc.step()


@pytest.mark.parametrize("limiter,fails_at", [("Koren", 1), ("vanAlbada", 1), ("HQUICK", 2)])
def test_oracle_third_order_riemann_failure_matches_reference(oracle_mod, limiter, fails_at):
    """ThirdOrder with these limiters on the slip-walled KH layer ends in the reference with
    "Fatal error in Riemann solver." at the listed step (20 cells: Koren, vanAlbada at the first
    step; 10 cells: HQUICK at the second); the oracle reports RiemannSolverError at the same step."""
    from schemi_b200 import cases

    c, p = cases.kelvin_helmholtz_2d(n=20 if fails_at == 1 else 10, periodic=False, limiter=limiter)
    c.order = "ThirdOrder"
    oc = oracle_mod.OracleCase(c)
    oc.upload(p)
    for _ in range(fails_at - 1):
        oc.step()
    with pytest.raises(RuntimeError, match="status 1"):
        oc.step()


def test_oracle_chemistry_jcg_failure_matches_reference(oracle_mod):
    """With the Jacobi-preconditioned CG solver the hot Cl2 case does not converge; the reference
    divides the first step (1e-15) by ten, finds it below the minimal time step, prints "Timestep
    become too small." and stops with systemError.  The oracle reports the same status."""
    from schemi_b200 import cases

    c, p = cases.chlorine_dissociation_2d(4, solver="JacobiConjugateGradient")
    oc = oracle_mod.OracleCase(c)
    oc.upload(p)
    with pytest.raises(RuntimeError, match="status 4"):
        oc.step()
