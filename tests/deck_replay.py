"""Replays a task-deck fixture (``golden/deck_<name>.npz``) with a driver binary and compares the
files it writes with the reference solver's.

A fixture holds the task directory as the reference read it, the ``set/main.txt`` of every run
made in that directory and every file the reference left behind (``golden/make_deck_golden.py``).
``timeOfCalculation.tsv`` is compared without its measured milliseconds (the value after every
"Time of ..." label: the run's and each stage's wall time).  Fixtures with a
non-zero ``tolerance`` (the chemistry deck) are compared value by value to that relative
tolerance, velocities and momenta on the scale of the largest sonic speed (and density); all
others byte for byte.  A run the reference refused must end with the same exit code and with
the message the reference printed.
"""

import os
import re
import subprocess

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixtures():
    return sorted(f[5:-4] for f in os.listdir(GOLDEN) if f.startswith("deck_") and f.endswith(".npz"))


def load(name):
    return np.load(os.path.join(GOLDEN, f"deck_{name}.npz"))


def _write(d, rel, data):
    path = os.path.join(d, rel)
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "wb") as f:
        f.write(data)


def unpack_inputs(z, d):
    for k in z.files:
        if k.startswith("in:"):
            _write(d, k[3:].replace("|", os.sep), z[k].tobytes())


def _tree(d):
    found = {}
    for root, _, names in os.walk(d):
        for n in names:
            full = os.path.join(root, n)
            rel = os.path.relpath(full, d)
            if not rel.startswith("set" + os.sep):
                with open(full, "rb") as f:
                    found[rel] = f.read()
    return found


def _velocity_scale(want):
    """Largest sonic speed, density and total concentration of the reference's outputs:
    velocities and momenta are compared on the first two, since a flow at rest carries only
    rounding-level velocities, and species concentrations, densities and fractions on the
    mixture's, since a species that is nearly absent carries values far below any rounding of
    the mixture (1e-44 and less in the real-gas tubes)."""
    c_max, rho_max, conc_max = 0.0, 0.0, 0.0
    for rel, data in want.items():
        if os.path.basename(rel).startswith("output_") and rel.endswith(".tsv"):
            lines = data.decode().strip("\n").split("\n")
            head = lines[0].split("\t")
            rows = np.array([[float(x) for x in ln.split("\t")] for ln in lines[1:]])
            c_max = max(c_max, float(np.abs(rows[:, head.index("sonic_speed")]).max()))
            rho_max = max(rho_max, float(np.abs(rows[:, head.index("density")]).max()))
            conc_max = max(conc_max, float(np.abs(rows[:, head.index("concentration")]).max()))
    return c_max, rho_max, conc_max


def _numbers_close(a: bytes, b: bytes, tol: float, rel: str, scale):
    la, lb = a.decode().split("\n"), b.decode().split("\n")
    if len(la) != len(lb):
        return f"{rel}: {len(la)} lines, reference {len(lb)}"
    c_max, rho_max, conc_max = scale
    floors = {}
    if os.path.basename(rel) == "velocity.dat":
        floors = {0: c_max, 1: c_max, 2: c_max}
    elif os.path.basename(rel).startswith("sub_"):
        floors = {0: conc_max}
    elif rel.endswith(".tsv") and la:
        for j, name in enumerate(lb[0].split("\t")):
            if name.startswith("velocity_"):
                floors[j] = c_max
            elif name.startswith("momentum_"):
                floors[j] = c_max * rho_max
            elif name.startswith("concentration_"):
                floors[j] = conc_max
            elif name.startswith("density_"):
                floors[j] = rho_max
            elif name.startswith(("x_", "w_")):
                floors[j] = 1.0
    for i, (x, y) in enumerate(zip(la, lb)):
        tx, ty = x.split("\t"), y.split("\t")
        if len(tx) != len(ty):
            return f"{rel} line {i}: {len(tx)} columns, reference {len(ty)}"
        for j, (u, v) in enumerate(zip(tx, ty)):
            try:
                fu, fv = float(u), float(v)
            except ValueError:
                if u != v:
                    return f"{rel} line {i} column {j}: {u!r}, reference {v!r}"
                continue
            if abs(fu - fv) > tol * max(abs(fu), abs(fv), floors.get(j, 0.0), 1e-300):
                return f"{rel} line {i} column {j}: {u}, reference {v}"
    return None


def _first_difference(a: bytes, b: bytes, rel: str):
    la, lb = a.decode().split("\n"), b.decode().split("\n")
    for i in range(min(len(la), len(lb))):
        if la[i] != lb[i]:
            return f"{rel} line {i}:\n  got       {la[i][:300]}\n  reference {lb[i][:300]}"
    return f"{rel}: {len(la)} lines, reference {len(lb)}"


ORDER = re.compile(rb"(#Approximation_order\r?\n)(SecondOrder|SecondOrderRK|ThirdOrder|ThirdOrderCada)(\r?\n)")


def step_order(name):
    """The fixture's approximation order (its first run's set/main.txt)."""
    m = ORDER.search(load(name)["run0:main.txt"].tobytes())
    return m.group(2).decode() if m else None


def replay(driver, name, d, timeout=600, gpu=False, reference_main=False):
    """Runs every run of fixture ``name`` in directory ``d`` with ``driver``; returns a list of
    differences from the reference's files (empty when they agree).  ``gpu``: the driver runs the
    CUDA library, and a fixture's ``gpu_tolerance`` (the real-gas mixtures whose transcendental
    functions round differently on the device) replaces its ``tolerance``.  ``reference_main``:
    the driver is the reference's own main with the step-solver adapter registered (it reads
    ./set from its working directory); every run's approximation order X becomes "GpuX", the
    name under which the adapter runs the library's step."""
    z = load(name)
    unpack_inputs(z, d)
    problems = []
    for r in range(int(z["runs"])):
        main_txt = z[f"run{r}:main.txt"].tobytes()
        if reference_main:
            main_txt, n = ORDER.subn(rb"\1Gpu\2\3", main_txt)
            assert n == 1, f"{name}: no approximation order to redirect"
        _write(d, os.path.join("set", "main.txt"), main_txt)
        if reference_main:
            res = subprocess.run([driver], cwd=d, stdin=subprocess.DEVNULL, capture_output=True,
                                 text=True, timeout=timeout)
        else:
            res = subprocess.run([driver, d], capture_output=True, text=True, timeout=timeout)
        if res.returncode != int(z["rc"][r]):
            problems.append(f"run {r}: exit {res.returncode}, reference {int(z['rc'][r])}\n"
                            + res.stdout[-1500:] + res.stderr[-1500:])
            return problems
        if res.returncode != 0 and "log_tails" in z.files:
            # a refused deck: the driver's message is the one the reference printed
            said = [x for x in res.stderr.strip().split("\n") if x.strip()]
            if not said or said[-1].strip() not in str(z["log_tails"][r]):
                problems.append(f"run {r}: message {said[-1:]!r} not in the reference's output "
                                f"{str(z['log_tails'][r])[-300:]!r}")
    want = {k[4:].replace("|", os.sep): z[k].tobytes() for k in z.files if k.startswith("out:")}
    got = _tree(d)
    if sorted(got) != sorted(want):
        problems.append(f"files: extra {sorted(set(got) - set(want))}, missing {sorted(set(want) - set(got))}")
    tol = float(z["tolerance"])
    if gpu and "gpu_tolerance" in z.files:
        tol = float(z["gpu_tolerance"])
    scale = _velocity_scale(want) if tol > 0 else None
    for rel, data in sorted(want.items()):
        if rel not in got:
            continue
        if rel == "timeOfCalculation.tsv":
            def untimed(text):
                lines = text.split("\n")
                return [x for i, x in enumerate(lines) if not (i > 0 and lines[i - 1].startswith("Time of"))]

            g, w = untimed(got[rel].decode()), untimed(data.decode())
            if g != w:
                problems.append(f"{rel}: {g}, reference {w}")
        elif tol == 0:
            if got[rel] != data:
                problems.append(_first_difference(got[rel], data, rel))
        else:
            p = _numbers_close(got[rel], data, tol, rel, scale)
            if p:
                problems.append(p)
    return problems
