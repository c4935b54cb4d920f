#!/usr/bin/env python
"""Benchmark of the B200 explicit finite-volume step (Schemi drop-in).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the 2D Kelvin-Helmholtz mixing layer on 1024 x 1024 cells (periodic in x, slip in y,
two ideal-gas species, HLLC + van Leer), seeded synthetic initial fields.  A "step" is one FV
step of the whole mesh: the fused reconstruction + Hancock + HLLC + update kernel and the CFL
reduction.  Conserved state is FP64; the headline arithmetic is FP64 (bit-exact with the
reference); the FP32-flux mode is reported beside it.

value     cell-updates/s, device time (CUDA events on the library's stream), L2 flushed
          between steps by writing a 256 MiB buffer on the same stream, max over ranks.
e2e       the same metric through the C-ABI with host buffers: fv_upload of the restart set
          from pinned memory + fv_run(K steps) + fv_download into pinned arrays, host wall
          clock (after one untimed pass of the same calls).
roofline  algorithmic bytes per cell-update = 2 * 8 * (N + 1 + D + 1) (conserved FP64 state read
          once and written once; N species densities, mixture density, D momenta, energy)
          over the measured HBM copy bandwidth of this pool (MEASURED_PEAKS.json).
cpu_baseline / --impl reference: the reference solver compiled from its own sources, with the
          per-face assignment at HancockStage.cpp:308,313,318 (oracle/_ref/schemi_patched,
          output byte-identical) as the value and the build as shipped (oracle/_ref/schemi)
          beside it, on the same KH workload at 128 x 128 cells (slip in x: the reference has no
          periodic patch), steps timed by differencing two runs.
accuracy  every section states its relative L1 / L-inf error against the FP64 oracle on the
          same inputs: KH 1024^2 after 3 steps (FP64 and FP32 flux), 16 sampled ensemble cases
          (the smallest, the largest and seeded others) after their ensemble steps, the reacting
          layer at 64^3 after 3 steps, the adjoint against the FP64 tangent oracle on 16 x 48;
          the oracle runs in spawned worker processes after the timed sections.
shock_tube_1d  config 1: the 1000-cell two-component tube to t = 0.2 through fv_run, us per step
          and the final fields against the reference's own output (tests/golden).
diffusion_deck  the reference's Diffusion_1000 deck (the diffusion stage after every advection,
          34,561 steps to t = 0.3) through fv_run: us per step, the final fields against the
          reference's output of that deck, and the reference binary's us per step on it.
gauss_seidel_deck  the same for the reference's PoiseuilleFlow_SI_100x100 deck (Gauss-Seidel
          diffusion of a van der Waals channel flow, 100 x 100) shortened to t = 2e-3.

batched   512 Richtmyer-Meshkov cases of seeded sizes 128^2..512^2 (FP32 flux) advanced by the
          persistent ensemble kernel, against the same cases one after the other.
reacting_3d  3D reacting shear layer 256^3 (A+B->2C, van der Waals, FP32 flux + FP64 chemistry):
          cell-updates/s of the whole step and the chemistry pass's share.
adjoint   Rayleigh-Taylor 512 x 1536 to t = 5 (64 seeded interface modes): gradient of the
          time-integrated mixing width through the hand-written adjoint (checkpoint every 50
          steps); backward (incl. recomputation) over forward device time, FP64 and FP32 flux,
          and a central finite difference (h = 1e-6) along a seeded direction.

Multi-GPU (torchrun): every rank advances its own replica of the single case (the single-case
step does not shard; "scaling": "weak"); the batched ensemble is sharded, its cases split over
the ranks by estimated work with no per-step exchange.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def profile_traffic(workload: str):
    """DRAM bytes per step kernel launch from the committed ncu summary (profiles/traffic.txt)."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith(workload + "="):
                    return float(line.split("=", 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(prefix="clocks_", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.out.close()

    def summary(self):
        sm, smax, reasons = [], None, set()
        try:
            with open(self.out.name) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) < 9:
                        continue
                    try:
                        sm.append(float(parts[1]))
                        smax = float(parts[2])
                    except ValueError:
                        continue
                    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
                    for name, val in zip(names, parts[5:9]):
                        if val.lower() == "active":
                            reasons.add(name)
        finally:
            try:
                os.unlink(self.out.name)
            except OSError:
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------- accuracy
# Every GPU result states its relative L1 and L-inf error against the FP64 oracle (the CPU
# restatement of the reference step, pinned bit for bit to the reference's outputs) on the same
# inputs.  Groups of conserved fields: each species density, the mixture density, the momentum
# vector (component errors summed over the components, on the scale of the vector's magnitude)
# and the total energy.
def conserved_errors(got: dict, want: dict, n_species: int) -> dict:
    import numpy as np

    groups = {f"rho{k + 1}": [f"rho{k + 1}"] for k in range(n_species)}
    groups["rho"] = ["rho"]
    groups["m"] = [f for f in ("mx", "my", "mz") if f in want and np.any(want[f])]
    groups["E"] = ["E"]
    out = {}
    for name, fields in groups.items():
        if not fields:
            continue
        diff = sum(np.abs(np.asarray(got[f]) - np.asarray(want[f])) for f in fields)
        mag = sum(np.abs(np.asarray(want[f])) for f in fields)
        out[name] = {"l1": float(diff.sum() / max(mag.sum(), 1e-300)),
                     "linf": float(diff.max() / max(mag.max(), 1e-300))}
    return {"l1": max(v["l1"] for v in out.values()), "linf": max(v["linf"] for v in out.values()),
            "fields": out}


def _oracle_state(case, prim, steps: int) -> dict:
    """Conserved fields of the FP64 oracle after `steps` steps from the restart set `prim`."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    oc = oracle.OracleCase(case)
    oc.upload(prim)
    for _ in range(steps):
        oc.step()
    d = oc.download()
    keep = [f"rho{k + 1}" for k in range(case.n_species)] + ["rho", "mx", "my", "mz", "E"]
    return {k: d[k] for k in keep}


def oracle_job(kind: str, arg: int, steps: int) -> dict:
    """One oracle run in a worker process (started with spawn before any CUDA call)."""
    from schemi_b200 import cases

    if kind == "kh":
        case, prim = cases.kelvin_helmholtz_2d(n=arg)
    elif kind == "rm":
        case, prim, _ = cases.richtmyer_meshkov(arg, precision="f64")
    elif kind == "reacting":
        case, prim = cases.reacting_shear_3d(n=arg, precision="f64")
    else:
        raise ValueError(kind)
    return _oracle_state(case, prim, steps)


def oracle_pool(workers: int):
    import concurrent.futures as cf
    import multiprocessing as mp

    return cf.ProcessPoolExecutor(max_workers=max(1, workers), mp_context=mp.get_context("spawn"))


def gpu_conserved(g) -> dict:
    d = g.download()
    keep = [f"rho{k + 1}" for k in range(g.case.n_species)] + ["rho", "mx", "my", "mz", "E"]
    return {k: d[k] for k in keep}


# ----------------------------------------------------------------------------- reference / CPU
def _reference_run(binary, case, prim, steps_target, workdir):
    """Run the reference binary to the time reached after `steps_target` steps; return wall s."""
    from schemi_b200.deck import write_deck

    os.makedirs(workdir, exist_ok=True)
    write_deck(case, workdir, prim, frequency_of_output=1 << 30, restart=True)
    t0 = time.perf_counter()
    r = subprocess.run([binary], cwd=workdir, stdin=subprocess.DEVNULL, stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL, timeout=1800)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"reference exited with {r.returncode}")
    return wall


def reference_throughput(n: int = 128, steps: int = 20, steps0: int = 2, processes: int = 1, patched: bool = True):
    """Cell-updates/s of the reference solver on KH n x n (slip x), by differencing a run of
    `steps` and a run of `steps0` steps (cancels start-up and file I/O); `processes` copies run
    concurrently and the aggregate rate is reported.  patched: the build with the per-face
    assignment at HancockStage.cpp:308,313,318 (oracle/_ref/schemi_patched, byte-identical
    output, without the O(faces^2) cost); else the build as shipped (oracle/_ref/schemi)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from schemi_b200 import cases

    binary = oracle.REF_BIN_PATCHED if patched else oracle.REF_BIN
    if not os.path.exists(binary):
        raise FileNotFoundError(binary)
    case, prim = cases.kelvin_helmholtz_2d(n=n, periodic=False)
    # the oracle reproduces the reference's time steps exactly: use it to find the end times
    oc = oracle.OracleCase(case)
    oc.upload(prim)
    t_at = {}
    for s in range(1, steps + 1):
        oc.step()
        t_at[s] = oc.time()[0]
    base = tempfile.mkdtemp(prefix="schemi_refbench_")
    import copy
    from concurrent.futures import ThreadPoolExecutor

    def one(idx, nst):
        c = copy.deepcopy(case)
        c.t_end = t_at[nst]
        return _reference_run(binary, c, prim, nst, os.path.join(base, f"p{idx}_{nst}"))

    with ThreadPoolExecutor(max_workers=processes) as ex:
        short = list(ex.map(lambda i: one(i, steps0), range(processes)))
    with ThreadPoolExecutor(max_workers=processes) as ex:
        long_ = list(ex.map(lambda i: one(i, steps), range(processes)))
    import shutil

    shutil.rmtree(base, ignore_errors=True)
    per = [(n * n * (steps - steps0)) / max(l - s, 1e-9) for l, s in zip(long_, short)]
    return sum(per), {"n": n, "steps": steps - steps0, "processes": processes,
                      "wall_long_s": statistics.mean(long_), "wall_short_s": statistics.mean(short)}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    procs = max(1, min(cores, 64))
    metric = "cell-updates/s per FV step"
    try:
        v, info = reference_throughput(n=128, steps=12, steps0=2, processes=procs, patched=True)
        v_shipped, info_s = reference_throughput(n=128, steps=12, steps0=2, processes=procs, patched=False)
    except Exception as e:  # the binaries are built here from the reference sources
        print(json.dumps({"impl": "reference", "unavailable": f"reference binary could not run: {e}"}))
        return 0
    sample = (f"{procs} concurrent processes of the reference binary with the per-face assignment at "
              f"HancockStage.cpp:308,313,318 (oracle/_ref/schemi_patched; output byte-identical to the build as "
              f"shipped), each the KH mixing layer at {info['n']}x{info['n']} with slip x (the reference has no "
              f"periodic patch), {info['steps']} steps timed by differencing runs of 12 and 2 steps")
    line = {
        "impl": "reference", "metric": metric, "value": v, "unit": "cell-updates/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "kelvin_helmholtz_2d", "cells": "128x128 sample of 1024x1024",
                   "flux": "HLLC", "limiter": "vanLeer", "species": 2},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": procs, "kind": "reference",
                         "sample": sample},
        "as_shipped": {"value": v_shipped, "unit": "cell-updates/s", "cores": procs,
                       "sample": "the same with the reference binary as shipped (oracle/_ref/schemi), whose "
                                 "per-step cost grows with the square of the face count"},
        "same_config": False,
        "config_note": "KH 128x128 sample with slip x: the reference cannot express the periodic x patch of the "
                       "1024x1024 workload; rates are per cell-update",
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ----------------------------------------------------------------------------- GPU arm
def time_steps(g, torch, steps, warmup, flush, load_seconds=1.0):
    """Device time of `steps` steps, L2 flushed before each, CUDA events on the handle's stream.

    Before the timed steps, untimed steps of the same kind keep the GPU under load for
    `load_seconds` so that the clock sampler sees the clocks of this load around the timed
    region (which can be a few milliseconds long)."""
    stream = torch.cuda.ExternalStream(g.stream_ptr)
    g.begin_steps()
    with torch.cuda.stream(stream):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(warmup):
            flush.add_(1)
            g.step_async()
        e1.record(stream)
    torch.cuda.synchronize()
    per = max(e0.elapsed_time(e1) / max(warmup, 1), 1e-3)
    n_load = int(min(200000, load_seconds * 1e3 / per))
    with torch.cuda.stream(stream):
        for _ in range(n_load):
            flush.add_(1)
            g.step_async()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for e0, e1 in ev:
            flush.add_(1)
            e0.record(stream)
            g.step_async()
            e1.record(stream)
    torch.cuda.synchronize()
    g.check()
    return [e0.elapsed_time(e1) for e0, e1 in ev]


def pinned_like(torch, arrays):
    """Page-locked host copies (numpy views) of `arrays`: the restart set a host hands to
    fv_upload, or the output arrays fv_download fills (name -> array)."""
    def one(a):
        t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
        v = t.numpy()
        v[:] = a
        return v

    if isinstance(arrays, dict):
        return {k: one(a) for k, a in arrays.items()}
    return [one(a) for a in arrays]


def e2e_run(g, prim_pinned, out_pinned, steps):
    """Public-API run with host buffers: fv_upload of the restart set from pinned memory +
    fv_run + fv_download into pinned output arrays, wall clock."""
    t0 = time.perf_counter()
    g.upload(prim_pinned)
    st = g.run(math.inf, max_steps=steps)
    g.download(out_pinned)
    wall = time.perf_counter() - t0
    ncell = g.n_cells
    h2d = len(prim_pinned) * 8 * ncell
    d2h = len(out_pinned) * 8 * ncell  # every field fv_download writes for the case
    return wall, st, h2d, d2h


BATCH_WARMUP_STEPS = 16


def batch_accuracy_sample(n_cases: int, count: int = 16):
    """Cases of the ensemble checked against the oracle: the smallest, the largest and seeded
    others (up to `count`)."""
    import numpy as np

    from schemi_b200 import cases

    sizes = [cases.richtmyer_meshkov_draws(i)[0] for i in range(n_cases)]
    pick = [int(np.argmin(sizes)), int(np.argmax(sizes))]
    rng = np.random.default_rng(4242)
    for i in rng.permutation(n_cases):
        if len(pick) >= min(count, n_cases):
            break
        if int(i) not in pick:
            pick.append(int(i))
    return sorted(pick)


def batch_accuracy(kept: dict, fut: dict, steps: int) -> dict:
    """Relative errors of the sampled ensemble cases against the oracle's states."""
    worst = {"l1": 0.0, "linf": 0.0}
    per_case = {}
    for i, k in sorted(kept.items()):
        e = conserved_errors(k["state"], fut[("rm", i)].result(), k["n_species"])
        per_case[str(i)] = {"cells": k["cells"], "l1": e["l1"], "linf": e["linf"]}
        worst = {q: max(worst[q], e[q]) for q in worst}
    return {"against": f"FP64 oracle, same restart sets, same step count ({BATCH_WARMUP_STEPS} + {steps} "
                       f"ensemble steps)", "cases_checked": len(per_case), "max_rel_l1": worst["l1"],
            "max_rel_linf": worst["linf"], "tolerance_rel_l1": 1e-5, "per_case": per_case}


def batched_vs_plain(n_cases: int, steps: int, torch, rank: int = 0, world: int = 1, dist=None, keep=(), kept=None):
    """Config-4 shape: `n_cases` Richtmyer-Meshkov cases of seeded sizes 128^2..512^2 (FP32 flux,
    HLLC + superbee, own end times), advanced `steps` ensemble steps by the batched persistent
    kernel, against the same cases advanced one after the other by the single-case path.  With
    several ranks the cases are sharded by estimated work (schemi_b200.ensemble, no per-step
    exchange); totals are summed and device times maxed over the ranks.  keep: case indices
    whose conserved fields (and step counts) are stored into `kept` after the run, for the
    comparison with the oracle."""
    from schemi_b200 import cases, ensemble, fv

    draws = [cases.richtmyer_meshkov_draws(i) for i in range(n_cases)]
    # work ~ cells x steps; steps ~ t_end / dt with dt ~ 0.5 / (n * 2.5) (post-shock signal speed)
    ws = 1.2 * math.sqrt(1.4)
    work = [ensemble.case_work(n * n, tr / ws, 0.5 / (n * 2.5)) for n, _, _, tr in draws]
    shares = ensemble.partition(work, world)
    mine = shares[rank]
    handles, t_end, cells, prims = [], [], 0, []
    for i in mine:
        case, prim, te = cases.richtmyer_meshkov(i, precision="f32flux")
        g = fv.FVCase(case)
        g.set_march_shape(64, 1, 32)  # best of a sweep of ensemble tile shapes on B200
        g.upload(prim)
        handles.append(g)
        t_end.append(te)
        prims.append(prim)
        cells += case.n_cells
    torch.cuda.synchronize()
    # plain: each case on its own, `steps` steps through fv_run (device time per case)
    plain_ms = 0.0
    plain_updates = 0
    for g, te in zip(handles, t_end):
        st = g.run(te, max_steps=steps)
        plain_ms += st.device_ms
        plain_updates += st.steps * g.n_cells
    # the ensemble starts again from the restart sets, so that every case has taken exactly
    # BATCH_WARMUP_STEPS + steps ensemble steps at the end (the oracle's step count)
    for g, prim in zip(handles, prims):
        g.upload(prim)
    batch = fv.FVBatch(handles)
    batch.run(t_end, max_steps=BATCH_WARMUP_STEPS)  # warm-up (graph capture, kernel configuration)
    if dist is not None and world > 1:
        dist.barrier()
    st = batch.run(t_end, max_steps=steps)
    totals = ensemble.combine_rank_totals(
        dist if world > 1 else None, "cuda",
        sums={"updates": float(st.cell_updates), "plain_updates": float(plain_updates), "cells": float(cells)},
        maxes={"ms": float(st.device_ms), "plain_ms": plain_ms})
    updates, plain_updates, cells = totals["updates"], totals["plain_updates"], int(totals["cells"])
    ms, plain_ms = totals["ms"], totals["plain_ms"]
    if kept is not None:
        for i, g in zip(mine, handles):
            if i in keep:
                kept[i] = {"cells": g.n_cells, "steps": BATCH_WARMUP_STEPS + steps, "state": gpu_conserved(g),
                           "n_species": g.case.n_species}
    out = {
        "cases": n_cases, "cells": cells, "steps": steps, "arith": "f32flux",
        "value": updates / (ms / 1e3), "unit": "cell-updates/s",
        "ms_per_ensemble_step": ms / steps,
        "plain_value": plain_updates / (plain_ms / 1e3),
        "launches_per_ensemble_step": st.launches / max(st.steps_max, 1),
        "bytes_per_cell_update": 2 * 8 * (2 + 1 + 2 + 1),
        "sharding": {"ranks": world, "cases_per_rank": [len(x) for x in shares],
                     "estimated_imbalance": ensemble.imbalance(work, shares)},
    }
    out["batched_over_plain"] = out["value"] / out["plain_value"]
    batch.close()
    for g in handles:
        g.close()
    return out


def reacting_3d(torch, peak, n: int, steps: int, warmup: int, flush, autotune_shapes: bool):
    """Config-3 shape: 3D reacting shear layer n^3 (van der Waals mixture of A, B, C; A+B->2C with
    the FP64 chemistry pass; FP32 flux), periodic x and z, slip y.  Device time per step of the
    whole step (fused march + chemistry + CFL), and of the same case without chemistry, so that the
    chemistry pass's share is the difference."""
    import copy

    from schemi_b200 import cases, fv

    case, prim = cases.reacting_shear_3d(n=n, precision="f32flux")
    out = {"workload": f"reacting_shear_3d {n}^3, A+B->2C, vdW, f32flux step + FP64 chemistry",
           "cells": case.n_cells}
    results = {}
    for label, c in (("with_chemistry", case), ("flow_only", None)):
        if c is None:
            c = copy.deepcopy(case)
            c.chemistry = "no"
        g = fv.FVCase(c)
        g.upload(prim)
        shape = None
        if autotune_shapes:
            from schemi_b200 import autotune

            shape = autotune.tune(g)
            g.upload(prim)
        torch.cuda.synchronize()
        with ClockSampler(torch.cuda.current_device()) as cs:
            ms = time_steps(g, torch, steps, warmup, flush)
        results[label] = {"ms_per_step": sum(ms) / steps, "kernels_per_step": g.kernels_per_step,
                          "march_shape": list(shape) if shape else None, "clocks": cs.summary()}
        g.close()
    w, f = results["with_chemistry"], results["flow_only"]
    ncell = case.n_cells
    step_bytes = 2 * 8 * (case.n_species + 1 + case.dims + 1)   # conserved state read + written
    chem_bytes = 8 * (case.n_species + 1 + 3 + 1) + 8 * (case.n_species + 1)  # read state, write rho_k, E
    out.update({
        "value": ncell / (w["ms_per_step"] / 1e3), "unit": "cell-updates/s", "ms_per_step": w["ms_per_step"],
        "flow_only_value": ncell / (f["ms_per_step"] / 1e3), "flow_only_ms_per_step": f["ms_per_step"],
        "chemistry_ms_per_step": w["ms_per_step"] - f["ms_per_step"],
        "chemistry_share": (w["ms_per_step"] - f["ms_per_step"]) / w["ms_per_step"],
        "kernels_per_step": w["kernels_per_step"], "march_shape": w["march_shape"], "clocks": w["clocks"],
        "roofline": {"bound": "hbm", "bytes_per_cell_update": step_bytes + chem_bytes,
                     "achieved": ncell * (step_bytes + chem_bytes) / (w["ms_per_step"] / 1e3) / 1e9, "peak": peak,
                     "unit": "GB/s"},
    })
    out["roofline"]["frac"] = out["roofline"]["achieved"] / peak
    return out


def adjoint_rt(torch, peak, t_end: float, autotune_shapes: bool):
    """Config-5 shape: Rayleigh-Taylor 512x1536 (64 seeded interface modes) to t_end; gradient of
    the time-integrated mixing width with respect to the mode amplitudes through the hand-written
    adjoint, checkpoint every 50 steps.  Per arithmetic: the plain forward (fv_run), the recorded
    forward (fv_record) and the backward sweep incl. recomputation (fv_adjoint), device-timed;
    FP64 also a central finite difference (h = 1e-6) along a seeded direction with the recorded
    step sizes (fv_replay)."""
    import numpy as np

    from schemi_b200 import adjoint, cases, fv

    nx, ny = 512, 1536
    a0 = torch.from_numpy(np.random.default_rng(2029).normal(0.0, 1e-3, size=64)).cuda()
    out = {"workload": f"rayleigh_taylor_2d {nx}x{ny} to t={t_end}, 64 modes, checkpoint every 50",
           "objective": "J = sum_n dt W(U^n), W = 4/Lx * integral X_h (1 - X_h) dA"}
    grads = {}
    for prec in ("f64", "f32flux"):
        case, _ = cases.rayleigh_taylor_2d(nx, ny, precision=prec, t_end=t_end)
        g = fv.FVCase(case)
        prim = adjoint.rayleigh_taylor_primitive(a0, nx, ny).contiguous()
        torch.cuda.synchronize()
        ptrs = [prim[i].data_ptr() for i in range(6)]
        g.upload_device(ptrs)
        shape = None
        if autotune_shapes:
            from schemi_b200 import autotune

            shape = autotune.tune(g)
        g.upload_device(ptrs)
        fwd = g.run(t_end)
        g.upload_device(ptrs)
        rec = g.record(t_end, 50)
        lam = torch.empty((case.n_conserved, case.n_cells), dtype=torch.float64, device="cuda")
        bwd = g.adjoint(None, 1.0, lam.data_ptr())
        # dJ/da through the restart-set conversion and the interface map (torch autograd)
        a = a0.clone().requires_grad_(True)
        U0 = adjoint.conserved_from_primitive(adjoint.rayleigh_taylor_primitive(a, nx, ny), case)
        (U0 * lam).sum().backward()
        grads[prec] = a.grad.detach().clone()
        kernel_ms = bwd.device_ms - bwd.recompute_ms
        nl = case.n_species + 2 + 2  # packed adjoint fields of a 2D case without transverse momentum
        kernel_bytes = 3 * nl * 8 * case.n_cells  # read U^n and lambda^{n+1}, write lambda^n
        gbs = kernel_bytes * bwd.steps / (kernel_ms / 1e3) / 1e9
        res = {
            "steps": rec.steps, "J": rec.objective, "march_shape": list(shape) if shape else None,
            "forward_ms": fwd.device_ms, "record_ms": rec.device_ms, "backward_ms": bwd.device_ms,
            "recompute_ms": bwd.recompute_ms, "adjoint_kernel_us_per_step": 1e3 * kernel_ms / bwd.steps,
            "backward_over_forward": bwd.device_ms / fwd.device_ms,
            "backward_over_record": bwd.device_ms / rec.device_ms,
            "adjoint_kernel_roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                        "frac": gbs / peak, "bytes_per_cell_step": 3 * nl * 8},
            "grad_norm": float(grads[prec].norm()),
        }
        if prec == "f64":
            d = torch.from_numpy(np.random.default_rng(77).normal(size=64)).cuda()
            d /= d.norm()
            h = 1e-6
            Js = []
            for s in (1.0, -1.0):
                p = adjoint.rayleigh_taylor_primitive(a0 + s * h * d, nx, ny).contiguous()
                torch.cuda.synchronize()
                g.upload_device([p[i].data_ptr() for i in range(6)])
                Js.append(g.replay().objective)
            fd = (Js[0] - Js[1]) / (2 * h)
            ad = float(grads[prec] @ d)
            res["fd_check"] = {"h": h, "direction": "seeded unit vector (seed 77)", "fd": fd, "adjoint": ad,
                               "rel_err": abs(ad - fd) / abs(fd)}
        out[prec] = res
        g.close()
    out["grad_rel_diff_f32flux_vs_f64"] = float((grads["f32flux"] - grads["f64"]).norm() / grads["f64"].norm())
    return out


ACC_STEPS = 3  # steps of the single-case accuracy checks (KH 1024^2, the 3D reacting layer)


def kh_accuracy(n: int, prec: str, want) -> dict:
    """KH n x n in `prec` arithmetic, ACC_STEPS steps through fv_step from the restart set,
    against the FP64 oracle's state after the same steps (want: a future of oracle_job)."""
    from schemi_b200 import cases, fv

    case, prim = cases.kelvin_helmholtz_2d(n=n, precision=prec)
    g = fv.FVCase(case)
    g.upload(prim)
    for _ in range(ACC_STEPS):
        g.step()
    got = gpu_conserved(g)
    g.close()
    e = conserved_errors(got, want.result(), case.n_species)
    return {"against": f"FP64 oracle, same restart set, {ACC_STEPS} steps", "rel_l1": e["l1"], "rel_linf": e["linf"],
            "tolerance": {"rel_linf": 1e-12} if prec == "f64" else {"rel_l1": 1e-5}, "fields": e["fields"]}


def tube_c1(torch) -> dict:
    """Config 1: the 1000-cell two-component shock tube (FP64, HLLC + minmod, CFL 0.5,
    transmissive ends) run to t = 0.2 through fv_run (the device time loop in CUDA graphs):
    microseconds per step, and the final fields against the reference solver's own output
    (tests/golden/shock_tube_1d_full.npz, written by the reference binary)."""
    import numpy as np

    from schemi_b200 import cases, fv

    case, prim = cases.shock_tube_1d()
    g = fv.FVCase(case)
    g.upload(prim)
    g.run(case.t_end)  # warm-up: graph capture and kernel configuration
    g.upload(prim)
    t0 = time.perf_counter()
    st = g.run(case.t_end)
    wall = time.perf_counter() - t0
    out = g.download()
    g.close()
    ref = np.load(os.path.join(ROOT, "tests", "golden", "shock_tube_1d_full.npz"))
    last = int(ref["n_steps"])
    errs = {}
    for f in ("c1", "c2", "vx", "p", "rho", "E"):
        key = f"{f}_{last}"
        if key in ref.files:
            b = ref[key]
            errs[f] = float(np.abs(out[f] - b).max() / max(np.abs(b).max(), 1e-300))
    return {"workload": "shock_tube_1d 1000 cells to t=0.2, FP64, HLLC + minmod", "steps": int(st.steps),
            "reference_steps": last, "device_us_per_step": 1e3 * st.device_ms / max(st.steps, 1),
            "wall_us_per_step": 1e6 * wall / max(st.steps, 1), "time": st.time,
            "rel_linf_vs_reference_output": max(errs.values()) if errs else None, "fields": errs,
            "tolerance_rel_linf": 1e-12}


def _deck_section(torch, case, prim, fixture: str, workload: str, ref_steps: int, ref_steps0: int) -> dict:
    """A restated deck of the reference through fv_run: microseconds per step on the device, the
    final fields against the reference's own output of that deck (tests/golden/<fixture>), and
    cpu_baseline: the reference binary (patched build) on the same deck, per step by differencing
    runs of ref_steps and ref_steps0 steps (the oracle finds their end times)."""
    import numpy as np

    from schemi_b200 import fv

    g = fv.FVCase(case)
    g.upload(prim)
    g.run(case.t_end, 20)  # warm-up: graph capture and kernel configuration
    g.upload(prim)
    t0 = time.perf_counter()
    st = g.run(case.t_end)
    wall = time.perf_counter() - t0
    out = g.download()
    kernels = g.kernels_per_step
    g.close()
    z = np.load(os.path.join(ROOT, "tests", "golden", fixture))
    txt = z["out:result|output_000001.tsv"].tobytes().decode().strip().split("\n")
    head = txt[0].split("\t")
    rows = np.array([[float(x) for x in ln.split("\t")] for ln in txt[1:]])
    errs = {}
    for f, col in (("c1", "concentration_1"), ("c2", "concentration_2"), ("vx", "velocity_x"),
                   ("vy", "velocity_y"), ("p", "pressure"), ("T", "temperature")):
        if f in out and col in head:
            b = rows[:, head.index(col)]
            errs[f] = float(np.abs(out[f] - b).max() / max(np.abs(b).max(), 1e-300))
    res = {"workload": workload, "steps": int(st.steps), "time": st.time,
           "device_us_per_step": 1e3 * st.device_ms / max(st.steps, 1),
           "wall_us_per_step": 1e6 * wall / max(st.steps, 1), "kernels_per_step": kernels,
           "rel_linf_vs_reference_output": max(errs.values()), "fields": errs, "tolerance_rel_linf": 1e-12}
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle

        oc = oracle.OracleCase(case)
        oc.upload(prim)
        t_at = {}
        for s in range(1, ref_steps + 1):
            oc.step()
            t_at[s] = oc.time()[0]
        import copy

        base = tempfile.mkdtemp(prefix="schemi_refdiff_")
        walls = {}
        for nst in (ref_steps0, ref_steps):
            c = copy.deepcopy(case)
            c.t_end = t_at[nst]
            walls[nst] = _reference_run(oracle.REF_BIN_PATCHED, c, prim, nst, os.path.join(base, str(nst)))
        import shutil

        shutil.rmtree(base, ignore_errors=True)
        us = 1e6 * (walls[ref_steps] - walls[ref_steps0]) / (ref_steps - ref_steps0)
        res["cpu_baseline"] = {"value": us, "unit": "us/step", "cores": 1, "kind": "reference",
                               "sample": f"oracle/_ref/schemi_patched on the same deck, steps {ref_steps0}..{ref_steps} "
                                         "by differencing two runs"}
        res["speedup_device_vs_reference"] = us / res["device_us_per_step"]
    except Exception as e:  # noqa: BLE001 -- the reference build may be absent
        res["cpu_baseline"] = {"unavailable": str(e)}
    return res


def diffusion_deck(torch, ref_steps: int = 300, ref_steps0: int = 20) -> dict:
    """The reference's Diffusion_1000 deck (1000 cells, the diffusion stage with the explicit
    solver after every advection, 34,561 steps to t = 0.3)."""
    from schemi_b200 import cases

    case, prim = cases.diffusion_tube_1d()
    return _deck_section(torch, case, prim, "deck_diffusion_1000.npz",
                         "diffusion_tube_1d (the reference's Diffusion_1000 deck) to t=0.3, FP64, HLLC + vanAlbada, "
                         "explicit diffusion with the molar-mass correction and the explicit enthalpy flow",
                         ref_steps, ref_steps0)


def gauss_seidel_deck(torch, ref_steps: int = 60, ref_steps0: int = 10) -> dict:
    """The reference's PoiseuilleFlow_SI_100x100 deck (van der Waals channel flow, 100 x 100, the
    diffusion stage with the Gauss-Seidel solver after every advection) shortened to t = 2e-3
    (309 steps)."""
    from schemi_b200 import cases

    case, prim = cases.poiseuille_2d()
    return _deck_section(torch, case, prim, "deck_poiseuille_100x100_short.npz",
                         "poiseuille_2d (the reference's PoiseuilleFlow_SI_100x100 deck) to t=2e-3, FP64, HLLC + "
                         "vanAlbada, van der Waals, Gauss-Seidel diffusion with the molar-mass correction and the "
                         "explicit enthalpy flow", ref_steps, ref_steps0)


def reacting_accuracy(n: int, want) -> dict:
    """The 3D reacting shear layer at n^3 (FP32 flux + FP64 chemistry), ACC_STEPS steps, against
    the FP64 oracle (flux, van der Waals EOS and the A+B->2C chemistry in FP64)."""
    from schemi_b200 import cases, fv

    case, prim = cases.reacting_shear_3d(n=n, precision="f32flux")
    g = fv.FVCase(case)
    g.upload(prim)
    for _ in range(ACC_STEPS):
        g.step()
    got = gpu_conserved(g)
    g.close()
    e = conserved_errors(got, want.result(), case.n_species)
    return {"against": f"FP64 oracle at {n}^3, same restart set, {ACC_STEPS} steps", "rel_l1": e["l1"],
            "rel_linf": e["linf"], "tolerance": {"rel_l1": 1e-5}, "fields": e["fields"]}


def adjoint_tangent_gap(torch, nx: int = 16, ny: int = 48, t_end: float = 0.5) -> dict:
    """Gradient of the adjoint against the FP64 CPU tangent oracle (forward-mode derivatives of an
    independent restatement of the same step) on a reduced Rayleigh-Taylor grid, along seeded
    directions: the largest gap on the scale of |grad| |d|."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import fv_tangent
    from schemi_b200 import adjoint, cases, fv

    case, _ = cases.rayleigh_taylor_2d(nx, ny, precision="f64", t_end=t_end)
    a = torch.from_numpy(np.random.default_rng(2029).normal(0.0, 1e-3, size=64))
    g = fv.FVCase(case)
    ad = a.clone().cuda().requires_grad_(True)
    J, _ = adjoint.TimeLoop.apply(adjoint.rayleigh_taylor_primitive(ad, nx, ny), g, t_end, 10, 0)
    J.backward()
    grad = ad.grad.detach().cpu()
    g.close()
    tc = fv_tangent.TangentCase(case)

    def U0(x):
        return tc.conserved_from_primitive(list(adjoint.rayleigh_taylor_primitive(x, nx, ny).reshape(6, ny, nx)))

    dts = tc.schedule(U0(a), t_end)
    f = lambda x: tc.objective(U0(x), dts, 0)  # noqa: E731
    rng = np.random.default_rng(11)
    worst = 0.0
    for _ in range(3):
        d = torch.from_numpy(rng.normal(size=64))
        _, dJ = fv_tangent.tangent(f, a, d)
        worst = max(worst, abs(float(grad @ d) - float(dJ)) / (float(grad.norm()) * float(d.norm())))
    return {"grid": f"{nx}x{ny} to t={t_end}", "directions": 3, "max_gap_over_grad_scale": worst,
            "tolerance": 1e-9}


def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    from schemi_b200 import cases
    from schemi_b200 import fv

    n = args.n
    peak, peak_kind = measured_peaks()
    flush = torch.zeros(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    results = {}
    for prec in ("f64", "f32flux"):
        case, prim = cases.kelvin_helmholtz_2d(n=n, precision=prec)
        g = fv.FVCase(case)
        g.upload(prim)
        if not args.no_autotune:
            from schemi_b200 import autotune

            shape = autotune.tune(g)   # cached per (mesh, species, EOS, precision, device)
            g.upload(prim)             # tuning advanced the state: start again from the restart set
        else:
            shape = None
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as cs:
            ms = time_steps(g, torch, args.steps, args.warmup, flush)
        clocks = cs.summary()
        total_ms = sum(ms)
        if world > 1:
            t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            total_ms = float(t.item())
        cells = case.n_cells
        nbytes = 2 * 8 * (case.n_species + 1 + case.dims + 1)
        value = world * cells * args.steps / (total_ms / 1e3)
        per_gpu = cells * args.steps / (total_ms / 1e3)
        achieved = per_gpu * nbytes / 1e9
        results[prec] = {
            "value": value, "ms_per_step": total_ms / args.steps, "clocks": clocks, "achieved_gbs": achieved,
            "bytes_per_cell_update": nbytes, "kernels_per_step": g.kernels_per_step, "path": g.path,
            "march_shape": list(shape) if shape else None,
        }
        # e2e through the C-ABI with pinned host buffers; one untimed pass first (the download's
        # device staging buffer is allocated on its first call)
        pinned = pinned_like(torch, prim)
        outs = pinned_like(torch, {name: np.zeros(g.n_cells) for name in g.download_fields()})
        e2e_run(g, pinned, outs, args.steps)
        wall, st, h2d, d2h = e2e_run(g, pinned, outs, args.steps)
        if world > 1:
            t = torch.tensor([wall], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            wall = float(t.item())
        results[prec]["e2e"] = {"value": world * cells * st.steps / wall, "unit": "cell-updates/s",
                                "h2d_bytes_per_step": h2d / max(st.steps, 1),
                                "d2h_bytes_per_step": (d2h + 96 * math.ceil(st.steps / 32)) / max(st.steps, 1)}
        g.close()

    head = results["f64"]
    line = {
        "metric": "cell-updates/s per FV step",
        "value": head["value"],
        "unit": "cell-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": head["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"kelvin_helmholtz_2d {n}x{n}", "cells_per_gpu": n * n, "species": 2,
                   "flux": "HLLC", "limiter": "vanLeer", "bc": "periodic x, slip y",
                   "l2": "flushed before every timed step (256 MiB write on the step stream)",
                   "parallelism": f"replicas x{world}", "march_shape_f64": head["march_shape"],
                   "march_shape_f32flux": results["f32flux"]["march_shape"]},
        "gpu_launches": head["kernels_per_step"] * args.steps,
        "e2e": head["e2e"],
        "clocks": head["clocks"],
        "roofline": {
            "bound": "hbm", "achieved": head["achieved_gbs"], "peak": peak, "unit": "GB/s",
            "frac": head["achieved_gbs"] / peak, "traffic": profile_traffic(f"kh{n}_f64"),
            "traffic_source": "ncu capture of the step kernel, summarised in profiles/traffic.txt",
            "peak_source": peak_kind, "bytes_per_cell_update": head["bytes_per_cell_update"],
        },
        "fp32_flux": {
            "value": results["f32flux"]["value"], "ms_per_step": results["f32flux"]["ms_per_step"],
            "e2e": results["f32flux"]["e2e"],
            "roofline": {"bound": "hbm", "achieved": results["f32flux"]["achieved_gbs"], "peak": peak,
                         "unit": "GB/s", "frac": results["f32flux"]["achieved_gbs"] / peak,
                         "traffic": profile_traffic(f"kh{n}_f32flux"),
                         "traffic_source": "ncu capture of the step kernel, summarised in profiles/traffic.txt"},
            "clocks": results["f32flux"]["clocks"],
        },
    }
    if rank == 0 and args.tube:
        line["shock_tube_1d"] = tube_c1(torch)
        line["diffusion_deck"] = diffusion_deck(torch)
        line["gauss_seidel_deck"] = gauss_seidel_deck(torch)
    sample = batch_accuracy_sample(args.batch_cases) if args.batch_cases > 0 and not args.no_accuracy else []
    kept = {}
    if args.batch_cases > 0:
        b = batched_vs_plain(args.batch_cases, args.steps, torch, rank, world, dist if world > 1 else None,
                             keep=sample, kept=kept)
        b["roofline_frac"] = b["value"] * b["bytes_per_cell_update"] / 1e9 / peak
        line["batched"] = b
    if args.reacting_n > 0:
        line["reacting_3d"] = reacting_3d(torch, peak, args.reacting_n, args.steps, args.warmup, flush,
                                          not args.no_autotune)
    if args.adjoint_t_end > 0 and rank == 0:
        line["adjoint"] = adjoint_rt(torch, peak, args.adjoint_t_end, not args.no_autotune)

    # ---- accuracy against the FP64 oracle, after every timed section (the oracle's worker
    # processes would otherwise share the host cores with the timed host-side work)
    pool = None
    if not args.no_accuracy:
        cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
        pool = oracle_pool(max(1, min(cores // max(world, 1), 24)))
        fut = {}
        # largest cases first: they take longest on the host
        for i in sorted(kept, key=lambda i: -kept[i]["cells"]):
            fut[("rm", i)] = pool.submit(oracle_job, "rm", i, kept[i]["steps"])
        if rank == 0:
            fut["kh"] = pool.submit(oracle_job, "kh", n, ACC_STEPS)
            if args.reacting_n > 0:
                fut["reacting"] = pool.submit(oracle_job, "reacting", args.reacting_acc_n, ACC_STEPS)
            line["accuracy"] = kh_accuracy(n, "f64", fut["kh"])
            line["fp32_flux"]["accuracy"] = kh_accuracy(n, "f32flux", fut["kh"])
            if args.reacting_n > 0:
                line["reacting_3d"]["accuracy"] = reacting_accuracy(args.reacting_acc_n, fut["reacting"])
            if args.adjoint_t_end > 0:
                line["adjoint"]["tangent_oracle"] = adjoint_tangent_gap(torch)
        if args.batch_cases > 0:
            acc = batch_accuracy(kept, fut, args.steps)
            if world > 1:
                # every rank checked its own sampled cases: the job's worst errors
                tot = ensemble_totals(dist, {"max_rel_l1": acc["max_rel_l1"], "max_rel_linf": acc["max_rel_linf"],
                                             "cases_checked": float(acc["cases_checked"])})
                acc.update({"max_rel_l1": tot["max_rel_l1"], "max_rel_linf": tot["max_rel_linf"],
                            "cases_checked": int(tot["cases_checked"]), "per_case": "rank 0 only"})
            line["batched"]["accuracy"] = acc
    if rank == 0 and not args.no_cpu_baseline:
        try:
            v, info = reference_throughput(n=128, steps=12, steps0=2, processes=1, patched=True)
            vs, _ = reference_throughput(n=128, steps=12, steps0=2, processes=1, patched=False)
            line["cpu_baseline"] = {
                "value": v, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                "sample": (f"reference binary with the per-face assignment at HancockStage.cpp:308,313,318 "
                           f"(oracle/_ref/schemi_patched, output byte-identical to the build as shipped), KH mixing "
                           f"layer {info['n']}x{info['n']} with slip x, {info['steps']} steps timed by differencing "
                           f"runs of 12 and 2 steps, one process"),
                "as_shipped": {"value": vs, "unit": "cell-updates/s", "cores": 1,
                               "sample": "the same with the build as shipped (oracle/_ref/schemi)"},
            }
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    if pool is not None:
        pool.shutdown(wait=True, cancel_futures=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def ensemble_totals(dist, worst: dict) -> dict:
    """Largest of per-rank figures over the ranks (the same collectives on every rank)."""
    from schemi_b200 import ensemble

    return ensemble.combine_rank_totals(dist, "cuda", sums={}, maxes=worst)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1024, help="cells per axis of the KH workload")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--batch-cases", type=int, default=512, help="cases of the batched ensemble (0: skip)")
    ap.add_argument("--reacting-n", type=int, default=256,
                    help="cells per axis of the 3D reacting shear layer workload (0: skip)")
    ap.add_argument("--adjoint-t-end", type=float, default=5.0,
                    help="end time of the Rayleigh-Taylor adjoint workload (0: skip)")
    ap.add_argument("--reacting-acc-n", type=int, default=64,
                    help="cells per axis of the reacting layer's accuracy check against the oracle")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the checks against the FP64 oracle")
    ap.add_argument("--no-tube", dest="tube", action="store_false", help="skip the 1000-cell shock tube section")
    ap.add_argument("--dry-run", action="store_true",
                    help="multi-rank plumbing only, on the CPU with gloo: launch, sharding, totals, JSON line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args.gpus)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE is {world}", file=sys.stderr)
        return 2
    if args.dry_run:
        return run_dry(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


def torchrun_command(n: int, argv) -> list:
    """The launch of this script as n ranks on one node (one process per GPU)."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
            "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__), *argv]


def launch_ranks(n: int) -> int:
    """`bench.py --gpus N` outside torchrun: start the N ranks itself and return their status."""
    return subprocess.run(torchrun_command(n, sys.argv[1:])).returncode


def run_dry(args) -> int:
    """The multi-rank plumbing of the GPU arm without a GPU: every rank takes its share of the
    ensemble (schemi_b200.ensemble), the totals are combined over gloo, and rank 0 prints the
    line's rank and sharding fields (no measurement)."""
    import torch.distributed as dist

    from schemi_b200 import cases, ensemble

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    ws = 1.2 * math.sqrt(1.4)
    draws = [cases.richtmyer_meshkov_draws(i) for i in range(args.batch_cases)]
    work = [ensemble.case_work(nn * nn, tr / ws, 0.5 / (nn * 2.5)) for nn, _, _, tr in draws]
    shares = ensemble.partition(work, world)
    cells = sum(draws[i][0] ** 2 for i in shares[rank])
    tot = ensemble.combine_rank_totals(dist if world > 1 else None, "cpu", sums={"cells": float(cells)},
                                       maxes={"rank": float(rank)})
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"dry_run": True, "n_gpus": world, "value": None,
                          "batched": {"cases": args.batch_cases, "cells": int(tot["cells"]),
                                      "sharding": {"ranks": world, "cases_per_rank": [len(x) for x in shares],
                                                   "estimated_imbalance": ensemble.imbalance(work, shares)}}}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
