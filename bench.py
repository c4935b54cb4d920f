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
cpu_baseline / --impl reference: the reference solver compiled from its own sources
          (oracle/_ref/schemi, as shipped) on the same KH workload at 128 x 128 cells (slip in x:
          the reference has no periodic patch), steps timed by differencing two runs.

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


def reference_throughput(n: int = 128, steps: int = 20, steps0: int = 2, processes: int = 1):
    """Cell-updates/s of the as-shipped reference on KH n x n (slip x), by differencing a run of
    `steps` and a run of `steps0` steps (cancels start-up and file I/O); `processes` copies run
    concurrently and the aggregate rate is reported."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from schemi_b200 import cases

    binary = oracle.REF_BIN
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
        v, info = reference_throughput(n=128, steps=12, steps0=2, processes=procs)
    except Exception as e:  # the binary is built here from the reference sources
        print(json.dumps({"impl": "reference", "unavailable": f"reference binary could not run: {e}"}))
        return 0
    sample = (f"{procs} concurrent processes of the as-shipped reference binary (oracle/_ref/schemi), each the KH "
              f"mixing layer at {info['n']}x{info['n']} with slip x, {info['steps']} steps timed by differencing "
              f"runs of 12 and 2 steps")
    line = {
        "impl": "reference", "metric": metric, "value": v, "unit": "cell-updates/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "kelvin_helmholtz_2d", "cells": "128x128 sample of 1024x1024",
                   "flux": "HLLC", "limiter": "vanLeer", "species": 2},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": procs, "kind": "reference",
                         "sample": sample},
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


def batched_vs_plain(n_cases: int, steps: int, torch, rank: int = 0, world: int = 1, dist=None):
    """Config-4 shape: `n_cases` Richtmyer-Meshkov cases of seeded sizes 128^2..512^2 (FP32 flux,
    HLLC + superbee, own end times), advanced `steps` ensemble steps by the batched persistent
    kernel, against the same cases advanced one after the other by the single-case path.  With
    several ranks the cases are sharded by estimated work (schemi_b200.ensemble, no per-step
    exchange); totals are summed and device times maxed over the ranks."""
    from schemi_b200 import cases, ensemble, fv

    draws = [cases.richtmyer_meshkov_draws(i) for i in range(n_cases)]
    # work ~ cells x steps; steps ~ t_end / dt with dt ~ 0.5 / (n * 2.5) (post-shock signal speed)
    ws = 1.2 * math.sqrt(1.4)
    work = [ensemble.case_work(n * n, tr / ws, 0.5 / (n * 2.5)) for n, _, _, tr in draws]
    shares = ensemble.partition(work, world)
    mine = shares[rank]
    handles, t_end, cells = [], [], 0
    for i in mine:
        case, prim, te = cases.richtmyer_meshkov(i, precision="f32flux")
        g = fv.FVCase(case)
        g.set_march_shape(64, 1, 32)  # best of a sweep of ensemble tile shapes on B200
        g.upload(prim)
        handles.append(g)
        t_end.append(te)
        cells += case.n_cells
    torch.cuda.synchronize()
    # plain: each case on its own, `steps` steps through fv_run (device time per case)
    plain_ms = 0.0
    plain_updates = 0
    for g, te in zip(handles, t_end):
        st = g.run(te, max_steps=steps)
        plain_ms += st.device_ms
        plain_updates += st.steps * g.n_cells
    batch = fv.FVBatch(handles)
    batch.run(t_end, max_steps=16)  # warm-up (graph capture, kernel configuration)
    if dist is not None and world > 1:
        dist.barrier()
    st = batch.run(t_end, max_steps=steps)
    updates, ms = float(st.cell_updates), float(st.device_ms)
    if dist is not None and world > 1:
        t = torch.tensor([updates, float(plain_updates), float(cells)], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        updates, plain_updates, cells = float(t[0]), float(t[1]), int(t[2])
        t = torch.tensor([ms, plain_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, plain_ms = float(t[0]), float(t[1])
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
            "peak_source": peak_kind, "bytes_per_cell_update": head["bytes_per_cell_update"],
        },
        "fp32_flux": {
            "value": results["f32flux"]["value"], "ms_per_step": results["f32flux"]["ms_per_step"],
            "e2e": results["f32flux"]["e2e"],
            "roofline": {"bound": "hbm", "achieved": results["f32flux"]["achieved_gbs"], "peak": peak,
                         "unit": "GB/s", "frac": results["f32flux"]["achieved_gbs"] / peak,
                         "traffic": profile_traffic(f"kh{n}_f32flux")},
            "clocks": results["f32flux"]["clocks"],
        },
    }
    if args.batch_cases > 0:
        b = batched_vs_plain(args.batch_cases, args.steps, torch, rank, world, dist)
        b["roofline_frac"] = b["value"] * b["bytes_per_cell_update"] / 1e9 / peak
        line["batched"] = b
    if args.reacting_n > 0:
        line["reacting_3d"] = reacting_3d(torch, peak, args.reacting_n, args.steps, args.warmup, flush,
                                          not args.no_autotune)
    if args.adjoint_t_end > 0 and rank == 0:
        line["adjoint"] = adjoint_rt(torch, peak, args.adjoint_t_end, not args.no_autotune)
    if rank == 0 and not args.no_cpu_baseline:
        try:
            v, info = reference_throughput(n=128, steps=12, steps0=2, processes=1)
            line["cpu_baseline"] = {
                "value": v, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                "sample": (f"as-shipped reference binary (oracle/_ref/schemi), KH mixing layer {info['n']}x{info['n']} "
                           f"with slip x, {info['steps']} steps timed by differencing runs of 12 and 2 steps"),
            }
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


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
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
