"""TEST INFRASTRUCTURE: Python access to the checkers of the CUDA path.

* :class:`OracleCase` -- ctypes binding of ``lib/libfv_oracle.so``, the FP64 CPU restatement of
  Schemi's explicit finite-volume step (fv_oracle.cpp).
* :func:`run_reference` -- runs the reference solver built from its own sources into
  ``_ref/`` (see the Makefile) on a deck written by :mod:`schemi_b200.deck`.

Only the tests, the smoke check and the bench's CPU-baseline leg import this module.
"""

from __future__ import annotations

import ctypes
import os
import shutil
import subprocess
import tempfile
import time
from typing import Dict, List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libfv_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "schemi")
REF_BIN_PATCHED = os.path.join(HERE, "_ref", "schemi_patched")

FV_F_COUNT = 22
FIELD_NAMES = ["c1", "c2", "c3", "c4", "vx", "vy", "vz", "p", "rho1", "rho2", "rho3", "rho4", "rho",
               "mx", "my", "mz", "E", "Uv", "T", "sonic", "c0"]

_lib = None


def build() -> None:
    """Compile the oracle library (and, when the reference sources are present, the reference)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        D = ctypes.c_double
        DP = ctypes.POINTER(D)
        lib.fvo_create.restype = P
        lib.fvo_create.argtypes = [P, ctypes.c_char_p, ctypes.c_int]
        lib.fvo_destroy.argtypes = [P]
        lib.fvo_upload.argtypes = [P, ctypes.POINTER(DP)]
        lib.fvo_step.argtypes = [P, DP, DP]
        lib.fvo_run.argtypes = [P, D, ctypes.c_longlong, DP, ctypes.POINTER(ctypes.c_longlong)]
        lib.fvo_download.argtypes = [P, ctypes.POINTER(DP)]
        lib.fvo_get_time.argtypes = [P, DP, DP]
        lib.fvo_set_time.argtypes = [P, D, D]
        lib.fvo_get_source_timestep.argtypes = [P, DP]
        lib.fvo_get_conserved.argtypes = [P, ctypes.POINTER(DP)]
        lib.fvo_set_conserved.argtypes = [P, ctypes.POINTER(DP)]
        lib.fvo_n_cells.restype = ctypes.c_longlong
        lib.fvo_set_chem_carry.argtypes = [P, ctypes.c_int]
        lib.fvo_n_cells.argtypes = [P]
        _lib = lib
    return _lib


def _ptrs(arrays: Sequence[Optional[np.ndarray]]):
    DP = ctypes.POINTER(ctypes.c_double)
    arr = (DP * len(arrays))()
    for i, a in enumerate(arrays):
        arr[i] = a.ctypes.data_as(DP) if a is not None else None
    return arr


class OracleCase:
    """One case advanced by the FP64 CPU restatement."""

    def __init__(self, case):
        lib = load()
        self.case = case
        self._cfg = case.fv_config()
        err = ctypes.create_string_buffer(256)
        self._h = lib.fvo_create(ctypes.byref(self._cfg), err, 256)
        if not self._h:
            raise ValueError(err.value.decode())
        self.n_cells = lib.fvo_n_cells(self._h)

    def __del__(self):
        if getattr(self, "_h", None):
            load().fvo_destroy(self._h)
            self._h = None

    def upload(self, prim: Sequence[np.ndarray]) -> None:
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in prim]
        self._keep = arrs
        _check(load().fvo_upload(self._h, _ptrs(arrs)))

    def step(self):
        du, dn = ctypes.c_double(), ctypes.c_double()
        _check(load().fvo_step(self._h, ctypes.byref(du), ctypes.byref(dn)))
        return du.value, dn.value

    def run(self, t_end: float, max_steps: int = 1 << 60):
        t, n = ctypes.c_double(), ctypes.c_longlong()
        _check(load().fvo_run(self._h, t_end, max_steps, ctypes.byref(t), ctypes.byref(n)))
        return t.value, n.value

    def time(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        load().fvo_get_time(self._h, ctypes.byref(t), ctypes.byref(dt))
        return t.value, dt.value

    def set_time(self, t: float, dt: float) -> None:
        load().fvo_set_time(self._h, t, dt)

    def source_timestep(self) -> float:
        d = ctypes.c_double()
        load().fvo_get_source_timestep(self._h, ctypes.byref(d))
        return d.value

    def download(self) -> Dict[str, np.ndarray]:
        out = [np.empty(self.n_cells) for _ in range(FV_F_COUNT)]
        N = self.case.n_species
        want = [None] * FV_F_COUNT
        idx = {}
        for k in range(N):
            want[k] = out[k]; idx[f"c{k + 1}"] = k
            want[8 + k] = out[8 + k]; idx[f"rho{k + 1}"] = 8 + k
        for name, i in (("vx", 4), ("vy", 5), ("vz", 6), ("p", 7), ("rho", 12), ("mx", 13), ("my", 14),
                        ("mz", 15), ("E", 16), ("Uv", 17), ("T", 18), ("sonic", 19), ("c0", 20)):
            want[i] = out[i]
            idx[name] = i
        _check(load().fvo_download(self._h, _ptrs(want)))
        return {name: out[i] for name, i in idx.items()}

    def conserved(self) -> List[np.ndarray]:
        nc = self.case.n_conserved
        out = [np.empty(self.n_cells) for _ in range(nc)]
        _check(load().fvo_get_conserved(self._h, _ptrs(out)))
        return out

    def set_conserved(self, fields: Sequence[np.ndarray]) -> None:
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in fields]
        _check(load().fvo_set_conserved(self._h, _ptrs(arrs)))

    def set_chem_carry(self, carry: bool) -> None:
        """Chemistry sub-cycling carried on to the following cells (the reference) or per cell."""
        _check(load().fvo_set_chem_carry(self._h, int(bool(carry))))


def _check(st: int) -> None:
    if st != 0:
        raise RuntimeError(f"oracle returned status {st}")


def reference_available(patched: bool = True) -> bool:
    return os.path.exists(REF_BIN_PATCHED if patched else REF_BIN)


def run_reference(case, prim: Sequence[np.ndarray], frequency_of_output: int = 1, patched: bool = True,
                  workdir: Optional[str] = None, keep: bool = False, timeout: float = 3600.0):
    """Run the reference solver on ``case`` from the restart set ``prim``.

    Returns (outputs, times, wall_seconds): ``outputs[i]`` are the columns of
    result/output_<i>.tsv (the state after step i when frequency_of_output == 1).
    """
    from schemi_b200.deck import read_output, read_times, write_deck

    binary = REF_BIN_PATCHED if patched else REF_BIN
    if not os.path.exists(binary):
        raise FileNotFoundError(binary)
    d = workdir or tempfile.mkdtemp(prefix="schemi_ref_")
    try:
        write_deck(case, d, prim, frequency_of_output=frequency_of_output, restart=True)
        t0 = time.perf_counter()
        res = subprocess.run([binary], cwd=d, stdin=subprocess.DEVNULL, stdout=subprocess.PIPE,
                             stderr=subprocess.STDOUT, timeout=timeout)
        wall = time.perf_counter() - t0
        if res.returncode != 0:
            raise RuntimeError("reference failed:\n" + res.stdout.decode(errors="replace")[-3000:])
        times = read_times(d)
        outputs = {i: read_output(d, i) for i in sorted(times) if i >= 1 and
                   os.path.exists(os.path.join(d, "result", f"output_{i:06d}.tsv"))}
        return outputs, times, wall
    finally:
        if not keep and workdir is None:
            shutil.rmtree(d, ignore_errors=True)
