"""ctypes binding of the C-ABI in include/fvstep.h (``schemi_b200/lib/libschemi_fv.so``).

:class:`FVCase` owns one ``fv_handle``.  The library is mandatory: loading fails loudly when it
is missing or when no CUDA device is visible -- there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os
from typing import Dict, List, Optional, Sequence

import numpy as np

from .case import Case, fv_config_t

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libschemi_fv.so")

FV_F_COUNT = 22
FIELD_INDEX = {"vx": 4, "vy": 5, "vz": 6, "p": 7, "rho": 12, "mx": 13, "my": 14, "mz": 15, "E": 16, "Uv": 17,
               "T": 18, "sonic": 19, "c0": 20}
ERRORS = {0: "noErrors", 1: "RiemannSolverError", 2: "negativeTemperatureError", 4: "systemError",
          5: "boundaryConditionError", 11: "initialisationError", 12: "NaNError"}
PATH_MARCH, PATH_GENERIC = 0, 1

_lib = None


class FVError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{ERRORS.get(status, status)}: {message}")
        self.status = status


class fv_run_stats_t(ctypes.Structure):
    _fields_ = [("time", ctypes.c_double), ("dt_next", ctypes.c_double), ("steps", ctypes.c_longlong),
                ("device_ms", ctypes.c_float)]


class fv_batch_stats_t(ctypes.Structure):
    _fields_ = [("cell_updates", ctypes.c_longlong), ("steps_max", ctypes.c_longlong),
                ("launches", ctypes.c_longlong), ("device_ms", ctypes.c_float)]


class fv_record_config_t(ctypes.Structure):
    _fields_ = [("checkpoint_every", ctypes.c_int), ("objective", ctypes.c_int), ("heavy_species", ctypes.c_int),
                ("pad", ctypes.c_int)]


class fv_record_stats_t(ctypes.Structure):
    _fields_ = [("objective", ctypes.c_double), ("time", ctypes.c_double), ("steps", ctypes.c_longlong),
                ("checkpoints", ctypes.c_longlong), ("device_ms", ctypes.c_float)]


class fv_adjoint_stats_t(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_longlong), ("recomputed", ctypes.c_longlong), ("device_ms", ctypes.c_float),
                ("recompute_ms", ctypes.c_float)]


OBJ_NONE, OBJ_MIXING_WIDTH = 0, 1


def library_path() -> str:
    return LIB_PATH


def load():
    """Load the CUDA library (raises when it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m schemi_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    P, I, D, LL = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
    DP = ctypes.POINTER(D)
    lib.fv_abi_version.restype = I
    lib.fv_create.argtypes = [ctypes.POINTER(fv_config_t), ctypes.POINTER(P)]
    lib.fv_destroy.argtypes = [P]
    lib.fv_last_error.restype = ctypes.c_char_p
    lib.fv_last_error.argtypes = [P]
    lib.fv_upload.argtypes = [P, ctypes.POINTER(DP)]
    lib.fv_upload_device.argtypes = [P, ctypes.POINTER(DP)]
    lib.fv_step.argtypes = [P, DP, DP]
    lib.fv_run.argtypes = [P, D, LL, ctypes.POINTER(fv_run_stats_t)]
    lib.fv_download.argtypes = [P, ctypes.POINTER(DP)]
    lib.fv_get_time.argtypes = [P, DP, DP]
    lib.fv_set_time.argtypes = [P, D, D]
    lib.fv_get_source_timestep.argtypes = [P, DP]
    lib.fv_state_device.argtypes = [P, ctypes.POINTER(DP), ctypes.POINTER(I), ctypes.POINTER(LL)]
    lib.fv_sync.argtypes = [P]
    lib.fv_step_path.argtypes = [P]
    lib.fv_set_march_shape.argtypes = [P, I, I, I]
    lib.fv_force_generic.argtypes = [P]
    lib.fv_time_step_kernel.argtypes = [P, I, ctypes.POINTER(ctypes.c_float)]
    lib.fv_set_staging.argtypes = [P, I]
    lib.fv_get_staging.argtypes = [P]
    lib.fv_begin_steps.argtypes = [P]
    lib.fv_step_async.argtypes = [P]
    lib.fv_check.argtypes = [P]
    lib.fv_stream.restype = P
    lib.fv_stream.argtypes = [P]
    lib.fv_kernels_per_step.restype = LL
    lib.fv_kernels_per_step.argtypes = [P]
    lib.fv_record.argtypes = [P, ctypes.POINTER(fv_record_config_t), D, LL, ctypes.POINTER(fv_record_stats_t)]
    lib.fv_replay.argtypes = [P, ctypes.POINTER(fv_record_stats_t)]
    lib.fv_adjoint.argtypes = [P, P, D, P, ctypes.POINTER(fv_adjoint_stats_t)]
    lib.fv_state_copy.argtypes = [P, P]
    if hasattr(lib, "fv_batch_create"):
        lib.fv_batch_create.argtypes = [ctypes.POINTER(P), I, ctypes.POINTER(P)]
        lib.fv_batch_run.argtypes = [P, DP, LL, ctypes.POINTER(fv_batch_stats_t)]
        lib.fv_batch_destroy.argtypes = [P]
    _lib = lib
    return lib


def _ptrs(arrays: Sequence[Optional[np.ndarray]]):
    DP = ctypes.POINTER(ctypes.c_double)
    arr = (DP * len(arrays))()
    for i, a in enumerate(arrays):
        arr[i] = a.ctypes.data_as(DP) if a is not None else None
    return arr


class FVCase:
    """One case on the GPU: the drop-in for the reference's step solver + CFL block."""

    def __init__(self, case: Case):
        self.lib = load()
        self.case = case
        self._cfg = case.fv_config()
        h = ctypes.c_void_p()
        st = self.lib.fv_create(ctypes.byref(self._cfg), ctypes.byref(h))
        if st != 0:
            raise FVError(st, "fv_create failed (see stderr)")
        self._h = h
        self.n_cells = case.n_cells

    def close(self):
        if getattr(self, "_h", None):
            self.lib.fv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != 0:
            msg = self.lib.fv_last_error(self._h)
            raise FVError(st, msg.decode() if msg else "")

    @property
    def handle(self):
        return self._h

    @property
    def path(self) -> int:
        return self.lib.fv_step_path(self._h)

    def upload(self, prim: Sequence[np.ndarray]) -> None:
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in prim]
        if len(arrs) != self.case.n_species + 4:
            raise ValueError("restart set is c_1..c_N, v_x, v_y, v_z, p")
        self._check(self.lib.fv_upload(self._h, _ptrs(arrs)))

    def upload_device(self, ptrs: Sequence[int]) -> None:
        DP = ctypes.POINTER(ctypes.c_double)
        arr = (DP * len(ptrs))(*[ctypes.cast(p, DP) for p in ptrs])
        self._check(self.lib.fv_upload_device(self._h, arr))

    def step(self):
        du, dn = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.fv_step(self._h, ctypes.byref(du), ctypes.byref(dn)))
        return du.value, dn.value

    def run(self, t_end: float, max_steps: int = 1 << 60) -> fv_run_stats_t:
        s = fv_run_stats_t()
        self._check(self.lib.fv_run(self._h, t_end, max_steps, ctypes.byref(s)))
        return s

    def time(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.fv_get_time(self._h, ctypes.byref(t), ctypes.byref(dt)))
        return t.value, dt.value

    def set_time(self, t: float, dt: float) -> None:
        self._check(self.lib.fv_set_time(self._h, t, dt))

    def source_timestep(self) -> float:
        """The limit the last step's diffusion stage set for the next step (fv_get_source_timestep)."""
        d = ctypes.c_double()
        self._check(self.lib.fv_get_source_timestep(self._h, ctypes.byref(d)))
        return d.value

    def download_fields(self) -> Dict[str, int]:
        """Names of the fields fv_download writes for this case, with their fv_download index."""
        names = {}
        for k in range(self.case.n_species):
            names[f"c{k + 1}"] = k
            names[f"rho{k + 1}"] = 8 + k
        names.update(FIELD_INDEX)
        return names

    def download(self, out: Optional[Dict[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
        """fv_download into new arrays, or into ``out`` (name -> contiguous float64 array of
        n_cells, e.g. views of pinned host memory, which the copies then reach by DMA)."""
        names = self.download_fields()
        arrs = [None] * FV_F_COUNT
        for name, i in names.items():
            if out is not None:
                a = out[name]
                if a.dtype != np.float64 or a.size != self.n_cells or not a.flags.c_contiguous:
                    raise ValueError(f"download buffer {name}: contiguous float64 of {self.n_cells} values")
                arrs[i] = a
            else:
                arrs[i] = np.empty(self.n_cells)
        self._check(self.lib.fv_download(self._h, _ptrs(arrs)))
        return {name: arrs[i] for name, i in names.items()}

    def state_device(self):
        nf = self.case.n_conserved
        DP = ctypes.POINTER(ctypes.c_double)
        arr = (DP * 16)()
        n_f, n_c = ctypes.c_int(), ctypes.c_longlong()
        self._check(self.lib.fv_state_device(self._h, arr, ctypes.byref(n_f), ctypes.byref(n_c)))
        return [ctypes.cast(arr[i], ctypes.c_void_p).value for i in range(n_f.value)], n_c.value

    def sync(self):
        self._check(self.lib.fv_sync(self._h))

    def set_march_shape(self, bx: int, by: int, rows: int) -> None:
        self._check(self.lib.fv_set_march_shape(self._h, bx, by, rows))

    def force_generic(self) -> None:
        self._check(self.lib.fv_force_generic(self._h))

    def set_staging(self, on: bool) -> None:
        self._check(self.lib.fv_set_staging(self._h, int(bool(on))))

    @property
    def staging(self) -> bool:
        return self.lib.fv_get_staging(self._h) == 1

    def begin_steps(self) -> None:
        self._check(self.lib.fv_begin_steps(self._h))

    def step_async(self) -> None:
        self._check(self.lib.fv_step_async(self._h))

    def check(self) -> None:
        self._check(self.lib.fv_check(self._h))

    @property
    def stream_ptr(self) -> int:
        return self.lib.fv_stream(self._h)

    @property
    def kernels_per_step(self) -> int:
        return self.lib.fv_kernels_per_step(self._h)

    def time_step_kernel(self, iters: int) -> float:
        ms = ctypes.c_float()
        self._check(self.lib.fv_time_step_kernel(self._h, iters, ctypes.byref(ms)))
        return ms.value

    # ---- adjoint (fv_record / fv_replay / fv_adjoint)
    @property
    def n_conserved(self) -> int:
        return self.case.n_conserved

    def record(self, t_end: float, checkpoint_every: int = 50, objective: int = OBJ_MIXING_WIDTH,
               heavy_species: int = 0, max_steps: int = 1 << 60) -> fv_record_stats_t:
        """Forward to t_end storing checkpoints and each step's dt and gravity; returns the
        mixing-width objective J = sum_n dt_{n-1} W(U^n) in ``.objective``."""
        rc = fv_record_config_t(checkpoint_every, objective, heavy_species, 0)
        s = fv_record_stats_t()
        # the handle keeps one trajectory: count the recordings so that a caller holding an older
        # one (TimeLoop's backward) can tell it has been replaced
        self.records = getattr(self, "records", 0) + 1
        self._check(self.lib.fv_record(self._h, ctypes.byref(rc), t_end, max_steps, ctypes.byref(s)))
        return s

    def replay(self) -> fv_record_stats_t:
        """The recorded number of steps again from the current state with the recorded dt."""
        s = fv_record_stats_t()
        self._check(self.lib.fv_replay(self._h, ctypes.byref(s)))
        return s

    def adjoint(self, dJ_dU_T_ptr: Optional[int], dJ_dJ: float, dJ_dU_0_ptr: int) -> fv_adjoint_stats_t:
        """Backward sweep: writes dJtot/dU^0 to the device array at dJ_dU_0_ptr (fv_state_device
        layout); dJ_dU_T_ptr may be None."""
        s = fv_adjoint_stats_t()
        self._check(self.lib.fv_adjoint(self._h, dJ_dU_T_ptr, float(dJ_dJ), dJ_dU_0_ptr, ctypes.byref(s)))
        return s

    def state_copy(self, dst_ptr: int) -> None:
        """Copies the conserved state to the device array at dst_ptr."""
        self._check(self.lib.fv_state_copy(self._h, dst_ptr))


class FVBatch:
    """Ensemble of FVCase handles advanced together by the batched persistent kernel."""

    def __init__(self, handles: Sequence[FVCase]):
        self.lib = load()
        self.handles = list(handles)
        arr = (ctypes.c_void_p * len(self.handles))(*[h.handle for h in self.handles])
        b = ctypes.c_void_p()
        st = self.lib.fv_batch_create(arr, len(self.handles), ctypes.byref(b))
        if st != 0:
            raise FVError(st, "fv_batch_create failed (see stderr)")
        self._b = b

    def run(self, t_end: Sequence[float], max_steps: int = 1 << 60) -> fv_batch_stats_t:
        te = np.ascontiguousarray(np.asarray(t_end, dtype=np.float64))
        if te.size != len(self.handles):
            raise ValueError("one end time per case")
        s = fv_batch_stats_t()
        st = self.lib.fv_batch_run(self._b, te.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), max_steps,
                                   ctypes.byref(s))
        if st != 0:
            raise FVError(st, "fv_batch_run")
        return s

    def close(self):
        if getattr(self, "_b", None):
            self.lib.fv_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

