"""kamayan_b200 -- B200-native finite-volume update for kamayan's hydro path.

Python host layer over the C ABI in ``include/kmy_hydro.h`` (loaded with
ctypes from ``kamayan_b200/lib/libkmy_hydro.so``).  The compute path is the
CUDA library only: if the shared library is missing, importing the bindings
raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from .deck import Deck, deck_text  # noqa: F401

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libkmy_hydro.so"

STATUS = {
    0: "OK",
    1: "BAD_PARAM",
    2: "OOM",
    3: "NONFINITE",
    4: "TIMEOUT",
    5: "CUDA",
    6: "STATE",
    7: "DT_RANGE",
}

# Every entry point declared in include/kmy_hydro.h.
EXPORTS = (
    "kmy_create", "kmy_destroy", "kmy_last_error", "kmy_get_info", "kmy_set_stream", "kmy_sync",
    "kmy_import_var", "kmy_export_var", "kmy_import_interior", "kmy_export_interior",
    "kmy_finalize_import", "kmy_pgen", "kmy_bind_container", "kmy_bind_primitives",
    "kmy_compute_fluxes", "kmy_compute_emf", "kmy_flux_divergence", "kmy_apply_dudt",
    "kmy_prepare_primitive", "kmy_fill_ghosts", "kmy_estimate_dt", "kmy_fill_derived",
    "kmy_task_stage", "kmy_rk_stage", "kmy_step", "kmy_evolve", "kmy_end_step", "kmy_get_time",
    "kmy_zone_cycles",
    "kmy_get_blocks", "kmy_set_dt", "kmy_save_restart", "kmy_load_restart",
    "kmy_set_path", "kmy_vortex_error", "kmy_conserved_sums", "kmy_launch_count",
    "kmy_graph_replays", "kmy_evolve_device_ms", "kmy_set_fault", "kmy_reconstruct_stencils", "kmy_autotune", "kmy_stage_kernel", "kmy_tune_key", "kmy_tune_cache_put",
    "kmy_tune_cache_get", "kmy_tune_cache_clear", "kmy_tune_cache_save", "kmy_tune_cache_load",
    "kmy_conserved_sums_noalloc",
    "kmy_server_create", "kmy_server_destroy", "kmy_server_last_error", "kmy_server_submit",
    "kmy_server_tick", "kmy_server_poll", "kmy_server_export", "kmy_server_release",
    "kmy_server_stats",
)


class KmyError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class TuneResult(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 16), ("ms", ctypes.c_double), ("applies", ctypes.c_int)]


class Info(ctypes.Structure):
    _fields_ = [
        ("ndim", ctypes.c_int), ("nblocks", ctypes.c_int), ("nx", ctypes.c_int * 3),
        ("nghost", ctypes.c_int), ("ncells_pad", ctypes.c_int * 3),
        ("nfaces_pad", ctypes.c_int * 3), ("nblocks_dim", ctypes.c_int * 3),
        ("ncons", ctypes.c_int), ("mhd", ctypes.c_int), ("nstages", ctypes.c_int),
        ("precision", ctypes.c_int), ("xmin", ctypes.c_double * 3), ("xmax", ctypes.c_double * 3),
        ("dx", ctypes.c_double * 3),
    ]


_lib = None
_dp = ctypes.POINTER(ctypes.c_double)


def lib() -> ctypes.CDLL:
    """Load libkmy_hydro.so (built by ``kamayan_b200.build``)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run `python -m kamayan_b200.build` first")
        L = ctypes.CDLL(str(LIB_PATH))
        vp, cp, i, d, sz = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t
        L.kmy_create.argtypes = [cp, i, ctypes.POINTER(vp)]
        L.kmy_destroy.argtypes = [vp]
        L.kmy_last_error.restype = cp
        L.kmy_last_error.argtypes = [vp]
        L.kmy_get_info.argtypes = [vp, ctypes.POINTER(Info)]
        L.kmy_set_stream.argtypes = [vp, vp]
        L.kmy_sync.argtypes = [vp]
        L.kmy_import_var.argtypes = [vp, cp, cp, i, _dp, sz]
        L.kmy_export_var.argtypes = [vp, cp, cp, i, _dp, sz]
        L.kmy_import_interior.argtypes = [vp, cp, cp, i, _dp, sz]
        L.kmy_export_interior.argtypes = [vp, cp, cp, i, _dp, sz]
        L.kmy_finalize_import.argtypes = [vp]
        L.kmy_bind_container.argtypes = [vp, cp, vp, sz, vp, sz, vp, sz]
        L.kmy_bind_primitives.argtypes = [vp, vp, sz]
        L.kmy_pgen.argtypes = [vp, cp]
        for n in ("kmy_compute_fluxes", "kmy_compute_emf", "kmy_prepare_primitive",
                  "kmy_fill_ghosts", "kmy_fill_derived"):
            getattr(L, n).argtypes = [vp, cp]
        L.kmy_flux_divergence.argtypes = [vp, cp, cp]
        L.kmy_apply_dudt.argtypes = [vp, cp, cp, cp, cp, d, d]
        L.kmy_estimate_dt.argtypes = [vp, cp, _dp]
        L.kmy_task_stage.argtypes = [vp, i, d]
        L.kmy_rk_stage.argtypes = [vp, i, d]
        L.kmy_step.argtypes = [vp, _dp]
        L.kmy_evolve.argtypes = [vp, d, i, ctypes.POINTER(i)]
        L.kmy_end_step.argtypes = [vp]
        L.kmy_get_time.argtypes = [vp, _dp, _dp, _dp, ctypes.POINTER(i)]
        L.kmy_get_blocks.argtypes = [vp, ctypes.POINTER(i), ctypes.POINTER(i), i, ctypes.POINTER(i)]
        L.kmy_save_restart.argtypes = [vp, cp]
        L.kmy_load_restart.argtypes = [cp, i, ctypes.POINTER(vp)]
        L.kmy_set_dt.argtypes = [vp, d]
        L.kmy_set_path.argtypes = [vp, i]
        L.kmy_vortex_error.argtypes = [vp, i, i, _dp]
        L.kmy_conserved_sums.argtypes = [vp, cp, _dp]
        L.kmy_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.kmy_zone_cycles.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.kmy_graph_replays.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.kmy_evolve_device_ms.argtypes = [vp, _dp]
        L.kmy_set_fault.argtypes = [vp, cp, i]
        L.kmy_reconstruct_stencils.argtypes = [cp, cp, i, _dp, i, _dp]
        L.kmy_autotune.argtypes = [vp, i, ctypes.POINTER(TuneResult), i, ctypes.POINTER(i)]
        L.kmy_stage_kernel.argtypes = [vp, cp, sz]
        L.kmy_tune_key.argtypes = [cp, cp, sz]
        L.kmy_tune_cache_put.argtypes = [cp, cp, d]
        L.kmy_tune_cache_get.argtypes = [cp, cp, sz, _dp]
        L.kmy_tune_cache_clear.argtypes = []
        L.kmy_tune_cache_save.argtypes = [cp]
        L.kmy_tune_cache_load.argtypes = [cp]
        ip3 = ctypes.POINTER(ctypes.c_int)
        L.kmy_conserved_sums_noalloc.argtypes = [vp, i, i, ip3, ip3, ip3, d, vp, vp]
        i64p = ctypes.POINTER(ctypes.c_int64)
        L.kmy_server_create.argtypes = [i, d, i, ctypes.POINTER(vp)]
        L.kmy_server_destroy.argtypes = [vp]
        L.kmy_server_last_error.restype = cp
        L.kmy_server_last_error.argtypes = [vp]
        L.kmy_server_submit.argtypes = [vp, cp, cp, i, i64p]
        L.kmy_server_tick.argtypes = [vp, ctypes.POINTER(i), ctypes.POINTER(i)]
        L.kmy_server_poll.argtypes = [vp, i64p, _dp, ctypes.POINTER(i), i, ctypes.POINTER(i)]
        L.kmy_server_export.argtypes = [vp, ctypes.c_int64, cp, i, _dp, sz]
        L.kmy_server_release.argtypes = [vp, ctypes.c_int64]
        L.kmy_server_stats.argtypes = [vp, _dp]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class Solver:
    """One mesh with its device-resident stage containers (one ``kmy_ctx``)."""

    def __init__(self, deck: str | Deck | None, device: int = 0, _handle=None):
        if _handle is not None:
            h = _handle
        else:
            text = deck.text() if isinstance(deck, Deck) else deck
            h = ctypes.c_void_p()
            rc = lib().kmy_create(text.encode(), device, ctypes.byref(h))
            if rc:
                raise KmyError(rc, "kmy_create rejected the deck (see stderr)")
        self._h = h
        self._lib = lib()  # kept so close() still works while the interpreter shuts down
        self._info = Info()
        self.ndim = self.info.ndim

    # An adaptive mesh changes its block count as it refines, so the mesh
    # description is read from the context on every use.
    @property
    def info(self) -> Info:
        self._check(lib().kmy_get_info(self._h, ctypes.byref(self._info)))
        return self._info

    @property
    def nblocks(self) -> int:
        return self.info.nblocks

    @property
    def cell_shape(self) -> tuple:
        i = self.info
        return (i.nblocks, i.ncells_pad[2], i.ncells_pad[1], i.ncells_pad[0])

    @property
    def face_shape(self) -> tuple:
        i = self.info
        return (i.nblocks, i.nfaces_pad[2], i.nfaces_pad[1], i.nfaces_pad[0])

    def save_restart(self, path: str) -> None:
        """Write the state needed to resume this solve (kmy_save_restart)."""
        self._check(lib().kmy_save_restart(self._h, str(path).encode()))

    @classmethod
    def from_restart(cls, path: str, device: int = 0) -> "Solver":
        """A new solver that resumes from a restart file (kmy_load_restart)."""
        h = ctypes.c_void_p()
        rc = lib().kmy_load_restart(str(path).encode(), device, ctypes.byref(h))
        if rc:
            raise KmyError(rc, f"kmy_load_restart failed for {path} (see stderr)")
        return cls(None, device, _handle=h)

    def blocks(self) -> tuple[np.ndarray, np.ndarray]:
        """Leaf blocks in block order: levels (nb,) and logical locations (nb, 3)."""
        n = ctypes.c_int()
        self._check(lib().kmy_get_blocks(self._h, None, None, 0, ctypes.byref(n)))
        lev = np.zeros(n.value, dtype=np.int32)
        loc = np.zeros((n.value, 3), dtype=np.int32)
        ip = ctypes.POINTER(ctypes.c_int)
        self._check(lib().kmy_get_blocks(self._h, lev.ctypes.data_as(ip), loc.ctypes.data_as(ip), n.value,
                                         ctypes.byref(n)))
        return lev, loc

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.kmy_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int) -> None:
        if rc:
            raise KmyError(rc, lib().kmy_last_error(self._h).decode())

    # --- state ---
    def _shape(self, var: str):
        return self.face_shape if var == "mag" else self.cell_shape

    def export(self, var: str, comp: int = 0, container: str = "base") -> np.ndarray:
        out = np.empty(self._shape(var), dtype=np.float64)
        self._check(lib().kmy_export_var(self._h, container.encode(), var.encode(), comp,
                                         _ptr(out), out.size))
        return out

    def import_(self, var: str, arr, comp: int = 0, container: str = "base") -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        self._check(lib().kmy_import_var(self._h, container.encode(), var.encode(), comp,
                                         _ptr(a), a.size))

    def import_ptr(self, var: str, ptr: int, n: int, comp: int = 0, container: str = "base") -> None:
        """Import n doubles from host address ptr (e.g. a pinned buffer)."""
        self._check(lib().kmy_import_var(self._h, container.encode(), var.encode(), comp,
                                         ctypes.cast(ptr, _dp), n))

    def export_ptr(self, var: str, ptr: int, n: int, comp: int = 0, container: str = "base") -> None:
        self._check(lib().kmy_export_var(self._h, container.encode(), var.encode(), comp,
                                         ctypes.cast(ptr, _dp), n))

    @property
    def interior_shape(self):
        i = self.info
        return (i.nblocks, i.nx[2], i.nx[1], i.nx[0])

    def export_interior(self, var: str, comp: int = 0, container: str = "base") -> np.ndarray:
        """Interior cells only, (nblocks, nk, nj, ni) (kmy_export_interior)."""
        out = np.empty(self.interior_shape, dtype=np.float64)
        self._check(lib().kmy_export_interior(self._h, container.encode(), var.encode(), comp,
                                              _ptr(out), out.size))
        return out

    def import_interior(self, var: str, arr, comp: int = 0, container: str = "base") -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        self._check(lib().kmy_import_interior(self._h, container.encode(), var.encode(), comp,
                                              _ptr(a), a.size))

    def import_interior_ptr(self, var: str, ptr: int, n: int, comp: int = 0, container: str = "base") -> None:
        """Import n interior-cell doubles from host address ptr (e.g. a pinned buffer)."""
        self._check(lib().kmy_import_interior(self._h, container.encode(), var.encode(), comp,
                                              ctypes.cast(ptr, _dp), n))

    def export_interior_ptr(self, var: str, ptr: int, n: int, comp: int = 0, container: str = "base") -> None:
        self._check(lib().kmy_export_interior(self._h, container.encode(), var.encode(), comp,
                                              ctypes.cast(ptr, _dp), n))

    def bind_container(self, container: str, cons_ptr: int, cons_bytes: int, ener_lo_ptr: int = 0,
                       ener_lo_bytes: int = 0, mag_ptr: int = 0, mag_bytes: int = 0) -> None:
        """Make caller-owned device arrays the storage of a container (kmy_bind_container)."""
        self._check(lib().kmy_bind_container(self._h, container.encode(), ctypes.c_void_p(cons_ptr), cons_bytes,
                                             ctypes.c_void_p(ener_lo_ptr or None), ener_lo_bytes,
                                             ctypes.c_void_p(mag_ptr or None), mag_bytes))

    def bind_primitives(self, prim_ptr: int, nbytes: int) -> None:
        self._check(lib().kmy_bind_primitives(self._h, ctypes.c_void_p(prim_ptr), nbytes))

    def finalize_import(self) -> None:
        self._check(lib().kmy_finalize_import(self._h))

    def pgen(self, problem: str) -> None:
        self._check(lib().kmy_pgen(self._h, problem.encode()))

    # --- stepping ---
    def step(self) -> float:
        dt = ctypes.c_double()
        self._check(lib().kmy_step(self._h, ctypes.byref(dt)))
        return dt.value

    def evolve(self, tlim: float, nlim: int = -1) -> int:
        n = ctypes.c_int()
        self._check(lib().kmy_evolve(self._h, tlim, nlim, ctypes.byref(n)))
        return n.value

    def rk_stage(self, stage: int, dt: float = -1.0) -> None:
        """One fused stage; dt < 0 takes the dt held by the device clock."""
        self._check(lib().kmy_rk_stage(self._h, stage, dt))

    def end_step(self) -> None:
        self._check(lib().kmy_end_step(self._h))

    def set_stream(self, cuda_stream: int) -> None:
        """Run on a caller-owned cudaStream_t (e.g. torch.cuda.Stream().cuda_stream)."""
        self._check(lib().kmy_set_stream(self._h, ctypes.c_void_p(cuda_stream)))

    def task_stage(self, stage: int, dt: float) -> None:
        self._check(lib().kmy_task_stage(self._h, stage, dt))

    def set_path(self, path: str) -> None:
        self._check(lib().kmy_set_path(self._h, {"fused": 0, "tasks": 1}[path]))

    def set_dt(self, dt: float) -> None:
        self._check(lib().kmy_set_dt(self._h, dt))

    def sync(self) -> None:
        self._check(lib().kmy_sync(self._h))

    @property
    def time(self) -> dict:
        t, dt, est = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        n = ctypes.c_int()
        self._check(lib().kmy_get_time(self._h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(est),
                                       ctypes.byref(n)))
        return dict(time=t.value, dt=dt.value, dt_est=est.value, ncycle=n.value)

    # --- per-task entry points ---
    def compute_fluxes(self, md0: str) -> None:
        self._check(lib().kmy_compute_fluxes(self._h, md0.encode()))

    def compute_emf(self, md0: str) -> None:
        self._check(lib().kmy_compute_emf(self._h, md0.encode()))

    def flux_divergence(self, md0: str, dudt: str = "dUdt") -> None:
        self._check(lib().kmy_flux_divergence(self._h, md0.encode(), dudt.encode()))

    def apply_dudt(self, base: str, md0: str, md1: str, dudt: str, beta: float, dt: float) -> None:
        self._check(lib().kmy_apply_dudt(self._h, base.encode(), md0.encode(), md1.encode(),
                                         dudt.encode(), beta, dt))

    def prepare_primitive(self, md1: str) -> None:
        self._check(lib().kmy_prepare_primitive(self._h, md1.encode()))

    def fill_ghosts(self, md: str = "base") -> None:
        self._check(lib().kmy_fill_ghosts(self._h, md.encode()))

    def estimate_dt(self, md: str = "base") -> float:
        out = ctypes.c_double()
        self._check(lib().kmy_estimate_dt(self._h, md.encode(), ctypes.byref(out)))
        return out.value

    def fill_derived(self, md: str = "base") -> None:
        self._check(lib().kmy_fill_derived(self._h, md.encode()))

    # --- diagnostics ---
    def vortex_error(self, var: str = "dens", comp: int = 0) -> float:
        out = ctypes.c_double()
        self._check(lib().kmy_vortex_error(self._h, {"dens": 0, "velocity": 1, "pres": 2, "magc": 3}[var], comp,
                                           ctypes.byref(out)))
        return out.value

    def conserved_sums(self, md: str = "base") -> np.ndarray:
        out = np.zeros(self.info.ncons)
        self._check(lib().kmy_conserved_sums(self._h, md.encode(), _ptr(out)))
        return out

    @property
    def zone_cycles(self) -> int:
        """Interior cells x completed steps since set-up (each step counted on
        the mesh it ran on)."""
        n = ctypes.c_int64()
        self._check(lib().kmy_zone_cycles(self._h, ctypes.byref(n)))
        return n.value

    @property
    def launch_count(self) -> int:
        n = ctypes.c_int64()
        self._check(lib().kmy_launch_count(self._h, ctypes.byref(n)))
        return n.value

    def set_fault(self, what: str, value: int = 1) -> None:
        """Failure-path test hook (kmy_set_fault)."""
        self._check(lib().kmy_set_fault(self._h, what.encode(), value))

    @property
    def graph_replays(self) -> int:
        """kmy_evolve chunks (adaptive steps) that replayed a cached CUDA graph."""
        n = ctypes.c_int64()
        self._check(lib().kmy_graph_replays(self._h, ctypes.byref(n)))
        return n.value

    @property
    def evolve_device_ms(self) -> float:
        """Device time (ms) of the last evolve call, host read-backs excluded
        (kmy_evolve_device_ms)."""
        v = ctypes.c_double()
        self._check(lib().kmy_evolve_device_ms(self._h, ctypes.byref(v)))
        return v.value

    def autotune(self, reps: int = 5) -> dict:
        """Time every stage kernel that applies on the current state, apply
        and cache the fastest; {name: ms per stage (None where it does not apply)}."""
        res = (TuneResult * 8)()
        n = ctypes.c_int()
        self._check(lib().kmy_autotune(self._h, reps, res, 8, ctypes.byref(n)))
        return {res[k].name.decode(): (res[k].ms if res[k].applies else None) for k in range(n.value)}

    @property
    def stage_kernel(self) -> str:
        buf = ctypes.create_string_buffer(64)
        self._check(lib().kmy_stage_kernel(self._h, buf, 64))
        return buf.value.decode()

    def interior(self, arr: np.ndarray) -> np.ndarray:
        i = self.info
        g = i.nghost
        g2 = g if i.ndim > 1 else 0
        g3 = g if i.ndim > 2 else 0
        return arr[:, g3:g3 + i.nx[2], g2:g2 + i.nx[1], g:g + i.nx[0]]


class Server:
    """Serving loop over the C ABI: continuously batched independent solves."""

    STATS = ("active", "queued", "finished", "bytes_in_use", "budget", "ticks", "cell_updates",
             "launches")

    def __init__(self, device: int = 0, hbm_fraction: float = 0.8, graphs: bool = True):
        h = ctypes.c_void_p()
        rc = lib().kmy_server_create(device, hbm_fraction, int(graphs), ctypes.byref(h))
        if rc:
            raise KmyError(rc, "kmy_server_create failed")
        self._h = h
        self._lib = lib()

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.kmy_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int) -> None:
        if rc:
            raise KmyError(rc, lib().kmy_server_last_error(self._h).decode())

    def submit(self, deck, problem: str, nsteps: int) -> int:
        text = deck.text() if isinstance(deck, Deck) else deck
        rid = ctypes.c_int64()
        self._check(lib().kmy_server_submit(self._h, text.encode(), problem.encode(), nsteps,
                                            ctypes.byref(rid)))
        return rid.value

    def tick(self) -> tuple[int, int]:
        a, q = ctypes.c_int(), ctypes.c_int()
        self._check(lib().kmy_server_tick(self._h, ctypes.byref(a), ctypes.byref(q)))
        return a.value, q.value

    def poll(self, max_items: int = 4096) -> list[tuple[int, float, int]]:
        ids = (ctypes.c_int64 * max_items)()
        secs = (ctypes.c_double * max_items)()
        st = (ctypes.c_int * max_items)()
        n = ctypes.c_int()
        self._check(lib().kmy_server_poll(self._h, ids, secs, st, max_items, ctypes.byref(n)))
        return [(ids[k], secs[k], st[k]) for k in range(n.value)]

    def export(self, rid: int, var: str, shape, comp: int = 0) -> np.ndarray:
        out = np.empty(shape, dtype=np.float64)
        self._check(lib().kmy_server_export(self._h, rid, var.encode(), comp, _ptr(out), out.size))
        return out

    def release(self, rid: int) -> None:
        self._check(lib().kmy_server_release(self._h, rid))

    @property
    def stats(self) -> dict:
        out = np.zeros(8)
        self._check(lib().kmy_server_stats(self._h, _ptr(out)))
        return dict(zip(self.STATS, out.tolist()))


# ---- the stage-kernel tuner's cache (host only; no GPU needed) --------------
def tune_key(deck) -> str:
    """Configuration part of the tuner's cache key for a deck."""
    buf = ctypes.create_string_buffer(256)
    text = deck.text() if isinstance(deck, Deck) else deck
    rc = lib().kmy_tune_key(text.encode(), buf, 256)
    if rc:
        raise KmyError(rc, "kmy_tune_key")
    return buf.value.decode()


def tune_cache_put(key: str, choice: str, ms: float = 0.0) -> None:
    rc = lib().kmy_tune_cache_put(key.encode(), choice.encode(), ms)
    if rc:
        raise KmyError(rc, f"kmy_tune_cache_put {choice!r}")


def tune_cache_get(key: str):
    """(choice, ms) for a key, or None."""
    buf = ctypes.create_string_buffer(32)
    ms = ctypes.c_double()
    rc = lib().kmy_tune_cache_get(key.encode(), buf, 32, ctypes.byref(ms))
    if rc == 6:
        return None
    if rc:
        raise KmyError(rc, "kmy_tune_cache_get")
    return buf.value.decode(), ms.value


def tune_cache_clear() -> None:
    lib().kmy_tune_cache_clear()


def tune_cache_save(path: str) -> None:
    rc = lib().kmy_tune_cache_save(str(path).encode())
    if rc:
        raise KmyError(rc, f"kmy_tune_cache_save {path}")


def tune_cache_load(path: str) -> None:
    rc = lib().kmy_tune_cache_load(str(path).encode())
    if rc:
        raise KmyError(rc, f"kmy_tune_cache_load {path}")


# ---- the device reconstruction functions on a batch of stencils --------------
RECON_IMPLS = {"fp64_tasks": 0, "fp64_brick": 1, "fp32_lane": 2, "fp32_brick": 3, "fp32_slab": 4, "fp64_slab": 5,
               "fp64_nr_math": 6}


def reconstruct_stencils(reconstruction: str, slope_limiter: str, impl: str, stencils) -> np.ndarray:
    """(n, 3) array of (vM, vP, lanes-disagree flag) for n 5-cell stencils."""
    st = np.ascontiguousarray(np.asarray(stencils, dtype=np.float64).reshape(-1, 5))
    out = np.zeros((st.shape[0], 3))
    rc = lib().kmy_reconstruct_stencils(reconstruction.encode(), slope_limiter.encode(), RECON_IMPLS[impl],
                                        _ptr(st), st.shape[0], _ptr(out))
    if rc:
        raise KmyError(rc, "kmy_reconstruct_stencils")
    return out
