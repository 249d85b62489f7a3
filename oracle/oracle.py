"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle is a C++ restatement of kamayan's finite-volume update
(``oracle/kmy_oracle.cpp``).  Only the test-suite, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` leg of ``bench.py`` use it, always as the checker or
as the timed CPU baseline -- never as part of the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libkmy_oracle.so"
# the host-tuned timing build (oracle/Makefile target `native`), which
# cpu_bench selects before the first load; the parity build otherwise.  It is
# built per host CPU (model and flags) so a copy from another machine is never
# loaded.
use_native = False


def _host_tag() -> str:
    import hashlib

    info = ""
    try:
        lines = Path("/proc/cpuinfo").read_text().splitlines()
        info = "\n".join(sorted({ln for ln in lines if ln.startswith(("model name", "flags"))}))
    except OSError:
        pass
    return hashlib.sha1(info.encode()).hexdigest()[:12]


def native_lib() -> Path:
    return HERE / "_build" / "native" / _host_tag() / "libkmy_oracle.so"

RECON = {"fog": 0, "plm": 1, "ppm": 2, "wenoz": 3}
LIMITER = {"minmod": 0, "van_leer": 1, "mc": 2}
RIEMANN = {"hll": 0, "hllc": 1}

_dp = ctypes.POINTER(ctypes.c_double)
_lib = None


def build() -> Path:
    """Compile the oracle with its Makefile (g++, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def build_native() -> Path:
    """Compile the host-tuned timing build (-march=native) for this machine."""
    out = native_lib()
    subprocess.run(["make", "-s", "-C", str(HERE), "native", f"NATIVE_DIR={out.parent}"], check=True)
    return out


def lib():
    global _lib
    if _lib is None:
        if use_native:
            path = build_native()
        else:
            if not LIB.exists():
                build()
            path = LIB
        L = ctypes.CDLL(str(path))
        L.kmyo_create.restype = ctypes.c_void_p
        L.kmyo_create.argtypes = [ctypes.c_char_p]
        L.kmyo_destroy.argtypes = [ctypes.c_void_p]
        L.kmyo_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_long)]
        for name in ("kmyo_get", "kmyo_set"):
            f = getattr(L, name)
            f.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, _dp,
                          ctypes.c_long]
        L.kmyo_pgen.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        for name in ("kmyo_fill_ghosts", "kmyo_calc_fluxes", "kmyo_calc_emf",
                     "kmyo_prepare_primitive", "kmyo_fill_derived"):
            getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.kmyo_fluxes_to_dudt.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_char_p]
        L.kmyo_apply_dudt.argtypes = [ctypes.c_void_p] + [ctypes.c_char_p] * 4 + [ctypes.c_double] * 2
        L.kmyo_estimate_dt.restype = ctypes.c_double
        L.kmyo_estimate_dt.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.kmyo_rk_stage.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.kmyo_step.restype = ctypes.c_double
        L.kmyo_step.argtypes = [ctypes.c_void_p]
        L.kmyo_evolve.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.kmyo_time.argtypes = [ctypes.c_void_p, _dp]
        L.kmyo_vortex_error.restype = ctypes.c_double
        L.kmyo_vortex_error.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.kmyo_reconstruct.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp]
        L.kmyo_eos.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp]
        L.kmyo_riemann.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp]
        ip = ctypes.POINTER(ctypes.c_int)
        L.kmyo_blocks.argtypes = [ctypes.c_void_p, ip, ip, ctypes.c_int]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def reconstruct(recon: str, limiter: str, stencil) -> tuple[float, float]:
    s = np.ascontiguousarray(stencil, dtype=np.float64)
    assert s.shape == (5,)
    vm, vp = ctypes.c_double(), ctypes.c_double()
    lib().kmyo_reconstruct(RECON[recon], LIMITER[limiter], _ptr(s), ctypes.byref(vm), ctypes.byref(vp))
    return vm.value, vp.value


def eos(gamma: float, abar: float, mode: str, rho, temp, sie, pres, bmod):
    v = np.array([rho, temp, sie, pres, bmod], dtype=np.float64)
    lib().kmyo_eos(gamma, abar, 0 if mode == "ener" else 1, _ptr(v))
    return dict(rho=v[0], temp=v[1], sie=v[2], pres=v[3], bmod=v[4])


def riemann(solver: str, mhd: bool, direction: int, vL, vR) -> np.ndarray:
    n = 10 if mhd else 7
    a = np.ascontiguousarray(vL, dtype=np.float64)
    b = np.ascontiguousarray(vR, dtype=np.float64)
    assert a.shape == (n,) and b.shape == (n,)
    out = np.zeros(8 if mhd else 5)
    lib().kmyo_riemann(RIEMANN[solver], int(mhd), direction, _ptr(a), _ptr(b), _ptr(out))
    return out


class OracleSim:
    """One mesh, its stage containers and shared primitives, in MeshData layout."""

    INFO = ("ndim", "nb", "nx1", "nx2", "nx3", "ng", "np1", "np2", "np3", "nf1", "nf2", "nf3",
            "ncons", "mhd", "nstages", "nbx1", "nbx2", "nbx3")

    def __init__(self, deck: str):
        self._h = lib().kmyo_create(deck.encode())
        if not self._h:
            raise ValueError("oracle rejected the deck")
        buf = (ctypes.c_long * 32)()
        n = lib().kmyo_info(self._h, buf)
        self.info = dict(zip(self.INFO, buf[:n]))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().kmyo_destroy(self._h)
            self._h = None

    def refresh(self) -> None:
        """Re-read the mesh description (the block count changes on an adaptive mesh)."""
        buf = (ctypes.c_long * 32)()
        n = lib().kmyo_info(self._h, buf)
        self.info = dict(zip(self.INFO, buf[:n]))

    def blocks(self):
        """(levels, locations) of the leaf blocks in block order."""
        self.refresh()
        nb = self.info["nb"]
        lev = (ctypes.c_int * nb)()
        loc = (ctypes.c_int * (3 * nb))()
        lib().kmyo_blocks(self._h, lev, loc, nb)
        return np.array(lev[:]), np.array(loc[:]).reshape(nb, 3)

    @property
    def cell_shape(self):
        self.refresh()
        i = self.info
        return (i["nb"], i["np3"], i["np2"], i["np1"])

    @property
    def face_shape(self):
        self.refresh()
        i = self.info
        return (i["nb"], i["nf3"], i["nf2"], i["nf1"])

    def _shape(self, var):
        return self.face_shape if var in ("mag", "flux", "emf") else self.cell_shape

    def get(self, var: str, comp: int = 0, container: str = "base") -> np.ndarray:
        out = np.empty(self._shape(var), dtype=np.float64)
        rc = lib().kmyo_get(self._h, container.encode(), var.encode(), comp, _ptr(out), out.size)
        if rc:
            raise KeyError(var)
        return out

    def set(self, var: str, arr, comp: int = 0, container: str = "base") -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        rc = lib().kmyo_set(self._h, container.encode(), var.encode(), comp, _ptr(a), a.size)
        if rc:
            raise KeyError(var)

    def pgen(self, problem: str) -> None:
        if lib().kmyo_pgen(self._h, problem.encode()):
            raise ValueError(problem)

    def step(self) -> float:
        return lib().kmyo_step(self._h)

    def evolve(self, tlim: float, nlim: int = -1) -> int:
        return lib().kmyo_evolve(self._h, tlim, nlim)

    def rk_stage(self, stage: int, dt: float) -> None:
        lib().kmyo_rk_stage(self._h, stage, dt)

    def estimate_dt(self, container: str = "base") -> float:
        return lib().kmyo_estimate_dt(self._h, container.encode())

    def fill_ghosts(self, container: str = "base") -> None:
        lib().kmyo_fill_ghosts(self._h, container.encode())

    def prepare_primitive(self, container: str = "base") -> None:
        lib().kmyo_prepare_primitive(self._h, container.encode())

    def fill_derived(self, container: str = "base") -> None:
        lib().kmyo_fill_derived(self._h, container.encode())

    @property
    def time(self) -> dict:
        out = np.zeros(4)
        lib().kmyo_time(self._h, _ptr(out))
        return dict(time=out[0], dt=out[1], dt_est=out[2], ncycle=int(out[3]))

    def vortex_error(self, var: str = "dens", comp: int = 0) -> float:
        v = {"dens": 0, "velocity": 1, "pres": 2, "magc": 3}[var]
        return lib().kmyo_vortex_error(self._h, v, comp)

    def interior(self, arr: np.ndarray) -> np.ndarray:
        i = self.info
        g1 = i["ng"]
        g2 = i["ng"] if i["ndim"] > 1 else 0
        g3 = i["ng"] if i["ndim"] > 2 else 0
        return arr[:, g3:g3 + i["nx3"], g2:g2 + i["nx2"], g1:g1 + i["nx1"]]


def deck_text(blocks: dict) -> str:
    """Render {"block": {"key": value}} as a Parthenon input deck."""
    lines = []
    for block, kv in blocks.items():
        lines.append(f"<{block}>")
        for k, v in kv.items():
            lines.append(f"{k} = {v}")
        lines.append("")
    return "\n".join(lines)


def cpu_threads() -> int:
    return len(os.sched_getaffinity(0))
