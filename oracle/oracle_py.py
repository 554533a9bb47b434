"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle restates the STREAmS-2 CPU backend time advance (see oracle/oracle.hpp); tests,
the smoke check and bench.py's CPU-baseline leg use it as the checker, never as the product.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"


def _load():
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} missing: run `make -C oracle`")
    lib = C.CDLL(str(LIB_PATH))
    P, D, I = C.c_void_p, C.POINTER(C.c_double), C.c_int
    sig = {
        "oracle_error": (C.c_char_p, []),
        "oracle_create": (P, [C.c_char_p, C.c_char_p]),
        "oracle_destroy": (None, [P]),
        "oracle_init_run": (None, [P]),
        "oracle_step": (None, [P]),
        "oracle_run": (None, [P, I]),
        "oracle_rk_sync": (None, [P]),
        "oracle_compute_dt": (None, [P]),
        "oracle_set_dt": (None, [P, C.c_double]),
        "oracle_face_flux": (None, [P, I, C.POINTER(C.c_int), D]),
        "oracle_face_flops": (None, [P, I, I, I, I, C.POINTER(C.c_longlong)]),
        "oracle_compute_residual": (None, [P]),
        "oracle_sizes": (None, [P, C.POINTER(C.c_int)]),
        "oracle_get_w": (None, [P, D]),
        "oracle_set_w": (None, [P, D]),
        "oracle_get_waux": (None, [P, D]),
        "oracle_get_fl": (None, [P, D]),
        "oracle_get_fln": (None, [P, D]),
        "oracle_get_wallprop": (None, [P, D]),
        "oracle_get_scalars": (None, [P, D]),
        "oracle_last_progress": (I, [P, D]),
        "oracle_get_residual": (None, [P, D]),
        "oracle_case_info": (None, [P, D]),
        "oracle_compute_stats": (None, [P, I]),
        "oracle_compute_stats_3d": (None, [P, I]),
        "oracle_set_stats": (None, [P, I, D]),
        "oracle_get_stats": (None, [P, I, D]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    def __init__(self, directory: str | os.PathLike = ".", ini_text: str | None = None):
        h = lib.oracle_create(str(directory).encode(), (ini_text or "").encode())
        if not h:
            raise RuntimeError("oracle: " + lib.oracle_error().decode())
        self._h = h
        s = (C.c_int * 4)()
        lib.oracle_sizes(h, s)
        self.nx, self.ny, self.nz, self.ng = list(s)

    def __del__(self):
        if getattr(self, "_h", None):
            lib.oracle_destroy(self._h)
            self._h = None

    @property
    def gshape(self):
        g = self.ng
        return (5, self.nz + 2 * g, self.ny + 2 * g, self.nx + 2 * g)

    def init_run(self):
        lib.oracle_init_run(self._h)

    def step(self):
        lib.oracle_step(self._h)

    def run(self, n: int):
        lib.oracle_run(self._h, n)

    def rk_sync(self):
        lib.oracle_rk_sync(self._h)

    def compute_dt(self):
        lib.oracle_compute_dt(self._h)

    def set_dt(self, dt: float):
        lib.oracle_set_dt(self._h, dt)

    def w(self) -> np.ndarray:
        a = np.zeros(self.gshape)
        lib.oracle_get_w(self._h, _d(a))
        return a

    def set_w(self, w: np.ndarray):
        w = np.ascontiguousarray(w, dtype=np.float64)
        lib.oracle_set_w(self._h, _d(w))

    def waux(self) -> np.ndarray:
        g = self.ng
        a = np.zeros((10, self.nz + 2 * g, self.ny + 2 * g, self.nx + 2 * g))
        lib.oracle_get_waux(self._h, _d(a))
        return a

    def face_flux(self, faces: np.ndarray) -> np.ndarray:
        """fhat at the faces (dir, i, j, k), one row each, from the current w_aux: (n, 5)."""
        f = np.ascontiguousarray(faces, dtype=np.int32).reshape(-1, 4)
        out = np.zeros((f.shape[0], 5))
        lib.oracle_face_flux(self._h, f.shape[0], f.ctypes.data_as(C.POINTER(C.c_int)), _d(out))
        return out

    def face_flops(self, direction: int, i: int, j: int, k: int) -> dict:
        """FP64 operations of one face flux as the oracle's code performs them (flops.hpp)."""
        out = (C.c_longlong * 6)()
        lib.oracle_face_flops(self._h, direction, i, j, k, out)
        names = ["add", "mul", "div", "sqrt", "special", "cmp"]
        d = dict(zip(names, list(out)))
        d["flops"] = d["add"] + d["mul"] + d["div"] + d["sqrt"] + d["special"]
        return d

    def fl(self) -> np.ndarray:
        a = np.zeros((5, self.nz, self.ny, self.nx))
        lib.oracle_get_fl(self._h, _d(a))
        return a

    def wallprop(self) -> np.ndarray:
        g = self.ng
        a = np.zeros((3, self.nz + 2 * g, self.nx + 2 * g))
        lib.oracle_get_wallprop(self._h, _d(a))
        return a[:, g:g + self.nz, g:g + self.nx]

    def scalars(self) -> dict:
        a = np.zeros(7)
        lib.oracle_get_scalars(self._h, _d(a))
        return dict(zip(["dt", "time", "dpdx", "rhobulk", "ubulk", "tbulk", "icyc"], a.tolist()))

    def last_progress(self):
        a = np.zeros(14)
        ok = lib.oracle_last_progress(self._h, _d(a))
        return a if ok else None

    def residual(self) -> dict:
        lib.oracle_compute_residual(self._h)
        a = np.zeros(7)
        lib.oracle_get_residual(self._h, _d(a))
        return dict(zip(["residual_rhou", "rhomin", "rhomax", "tmin", "tmax", "pmin", "pmax"], a.tolist()))

    def case_info(self) -> dict:
        a = np.zeros(8)
        lib.oracle_case_info(self._h, _d(a))
        return dict(zip(["u0", "rho0", "l0", "mu0", "volchan", "t_bulk_target", "num_iter", "print_control"],
                        a.tolist()))

    def compute_stats(self, itav: int):
        lib.oracle_compute_stats(self._h, itav)

    def compute_stats_3d(self, itav: int):
        lib.oracle_compute_stats_3d(self._h, itav)

    def _stats_shape(self, which: int):
        return (self.ny, self.nx, 70) if which in (0, 1) else (self.nz, self.ny, self.nx, 14)

    def stats(self, which: int = 0) -> np.ndarray:
        """w_stat (0), w_stat_z (1) as (ny, nx, 70) or w_stat_3d (2) as (nz, ny, nx, 14) arrays."""
        a = np.zeros(self._stats_shape(which))
        lib.oracle_get_stats(self._h, which, _d(a))
        return a

    def set_stats(self, which: int, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(self._stats_shape(which))
        lib.oracle_set_stats(self._h, which, _d(a))
