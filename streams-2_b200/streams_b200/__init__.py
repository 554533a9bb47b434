"""Python binding of the B200 backend C ABI (ctypes).

This is a thin host-side mirror of the solver-object interface of STREAmS-2
(``equation_singleideal_<backend>_object``, code/src/singleideal/singleideal_cpu.F90:99-135):
``Solver`` wraps one device context and exposes ``init_run``, ``compute_dt``, ``rk_sync``,
``compute_residual``, ``copy_from_field``/``copy_to_field`` and a no-sync ``advance`` loop;
``Case`` wraps the host set-up of a ``singleideal.ini`` case.  All compute happens in the
compiled library ``lib/libstreams_b200.so``, mapped on the first call into it; that call fails
loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_DEFAULT_LIB = _HERE.parent / "lib" / "libstreams_b200.so"
# STREAMS_B200_LIB selects another build of the same library (for example one compiled with
# different launch bounds); the default is the in-tree build.
LIB_PATH = Path(os.environ.get("STREAMS_B200_LIB", str(_DEFAULT_LIB)))

OK, EINVAL, ECUDA, ENOMEM, ENAN, ETIMEOUT, ENODEV = 0, -1, -2, -3, -4, -5, -6


class Params(C.Structure):
    """Mirror of ``streams_b200_params`` (include/streams_b200.h)."""

    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("ng", C.c_int),
        ("ep_order", C.c_int), ("nkeep", C.c_int), ("weno_scheme", C.c_int), ("weno_version", C.c_int),
        ("flux_splitting", C.c_int), ("conservative_viscous", C.c_int),
        ("sensor_threshold", C.c_double),
        ("bctags", C.c_int * 6), ("force_zero_flux", C.c_int * 6),
        ("eul_imin", C.c_int), ("eul_imax", C.c_int), ("eul_jmin", C.c_int),
        ("eul_jmax", C.c_int), ("eul_kmin", C.c_int), ("eul_kmax", C.c_int),
        ("is_y_staggered", C.c_int),
        ("visc_model", C.c_int), ("calorically_perfect", C.c_int),
        ("mu0", C.c_double), ("t0", C.c_double), ("rgas0", C.c_double), ("rho0", C.c_double),
        ("u0", C.c_double), ("l0", C.c_double),
        ("sutherland_s", C.c_double), ("t_ref_dim", C.c_double), ("powerlaw_vtexp", C.c_double),
        ("prandtl", C.c_double),
        ("cp0", C.c_double), ("cv0", C.c_double), ("cp_last", C.c_double), ("cv_last", C.c_double),
        ("channel_case", C.c_int),
        ("theta_wall", C.c_double), ("t_wall", C.c_double), ("t_bulk_target", C.c_double),
        ("volchan", C.c_double),
        ("nrk", C.c_int),
        ("rhork", C.c_double * 4), ("gamrk", C.c_double * 4),
        ("cfl", C.c_double),
        ("precision", C.c_int),
        ("bctags_nr", C.c_int * 6), ("winf", C.c_double * 5), ("p0", C.c_double),
        ("recyc", C.c_int), ("i_recyc", C.c_int), ("jbl_inflow", C.c_int),
        ("betarecyc", C.c_double), ("rng_seed", C.c_uint), ("rng_draws", C.c_longlong),
        ("xshock_imp", C.c_double), ("shock_angle", C.c_double), ("tanhfacs", C.c_double),
        ("winf_past_shock", C.c_double * 5),
        ("indx_cp_l", C.c_int), ("indx_cp_r", C.c_int),
        ("cp_coeff", C.c_double * 12), ("cv_coeff", C.c_double * 12),
    ]


class Grid(C.Structure):
    """Mirror of ``streams_b200_grid``."""

    _fields_ = [(n, C.POINTER(C.c_double)) for n in
                ("x", "y", "z", "yn", "dcsidx", "detady", "dzitdz", "dcsidxs", "detadys", "dzitdzs",
                 "coeff_deriv1")] + [(n, C.POINTER(C.c_int)) for n in ("ep_ord_x", "ep_ord_y", "ep_ord_z")] + \
        [(n, C.POINTER(C.c_double)) for n in ("dcsidx2", "detady2", "dzitdz2", "coeff_deriv2",
                                               "wmean_inflow", "yplus_inflow", "eta_inflow", "yplus_recyc",
                                               "eta_recyc", "weta_inflow")] + \
        [(n, C.POINTER(C.c_int)) for n in ("map_j_inn", "map_j_out")]


class BackendError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"streams_b200 error {code}: {msg}")
        self.code = code


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C streams-2_b200` "
                          "(or __graft_entry__.build()); there is no CPU fallback")
    lib = C.CDLL(str(LIB_PATH))
    P, V, D, I, LL = C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_longlong
    sig = {
        "streams_b200_abi_version": (I, []),
        "streams_b200_global_error": (C.c_char_p, []),
        "streams_b200_create": (I, [C.POINTER(Params), C.POINTER(Grid), C.POINTER(P)]),
        "streams_b200_destroy": (I, [P]),
        "streams_b200_last_error": (C.c_char_p, [P]),
        "streams_b200_footprint_bytes": (LL, [C.POINTER(Params)]),
        "streams_b200_copy_from_field": (I, [P, D]),
        "streams_b200_copy_to_field": (I, [P, D]),
        "streams_b200_copy_from_device": (I, [P, V]),
        "streams_b200_copy_to_device": (I, [P, V]),
        "streams_b200_init_run": (I, [P]),
        "streams_b200_compute_dt": (I, [P, D]),
        "streams_b200_set_dt": (I, [P, C.c_double]),
        "streams_b200_set_time": (I, [P, C.c_double]),
        "streams_b200_rk_sync": (I, [P]),
        "streams_b200_advance": (I, [P, I, I, I, I]),
        "streams_b200_get_scalars": (I, [P, D]),
        "streams_b200_compute_residual": (I, [P, D]),
        "streams_b200_count_weno": (I, [P, D]),
        "streams_b200_get_wallprop": (I, [P, D]),
        "streams_b200_compute_stats": (I, [P, I]),
        "streams_b200_compute_stats_3d": (I, [P, I]),
        "streams_b200_get_stats": (I, [P, I, D, LL]),
        "streams_b200_set_stats": (I, [P, I, D, LL]),
        "streams_b200_synchronize": (I, [P]),
        "streams_b200_query": (I, [P]),
        "streams_b200_launch_count": (LL, [P]),
        "streams_b200_debug_fetch": (I, [P, I, D, LL]),
        "streams_b200_get_stream": (I, [P, C.POINTER(P)]),
        "streams_b200_profile_enable": (I, [P, I]),
        "streams_b200_profile_read": (I, [P, I, D, C.POINTER(LL)]),
        "streams_b200_kernel_count": (I, []),
        "streams_b200_kernel_name": (C.c_char_p, [I]),
        "streams_b200_kernel_binary_versions": (I, [C.POINTER(C.c_int), I]),
        "streams_b200_compute_dt_noalloc": (I, [I, I, I, I] + [V] * 8 + [C.c_double] * 4 + [V, V]),
        "streams_b200_case_load": (I, [C.c_char_p, C.c_char_p, C.POINTER(P)]),
        "streams_b200_case_free": (I, [P]),
        "streams_b200_case_error": (C.c_char_p, []),
        "streams_b200_case_params": (I, [P, I, C.POINTER(Params)]),
        "streams_b200_case_grid": (I, [P, C.POINTER(Grid)]),
        "streams_b200_case_field": (D, [P]),
        "streams_b200_case_info": (I, [P, D]),
        "streams_b200_case_write_restart": (I, [P, C.c_char_p]),
        "streams_b200_case_write_state": (I, [P, D, I, C.c_double, C.c_char_p]),
        "streams_b200_run_case": (I, [P, I, I, C.c_char_p, D, D]),
        "streams_b200_run_case_stats": (I, [P, I, I, C.c_char_p, D, D, D, D, D, C.c_char_p]),
        "streams_b200_case_write_state_stats": (I, [P, D, I, C.c_double, D, D, I, C.c_double, C.c_char_p]),
        "streams_b200_case_stats_info": (I, [P, D]),
        "streams_b200_case_stats": (I, [P, I, D, LL]),
        "streams_b200_set_tuning": (I, [P, LL, I]),
        "streams_b200_get_tuning": (I, [P, C.POINTER(LL), C.POINTER(I)]),
        "streams_b200_set_weno_split": (I, [P, C.c_double]),
        "streams_b200_get_weno_split": (I, [P, D]),
        "streams_b200_batch_create": (I, [C.POINTER(P), I, I, I, C.POINTER(P)]),
        "streams_b200_batch_advance": (I, [P, I]),
        "streams_b200_batch_synchronize": (I, [P]),
        "streams_b200_batch_invalidate": (I, [P]),
        "streams_b200_batch_stats": (I, [P, C.POINTER(LL), C.POINTER(LL)]),
        "streams_b200_batch_set_shared_launches": (I, [P, I]),
        "streams_b200_batch_class": (I, [P, C.POINTER(LL)]),
        "streams_b200_batch_groups": (I, [P, C.POINTER(I), C.POINTER(I)]),
        "streams_b200_batch_last_error": (C.c_char_p, [P]),
        "streams_b200_batch_destroy": (I, [P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


class _Library:
    """The compiled library, mapped on first use: importing the package (for example for the
    input-file builders of ``streams_b200.cases``) maps no shared object, and the first call
    into the C ABI fails loudly when the library is missing.  There is no CPU fallback."""

    def __init__(self):
        self._cdll = None

    def _get(self) -> C.CDLL:
        if self._cdll is None:
            self._cdll = _load()
        return self._cdll

    def __getattr__(self, name):
        return getattr(self._get(), name)


lib = _Library()

# Every symbol the C headers declare (checked by the CPU test suite).
EXPORTED = [
    "streams_b200_abi_version", "streams_b200_global_error", "streams_b200_create", "streams_b200_destroy",
    "streams_b200_last_error", "streams_b200_footprint_bytes", "streams_b200_copy_from_field",
    "streams_b200_copy_to_field", "streams_b200_copy_from_device", "streams_b200_copy_to_device",
    "streams_b200_init_run", "streams_b200_compute_dt", "streams_b200_set_dt", "streams_b200_rk_sync",
    "streams_b200_advance", "streams_b200_get_scalars", "streams_b200_set_time", "streams_b200_compute_residual",
    "streams_b200_count_weno", "streams_b200_get_wallprop", "streams_b200_synchronize", "streams_b200_query",
    "streams_b200_compute_stats", "streams_b200_compute_stats_3d", "streams_b200_get_stats",
    "streams_b200_set_stats",
    "streams_b200_launch_count", "streams_b200_debug_fetch", "streams_b200_get_stream",
    "streams_b200_profile_enable", "streams_b200_profile_read", "streams_b200_kernel_count",
    "streams_b200_kernel_name", "streams_b200_kernel_binary_versions", "streams_b200_compute_dt_noalloc", "streams_b200_case_load", "streams_b200_case_free", "streams_b200_case_error",
    "streams_b200_case_params", "streams_b200_case_grid", "streams_b200_case_field", "streams_b200_case_info",
    "streams_b200_case_write_restart", "streams_b200_case_write_state", "streams_b200_run_case",
    "streams_b200_run_case_stats", "streams_b200_case_write_state_stats", "streams_b200_case_stats_info",
    "streams_b200_case_stats",
    "streams_b200_set_tuning",
    "streams_b200_get_tuning", "streams_b200_set_weno_split", "streams_b200_get_weno_split",
    "streams_b200_batch_create", "streams_b200_batch_advance",
    "streams_b200_batch_synchronize", "streams_b200_batch_invalidate", "streams_b200_batch_stats",
    "streams_b200_batch_set_shared_launches", "streams_b200_batch_groups", "streams_b200_batch_class",
    "streams_b200_batch_last_error", "streams_b200_batch_destroy",
]


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Case:
    """Host set-up of a case (``singleideal.ini`` in ``directory`` or ``ini_text``)."""

    def __init__(self, directory: str | os.PathLike = ".", ini_text: str | None = None):
        h = C.c_void_p()
        rc = lib.streams_b200_case_load(str(directory).encode(), (ini_text or "").encode(), C.byref(h))
        if rc != OK:
            raise BackendError(rc, lib.streams_b200_case_error().decode())
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.streams_b200_case_free(h)
            self._h = None

    def params(self, precision: int = 0) -> Params:
        p = Params()
        lib.streams_b200_case_params(self._h, precision, C.byref(p))
        return p

    def grid(self) -> Grid:
        g = Grid()
        lib.streams_b200_case_grid(self._h, C.byref(g))
        return g

    @property
    def shape(self):
        p = self.params()
        return p.nx, p.ny, p.nz, p.ng

    def field(self) -> np.ndarray:
        """Initial conserved field as an array w[m, k, j, i] (ghosts included; a copy)."""
        nx, ny, nz, ng = self.shape
        n = (nx + 2 * ng) * (ny + 2 * ng) * (nz + 2 * ng) * 5
        ptr = lib.streams_b200_case_field(self._h)
        a = np.ctypeslib.as_array(ptr, shape=(n,)).copy()
        return a.reshape(5, nz + 2 * ng, ny + 2 * ng, nx + 2 * ng)

    def info(self) -> dict:
        out = np.zeros(12)
        lib.streams_b200_case_info(self._h, _dptr(out))
        keys = ["u0", "rho0", "l0", "mu0", "num_iter", "print_control", "iter_dt_recompute", "icyc0", "time0",
                "cfl", "volchan", "t_bulk_target"]
        return dict(zip(keys, out.tolist()))

    def write_restart(self, directory: str | os.PathLike) -> None:
        rc = lib.streams_b200_case_write_restart(self._h, str(directory).encode())
        if rc != OK:
            raise BackendError(rc, lib.streams_b200_case_error().decode())

    def write_state(self, w: np.ndarray, icyc: int, time: float, directory: str | os.PathLike) -> None:
        """Restart files (rst.bin, field_info0.dat, grid files, singleideal.ini with
        restart_type = 1) of the field w at step icyc and time; Case(directory) resumes it."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        nx, ny, nz, ng = self.shape
        if w.shape != (5, nz + 2 * ng, ny + 2 * ng, nx + 2 * ng):
            raise ValueError("w must be the ghosted field of this case")
        rc = lib.streams_b200_case_write_state(self._h, _dptr(w), int(icyc), float(time), str(directory).encode())
        if rc != OK:
            raise BackendError(rc, lib.streams_b200_case_error().decode())

    def run(self, nsteps: int = -1, precision: int = 0, progress_path: str | None = None,
            return_field: bool = False):
        """The solver's run() loop on the device; returns (last progress row, final field or None)."""
        row = np.zeros(14)
        w = None
        if return_field:
            nx, ny, nz, ng = self.shape
            w = np.zeros((5, nz + 2 * ng, ny + 2 * ng, nx + 2 * ng))
        rc = lib.streams_b200_run_case(self._h, nsteps, precision,
                                       progress_path.encode() if progress_path else None,
                                       _dptr(row), _dptr(w) if w is not None else None)
        if rc != OK:
            raise BackendError(rc, lib.streams_b200_case_error().decode())
        return row, w

    def stats_info(self) -> dict:
        """[output] statistics settings and the restart's averaging clock."""
        out = np.zeros(5)
        lib.streams_b200_case_stats_info(self._h, _dptr(out))
        return dict(zip(["dtstat", "enable_stat_time", "enable_stat_3d", "itav", "time_from_last_stat"],
                        out.tolist()))

    def restart_stats(self, which: int = 0) -> np.ndarray:
        """Averages read on a restart_type = 2 restart (zeros otherwise): w_stat as (ny, nx, 70),
        w_stat_3d (which = 2) as (nz, ny, nx, 14)."""
        nx, ny, nz, _ = self.shape
        shape = (ny, nx, 70) if which == 0 else (nz, ny, nx, 14)
        out = np.zeros(shape)
        rc = lib.streams_b200_case_stats(self._h, which, _dptr(out), out.size)
        if rc != OK:
            raise BackendError(rc, "case statistics: which must be 0 or 2")
        return out

    def write_state_stats(self, w: np.ndarray, icyc: int, time: float, w_stat: np.ndarray | None,
                          w_stat_3d: np.ndarray | None, itav: int, time_from_last_stat: float,
                          directory: str | os.PathLike) -> None:
        """write_state plus stat.bin / stat3d.bin and the averaging clock (restart_type = 2)."""
        w = np.ascontiguousarray(w, dtype=np.float64)
        a2 = None if w_stat is None else np.ascontiguousarray(w_stat, dtype=np.float64)
        a3 = None if w_stat_3d is None else np.ascontiguousarray(w_stat_3d, dtype=np.float64)
        rc = lib.streams_b200_case_write_state_stats(
            self._h, _dptr(w), int(icyc), float(time), _dptr(a2) if a2 is not None else None,
            _dptr(a3) if a3 is not None else None, int(itav), float(time_from_last_stat), str(directory).encode())
        if rc != OK:
            raise BackendError(rc, lib.streams_b200_case_error().decode())

    def run_stats(self, nsteps: int = -1, precision: int = 0, progress_path: str | None = None,
                  output_dir: str | os.PathLike | None = None) -> dict:
        """run() with the statistics of [output] dtstat: returns the last progress row, the final
        field, w_stat (ny, nx, 70), w_stat_3d (nz, ny, nx, 14) and the averaging clock; with
        output_dir the end-of-run files are written there."""
        nx, ny, nz, ng = self.shape
        row = np.zeros(14)
        w = np.zeros((5, nz + 2 * ng, ny + 2 * ng, nx + 2 * ng))
        s2 = np.zeros((ny, nx, 70))
        info = self.stats_info()
        s3 = np.zeros((nz, ny, nx, 14)) if info["enable_stat_3d"] > 0 else None
        clock = np.zeros(2)
        rc = lib.streams_b200_run_case_stats(
            self._h, nsteps, precision, progress_path.encode() if progress_path else None, _dptr(row), _dptr(w),
            _dptr(s2), _dptr(s3) if s3 is not None else None, _dptr(clock),
            str(output_dir).encode() if output_dir is not None else None)
        if rc != OK:
            raise BackendError(rc, lib.streams_b200_case_error().decode())
        return {"row": row, "w": w, "w_stat": s2, "w_stat_3d": s3, "itav": int(clock[0]),
                "time_from_last_stat": float(clock[1])}


class Solver:
    """One device context: the B200 counterpart of the backend solver object."""

    def __init__(self, params: Params, grid: Grid, keepalive=None):
        self._keep = keepalive
        h = C.c_void_p()
        rc = lib.streams_b200_create(C.byref(params), C.byref(grid), C.byref(h))
        if rc != OK:
            raise BackendError(rc, lib.streams_b200_global_error().decode())
        self._h = h
        self.params = params
        self.shape = (params.nx, params.ny, params.nz, params.ng)

    @classmethod
    def from_case(cls, case: Case, precision: int = 0) -> "Solver":
        s = cls(case.params(precision), case.grid(), keepalive=case)
        # upload the case's initial field straight from the set-up's own buffer
        s._check(lib.streams_b200_copy_from_field(s._h, lib.streams_b200_case_field(case._h)))
        s.synchronize()
        return s

    def copy_from_host_ptr(self, ptr: int) -> None:
        """Upload w from a host address (e.g. a pinned buffer); asynchronous on the context stream."""
        self._check(lib.streams_b200_copy_from_field(self._h, C.cast(C.c_void_p(ptr), C.POINTER(C.c_double))))

    def copy_to_host_ptr(self, ptr: int) -> None:
        """Download w (ghosts rebuilt) to a host address; returns after the copy completed."""
        self._check(lib.streams_b200_copy_to_field(self._h, C.cast(C.c_void_p(ptr), C.POINTER(C.c_double))))

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            lib.streams_b200_destroy(h)
            self._h = None

    __del__ = close

    def _check(self, rc: int):
        if rc != OK:
            raise BackendError(rc, lib.streams_b200_last_error(self._h).decode())

    def copy_from_field(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, dtype=np.float64)
        self._check(lib.streams_b200_copy_from_field(self._h, _dptr(w)))
        self._sync_keep = w  # the copy is asynchronous: keep the host buffer alive
        self.synchronize()

    def copy_to_field(self) -> np.ndarray:
        nx, ny, nz, ng = self.shape
        w = np.zeros((5, nz + 2 * ng, ny + 2 * ng, nx + 2 * ng))
        self._check(lib.streams_b200_copy_to_field(self._h, _dptr(w)))
        return w

    def init_run(self):
        self._check(lib.streams_b200_init_run(self._h))

    def compute_dt(self) -> float:
        dt = C.c_double()
        self._check(lib.streams_b200_compute_dt(self._h, C.byref(dt)))
        return dt.value

    def set_dt(self, dt: float):
        self._check(lib.streams_b200_set_dt(self._h, dt))

    def set_time(self, t: float):
        self._check(lib.streams_b200_set_time(self._h, t))

    def rk_sync(self):
        self._check(lib.streams_b200_rk_sync(self._h))

    def advance(self, nsteps: int, iter_dt_recompute: int = 1, icyc_start: int = 0, icyc0: int = 0):
        self._check(lib.streams_b200_advance(self._h, nsteps, iter_dt_recompute, icyc_start, icyc0))

    def scalars(self) -> dict:
        out = np.zeros(7)
        self._check(lib.streams_b200_get_scalars(self._h, _dptr(out)))
        return dict(zip(["dt", "time", "dpdx", "rhobulk", "ubulk", "tbulk", "tbdiff"], out.tolist()))

    def compute_residual(self) -> dict:
        out = np.zeros(7)
        rc = lib.streams_b200_compute_residual(self._h, _dptr(out))
        if rc not in (OK, ENAN):
            self._check(rc)
        d = dict(zip(["residual_rhou", "rhomin", "rhomax", "tmin", "tmax", "pmin", "pmax"], out.tolist()))
        d["nan"] = rc == ENAN
        return d

    def count_weno(self):
        out = np.zeros(3)
        self._check(lib.streams_b200_count_weno(self._h, _dptr(out)))
        return out

    def wallprop(self) -> np.ndarray:
        nx, ny, nz, ng = self.shape
        out = np.zeros(3 * nx * nz)
        self._check(lib.streams_b200_get_wallprop(self._h, _dptr(out)))
        return out.reshape(3, nz, nx)

    def synchronize(self):
        self._check(lib.streams_b200_synchronize(self._h))

    def batch_class(self) -> int | None:
        """Class for shared launches in a Batch (solvers of one class form a group), or None
        for a solver that always advances on its own branch."""
        k = C.c_longlong()
        self._check(lib.streams_b200_batch_class(self._h, C.byref(k)))
        return None if k.value < 0 else int(k.value)

    def busy(self) -> bool:
        """Whether work issued on the context's stream is still pending (non-blocking)."""
        rc = lib.streams_b200_query(self._h)
        if rc < 0:
            self._check(rc)
        return rc == 1

    NV_STAT, NV_STAT_3D = 70, 14

    def compute_stats(self, itav: int) -> None:
        """compute_stats after a step: fold the step's z-averaged statistics into w_stat, which
        already averages itav samples (manage_output then increments itav)."""
        self._check(lib.streams_b200_compute_stats(self._h, int(itav)))

    def compute_stats_3d(self, itav: int) -> None:
        """compute_stats_3d after a step: the 14 point statistics averaged in time."""
        self._check(lib.streams_b200_compute_stats_3d(self._h, int(itav)))

    def _stats_shape(self, which: int):
        nx, ny, nz, _ = self.shape
        if which in (0, 1):
            return (ny, nx, self.NV_STAT)
        if which == 2:
            return (nz, ny, nx, self.NV_STAT_3D)
        raise ValueError("which: 0 w_stat, 1 w_stat_z, 2 w_stat_3d")

    def stats(self, which: int = 0) -> np.ndarray:
        """w_stat (0) or w_stat_z (1) as (ny, nx, 70) arrays, w_stat_3d (2) as (nz, ny, nx, 14):
        the reference's Fortran arrays w_stat(70, nx, ny) ... with the index order reversed."""
        out = np.zeros(self._stats_shape(which))
        self._check(lib.streams_b200_get_stats(self._h, which, _dptr(out), out.size))
        return out

    def set_stats(self, which: int, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(self._stats_shape(which))
        self._check(lib.streams_b200_set_stats(self._h, which, _dptr(a), a.size))

    def debug_fetch(self, which: int) -> np.ndarray:
        """Internal arrays: 0 aux (7 ghosted), 1 last stage RHS fl (5), 2 sensor, 3 div/3."""
        nx, ny, nz, ng = self.shape
        gs = (nz + 2 * ng, ny + 2 * ng, nx + 2 * ng)
        shapes = {0: (7,) + gs, 1: (5, nz, ny, nx), 2: (nz, ny, nx), 3: (nz, ny, nx)}
        out = np.zeros(shapes[which])
        self._check(lib.streams_b200_debug_fetch(self._h, which, _dptr(out), out.size))
        return out

    @property
    def stream_handle(self) -> int:
        """The context's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        h = C.c_void_p()
        self._check(lib.streams_b200_get_stream(self._h, C.byref(h)))
        return int(h.value or 0)

    def profile(self, on: int):
        self._check(lib.streams_b200_profile_enable(self._h, on))

    def profile_report(self) -> dict:
        """{kernel name: (total device ms, launches)} from the event profiler."""
        out = {}
        for kid in range(lib.streams_b200_kernel_count()):
            ms, n = C.c_double(), C.c_longlong()
            self._check(lib.streams_b200_profile_read(self._h, kid, C.byref(ms), C.byref(n)))
            if n.value:
                out[lib.streams_b200_kernel_name(kid).decode()] = (ms.value, int(n.value))
        return out

    @property
    def launches(self) -> int:
        return int(lib.streams_b200_launch_count(self._h))

    def set_tuning(self, march_threads: int, march_minseg: int) -> None:
        """Launch shape of the y/z flux passes (see streams_b200_set_tuning)."""
        self._check(lib.streams_b200_set_tuning(self._h, int(march_threads), int(march_minseg)))

    def get_tuning(self) -> tuple[int, int]:
        t, m = C.c_longlong(), C.c_int()
        self._check(lib.streams_b200_get_tuning(self._h, C.byref(t), C.byref(m)))
        return int(t.value), int(m.value)

    def set_weno_split(self, max_fraction: float) -> None:
        """Largest WENO face fraction of a direction at which its hybrid pass reads the WENO
        faces from the face buffer (see streams_b200_set_weno_split): 0 keeps them in the hybrid
        passes, 1 always computes them apart."""
        self._check(lib.streams_b200_set_weno_split(self._h, float(max_fraction)))

    def get_weno_split(self) -> float:
        v = np.zeros(1)
        self._check(lib.streams_b200_get_weno_split(self._h, _dptr(v)))
        return float(v[0])


class Batch:
    """Many independent solvers advanced together through one CUDA graph per replay.

    Every solver keeps its own fields, stream and flow parameters; the graph holds each box's
    step sequence as a parallel branch, so small boxes share the GPU instead of running one
    after another.  Results equal advancing each solver alone with the same tuning.
    """

    def __init__(self, solvers, steps_per_graph: int = 10, dt_every: int = 1):
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[s._h for s in self.solvers])
        h = C.c_void_p()
        rc = lib.streams_b200_batch_create(arr, len(self.solvers), steps_per_graph, dt_every, C.byref(h))
        if rc != OK:
            raise BackendError(rc, lib.streams_b200_global_error().decode())
        self._h = h
        self.steps_per_graph = steps_per_graph

    def _check(self, rc: int):
        if rc != OK:
            raise BackendError(rc, lib.streams_b200_batch_last_error(self._h).decode())

    def advance(self, nsteps: int) -> None:
        """Advance every box by nsteps (asynchronous)."""
        self._check(lib.streams_b200_batch_advance(self._h, int(nsteps)))

    def synchronize(self) -> None:
        self._check(lib.streams_b200_batch_synchronize(self._h))

    def invalidate(self) -> None:
        self._check(lib.streams_b200_batch_invalidate(self._h))

    def stats(self) -> tuple[int, int]:
        """(graph replays so far, kernel launches per replay)."""
        r, n = C.c_longlong(), C.c_longlong()
        self._check(lib.streams_b200_batch_stats(self._h, C.byref(r), C.byref(n)))
        return int(r.value), int(n.value)

    def set_shared_launches(self, groups_per_class: int) -> None:
        """Boxes of a class advance by shared launches in ``groups_per_class`` groups (1, the
        default), or each on its own branch (0)."""
        self._check(lib.streams_b200_batch_set_shared_launches(self._h, int(groups_per_class)))

    def groups(self) -> tuple[int, int]:
        """(groups sharing launches, boxes in them)."""
        g, n = C.c_int(), C.c_int()
        self._check(lib.streams_b200_batch_groups(self._h, C.byref(g), C.byref(n)))
        return int(g.value), int(n.value)

    def tune_form(self, forms=(1, 0, 2), replays: int = 2) -> tuple[int, int, dict]:
        """Pick the launch form (``set_shared_launches`` groups per class; 0: a graph branch per
        box) by timing ``replays`` graph replays of each on the live boxes, after one replay of
        warm-up (the capture); the batch is left in the fastest form.  The steps taken are steps
        of the solves (every form gives the same results), so the caller counts them.  Returns
        (form, steps advanced, seconds per replay of each form)."""
        import time
        spg = self.steps_per_graph
        self.advance(1)  # leave the first-step / lead phase before timing replays
        done = 1
        times = {}
        for f in forms:
            self.set_shared_launches(f)
            self.advance(spg)
            self.synchronize()
            t0 = time.perf_counter()
            self.advance(replays * spg)
            self.synchronize()
            times[f] = (time.perf_counter() - t0) / replays
            done += (1 + replays) * spg
        best = min(times, key=times.get)
        self.set_shared_launches(best)
        return best, done, times

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            lib.streams_b200_batch_destroy(h)
            self._h = None

    __del__ = close
