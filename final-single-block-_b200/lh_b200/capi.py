"""ctypes binding of the C ABI in include/lh_gpu.h (liblh_gpu.so).

The shared library is built in-tree (``final-single-block-_b200/build``) by
``__graft_entry__.build()`` or ``make -C final-single-block-_b200/csrc``.
Nothing here falls back to another implementation: if the library or a
CUDA device is missing the calls fail with :class:`LHError`.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.environ.get("LH_LIBPATH") or os.path.join(os.path.dirname(PKG), "build", "liblh_gpu.so")

LH_OK, LH_EINVAL, LH_ECUDA, LH_ENOMEM, LH_EDEVICE, LH_ESTATE = 0, -1, -2, -3, -4, -5
GRID_POLY, GRID_TANH = 0, 1
DT_CFL, DT_FIXED = 0, 1

# every symbol include/lh_gpu.h declares
EXPORTS = [
    "lh_ctx_create", "lh_ctx_destroy", "lh_last_error", "lh_get_sizes", "lh_get_grid", "lh_host_grid",
    "lh_upload_state", "lh_download_state", "lh_download_nu", "lh_substep", "lh_step",
    "lh_get_scalars", "lh_step_host", "lh_synchronize", "lh_get_stream", "lh_profile",
    "lh_error_div", "lh_get_intermediate", "lh_four_to_phys", "lh_phys_to_four", "lh_lusolu",
    "lh_lusolp", "lh_lusolu_noalloc", "lh_batch_create", "lh_batch_destroy", "lh_batch_last_error",
    "lh_instance_bytes", "lh_batch_add", "lh_batch_remove", "lh_batch_step",
    "lh_batch_download", "lh_batch_scalars", "lh_batch_set_scalars", "lh_batch_count", "lh_batch_synchronize",
    "lh_spectra_accumulate", "lh_spectra_reset", "lh_get_spectra",
    "lh_stats_accumulate", "lh_stats_reset", "lh_get_stats", "lh_pressure_snapshot", "lh_omega_x",
    "lh_tridiag_factor", "lh_tridiag_solve", "lh_set_dg", "lh_set_scalars", "lh_autotune",
]


class LHError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class GridDesc(ctypes.Structure):
    _fields_ = [
        ("Nx", ctypes.c_int), ("Nz", ctypes.c_int), ("ny", ctypes.c_int),
        ("Re", ctypes.c_double), ("alp", ctypes.c_double), ("bet", ctypes.c_double),
        ("mpgx", ctypes.c_double), ("flag_ctpress", ctypes.c_int), ("grid_type", ctypes.c_int),
        ("dyq", ctypes.c_double), ("ppp", ctypes.c_int), ("gamma", ctypes.c_double),
        ("dt_mode", ctypes.c_int), ("CFL", ctypes.c_double), ("dt", ctypes.c_double),
    ]


class Sizes(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("Nx", "Nz", "Mx", "Mz", "nyu", "nyv", "ncols", "igal", "kgal")]


@dataclass
class Desc:
    """Instance description (the input.in values, start.f90:85-252)."""
    Nx: int = 32
    Nz: int = 32
    ny: int = 153
    Re: float = 3250.0
    alp: float = 1.0
    bet: float = 2.0
    mpgx: float = -3.0675e-3
    flag_ctpress: int = 1
    grid_type: int = GRID_POLY
    dyq: float = 10.0
    ppp: int = 5
    gamma: float = 2.0
    dt_mode: int = DT_CFL
    CFL: float = 0.7
    dt: float = 1e-3

    def c(self) -> GridDesc:
        return GridDesc(self.Nx, self.Nz, self.ny, self.Re, self.alp, self.bet, self.mpgx,
                        self.flag_ctpress, self.grid_type, self.dyq, self.ppp, self.gamma,
                        self.dt_mode, self.CFL, self.dt)

    @property
    def nyu(self) -> int:
        return self.ny - 1

    @property
    def nyv(self) -> int:
        return self.ny - 2

    @property
    def ncols(self) -> int:
        return (self.Nx // 2 + 1) * self.Nz

    def points(self) -> int:
        """Grid points Nx*Nz*ny (the unit of the throughput metric)."""
        return self.Nx * self.Nz * self.ny


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise LHError(LH_EINVAL, f"{LIBPATH} not built; run __graft_entry__.build()")
    L = ctypes.CDLL(LIBPATH)
    P = ctypes.POINTER
    i, d, v, sz = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_size_t
    dp = P(ctypes.c_double)
    sig = {
        "lh_ctx_create": (i, [P(GridDesc), P(v)]),
        "lh_ctx_destroy": (i, [v]),
        "lh_last_error": (ctypes.c_char_p, [v]),
        "lh_get_sizes": (i, [v, P(Sizes)]),
        "lh_get_grid": (i, [v, i, dp, i]),
        "lh_host_grid": (i, [P(GridDesc), i, dp, i]),
        "lh_upload_state": (i, [v, dp, dp, dp, dp]),
        "lh_download_state": (i, [v, dp, dp, dp, dp]),
        "lh_download_nu": (i, [v, dp, dp, dp]),
        "lh_substep": (i, [v, i]),
        "lh_step": (i, [v, i]),
        "lh_get_scalars": (i, [v, dp, dp, P(i), dp, dp]),
        "lh_step_host": (i, [v, dp, dp, dp, dp, i]),
        "lh_synchronize": (i, [v]),
        "lh_get_stream": (i, [v, P(v)]),
        "lh_profile": (i, [v, i, dp, P(i)]),
        "lh_error_div": (i, [v, dp]),
        "lh_get_intermediate": (i, [v, i, dp, sz]),
        "lh_four_to_phys": (i, [v, dp, i]),
        "lh_phys_to_four": (i, [v, dp, i]),
        "lh_lusolu": (i, [v, i, i, d, dp, dp]),
        "lh_lusolp": (i, [v, dp]),
        "lh_lusolu_noalloc": (i, [v, i, i, d, v, v]),
        "lh_batch_create": (i, [sz, P(v)]),
        "lh_batch_destroy": (i, [v]),
        "lh_batch_last_error": (ctypes.c_char_p, [v]),
        "lh_instance_bytes": (sz, [P(GridDesc)]),
        "lh_batch_add": (i, [v, P(GridDesc), dp, dp, dp, dp, P(i)]),
        "lh_batch_remove": (i, [v, i]),
        "lh_batch_step": (i, [v, i]),
        "lh_batch_download": (i, [v, i, dp, dp, dp, dp]),
        "lh_batch_scalars": (i, [v, i, dp, dp, P(i)]),
        "lh_batch_set_scalars": (i, [v, i, d, i, d]),
        "lh_batch_count": (i, [v]),
        "lh_batch_synchronize": (i, [v]),
        "lh_spectra_accumulate": (i, [v]),
        "lh_spectra_reset": (i, [v]),
        "lh_get_spectra": (i, [v, i, dp, sz, P(i)]),
        "lh_stats_accumulate": (i, [v]),
        "lh_stats_reset": (i, [v]),
        "lh_get_stats": (i, [v, dp, sz, P(i)]),
        "lh_pressure_snapshot": (i, [v]),
        "lh_omega_x": (i, [v, dp, sz]),
        "lh_tridiag_factor": (i, [v, i, i, d, dp, sz]),
        "lh_tridiag_solve": (i, [v, i, dp, dp]),
        "lh_set_dg": (i, [v, dp]),
        "lh_set_scalars": (i, [v, d, i, d]),
        "lh_autotune": (i, [v, i, P(i)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _dp(a):
    if a is None:
        return None
    if isinstance(a, int):  # raw address (pinned / device-owned host buffer)
        return ctypes.cast(a, ctypes.POINTER(ctypes.c_double))
    assert a.dtype in (np.float64, np.complex128) and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def col_layout(a: np.ndarray) -> np.ndarray:
    """[column, j] complex array -> contiguous buffer in the reference layout."""
    return np.ascontiguousarray(np.asarray(a, np.complex128))


class Engine:
    """One channel instance behind the C ABI (the drop-in for the reference step)."""

    def __init__(self, desc: Desc):
        self.L = lib()
        self.desc = desc
        h = ctypes.c_void_p()
        rc = self.L.lh_ctx_create(ctypes.byref(desc.c()), ctypes.byref(h))
        if rc != LH_OK:
            raise LHError(rc, f"lh_ctx_create failed for {desc}")
        self.h = h
        s = Sizes()
        self.L.lh_get_sizes(self.h, ctypes.byref(s))
        self.sizes = s

    def close(self):
        if getattr(self, "h", None):
            self.L.lh_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc: int, what: str):
        if rc != LH_OK:
            raise LHError(rc, f"{what}: {self.L.lh_last_error(self.h).decode()}")

    # ---- state ----------------------------------------------------------
    def upload(self, u1, u2, u3, p=None):
        bufs = [col_layout(x) for x in (u1, u2, u3)]
        pb = col_layout(p) if p is not None else None
        self._keep = (bufs, pb)
        self._ck(self.L.lh_upload_state(self.h, *[_dp(b) for b in bufs], _dp(pb)), "upload")

    def download(self):
        s, d = self.sizes, self.desc
        u1 = np.zeros((s.ncols, s.nyu + 2), np.complex128)
        u2 = np.zeros((s.ncols, s.nyv + 2), np.complex128)
        u3 = np.zeros((s.ncols, s.nyu + 2), np.complex128)
        p = np.zeros((s.ncols, s.nyu), np.complex128)
        self._ck(self.L.lh_download_state(self.h, _dp(u1), _dp(u2), _dp(u3), _dp(p)), "download")
        return {"u1": u1, "u2": u2, "u3": u3, "p": p}

    def download_nu(self):
        s = self.sizes
        n1 = np.zeros((s.ncols, s.nyu), np.complex128)
        n2 = np.zeros((s.ncols, s.nyv), np.complex128)
        n3 = np.zeros((s.ncols, s.nyu), np.complex128)
        self._ck(self.L.lh_download_nu(self.h, _dp(n1), _dp(n2), _dp(n3)), "download_nu")
        return n1, n2, n3

    def intermediate(self, which: int) -> np.ndarray:
        n = self.L.lh_get_intermediate(self.h, which, None, 0)
        if n < 0:
            self._ck(n, "intermediate")
        out = np.zeros(n // 2, np.complex128)
        rc = self.L.lh_get_intermediate(self.h, which, _dp(out), n)
        if rc < 0:
            self._ck(rc, "intermediate")
        return out.reshape(self.sizes.ncols, -1)

    # ---- stepping --------------------------------------------------------
    def substep(self, kRK: int):
        self._ck(self.L.lh_substep(self.h, kRK), "substep")

    def step(self, n: int = 1):
        self._ck(self.L.lh_step(self.h, n), "step")

    def synchronize(self):
        self._ck(self.L.lh_synchronize(self.h), "synchronize")

    def scalars(self) -> dict:
        t, dt, mp, qx = (ctypes.c_double() for _ in range(4))
        it = ctypes.c_int()
        self._ck(self.L.lh_get_scalars(self.h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(it),
                                       ctypes.byref(mp), ctypes.byref(qx)), "scalars")
        return {"t": t.value, "dt": dt.value, "iter": it.value, "mpgx": mp.value, "Qx": qx.value}

    def error_div(self) -> float:
        e = ctypes.c_double()
        self._ck(self.L.lh_error_div(self.h, ctypes.byref(e)), "error_div")
        return e.value

    # ---- spectra of flagged steps (spectra.f90) --------------------------
    SPECTRA = ("spU", "spV", "spW", "spUV", "spP")

    def spectra_accumulate(self):
        """Add the current state's spectra terms (the reference's flagged-step call)."""
        self._ck(self.L.lh_spectra_accumulate(self.h), "spectra_accumulate")

    def spectra_reset(self):
        self._ck(self.L.lh_spectra_reset(self.h), "spectra_reset")

    def spectra(self) -> tuple[dict, int]:
        """The accumulated spectra as {name: array[column, j]} and the count."""
        out, cnt = {}, ctypes.c_int()
        for w, name in enumerate(self.SPECTRA):
            n = self.L.lh_get_spectra(self.h, w, None, 0, None)
            if n < 0:
                self._ck(n, "spectra")
            a = np.zeros(n)
            self._ck(min(0, self.L.lh_get_spectra(self.h, w, _dp(a), n, ctypes.byref(cnt))), "spectra")
            out[name] = a.reshape(self.sizes.ncols, n // self.sizes.ncols)
        return out, cnt.value

    # ---- stats of flagged steps (stats.f90) ------------------------------
    STATS = ("Um", "U2m", "Vm", "V2m", "Wm", "W2m", "UVm", "UWm", "VWm", "Pm", "P2m", "wxm", "wx2m")

    def stats_accumulate(self):
        self._ck(self.L.lh_stats_accumulate(self.h), "stats_accumulate")

    def stats_reset(self):
        self._ck(self.L.lh_stats_reset(self.h), "stats_reset")

    def pressure_snapshot(self):
        """ppPL <- p, as nonlinear() does at output steps (FOU3D.f90:149-152)."""
        self._ck(self.L.lh_pressure_snapshot(self.h), "pressure_snapshot")

    def stats(self) -> tuple[np.ndarray, int]:
        """The plane sums as array[13, nyu+2] (rows named by STATS) and the
        accumulation count."""
        n = self.L.lh_get_stats(self.h, None, 0, None)
        if n < 0:
            self._ck(n, "stats")
        a, cnt = np.zeros(n), ctypes.c_int()
        self._ck(min(0, self.L.lh_get_stats(self.h, _dp(a), n, ctypes.byref(cnt))), "stats")
        q = len(self.STATS)
        return a.reshape(q, n // q), cnt.value

    def omega_x(self) -> np.ndarray:
        """omega_x of the current state (FOU3D.f90:314-338): [nyu+2, Nz, Nx+2],
        physical values in [:, :, :Nx]."""
        n = self.L.lh_omega_x(self.h, None, 0)
        if n < 0:
            self._ck(n, "omega_x")
        a = np.zeros(n)
        self._ck(min(0, self.L.lh_omega_x(self.h, _dp(a), n)), "omega_x")
        sz = self.sizes
        return a.reshape(sz.nyu + 2, sz.Nz, sz.Nx + 2)

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._ck(self.L.lh_get_stream(self.h, ctypes.byref(s)), "stream")
        return s.value or 0

    def profile(self, nsteps: int = 1):
        ms = (ctypes.c_double * 5)()
        n = (ctypes.c_int * 5)()
        self._ck(self.L.lh_profile(self.h, nsteps, ms, n), "profile")
        names = ["z_inverse", "x_products", "z_forward", "dt", "column"]
        return {k: (ms[i], n[i]) for i, k in enumerate(names)}

    def step_host(self, bufs, nsteps: int = 1):
        """Upload host buffers, run nsteps, download into the same buffers."""
        u1, u2, u3, p = bufs
        self._ck(self.L.lh_step_host(self.h, _dp(u1), _dp(u2), _dp(u3), _dp(p), nsteps), "step_host")

    # ---- unit entries ------------------------------------------------------
    def four_to_phys(self, planes: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(planes, np.float64).copy()
        n = a.size // (self.sizes.igal * self.sizes.kgal)
        self._ck(self.L.lh_four_to_phys(self.h, _dp(a), n), "four_to_phys")
        return a

    def phys_to_four(self, planes: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(planes, np.float64).copy()
        n = a.size // (self.sizes.igal * self.sizes.kgal)
        self._ck(self.L.lh_phys_to_four(self.h, _dp(a), n), "phys_to_four")
        return a

    def lusolu(self, grid: int, kRK: int, dt: float, rhs: np.ndarray) -> np.ndarray:
        r = col_layout(rhs)
        u = np.zeros_like(r)
        self._ck(self.L.lh_lusolu(self.h, grid, kRK, dt, _dp(r), _dp(u)), "lusolu")
        return u

    def lusolp(self, x: np.ndarray) -> np.ndarray:
        a = col_layout(x).copy()
        self._ck(self.L.lh_lusolp(self.h, _dp(a)), "lusolp")
        return a

    def tridiag_factor(self, grid: int, kRK: int = 1, dt: float = 0.0) -> np.ndarray:
        """Factors a(3, j, column) as an array [column, j, 3] (LU_build +
        LU_dec, or DG for grid 3)."""
        n = self.L.lh_tridiag_factor(self.h, grid, kRK, dt, None, 0)
        if n < 0:
            self._ck(n, "tridiag_factor")
        a = np.zeros(n)
        rc = self.L.lh_tridiag_factor(self.h, grid, kRK, dt, _dp(a), n)
        if rc < 0:
            self._ck(rc, "tridiag_factor")
        return a.reshape(self.sizes.ncols, -1, 3)

    def tridiag_solve(self, grid: int, a: np.ndarray, x: np.ndarray) -> np.ndarray:
        fa = np.ascontiguousarray(a, np.float64)
        xb = col_layout(x).copy()
        self._ck(self.L.lh_tridiag_solve(self.h, grid, _dp(fa), _dp(xb)), "tridiag_solve")
        return xb

    def set_dg(self, a: np.ndarray):
        self._ck(self.L.lh_set_dg(self.h, _dp(np.ascontiguousarray(a, np.float64))), "set_dg")

    def set_scalars(self, t: float, it: int, mpgx: float):
        """Continue a run: t, iter and mpgx of a restart file (getini, flag_init = 2)."""
        self._ck(self.L.lh_set_scalars(self.h, float(t), int(it), float(mpgx)), "set_scalars")

    def autotune(self, force: bool = False) -> dict:
        """Tune this size's launch shapes (or read them from the cache)."""
        out = (ctypes.c_int * 6)()
        self._ck(self.L.lh_autotune(self.h, 1 if force else 0, out), "autotune")
        keys = ("cbz", "rbx", "cbf", "staging_mb", "col_waves")
        r = {k: out[i] for i, k in enumerate(keys)}
        r["source"] = {1: "measured", 2: "cache"}.get(out[5], "?")
        return r

    def grid(self, which: int) -> np.ndarray:
        n = self.L.lh_get_grid(self.h, which, None, 0)
        out = np.zeros(n)
        self.L.lh_get_grid(self.h, which, _dp(out), n)
        return out


class Batch:
    """Many independent instances advanced in shared launches."""

    def __init__(self, hbm_budget: int = 0):
        self.L = lib()
        h = ctypes.c_void_p()
        rc = self.L.lh_batch_create(hbm_budget, ctypes.byref(h))
        if rc != LH_OK:
            raise LHError(rc, "lh_batch_create failed")
        self.h = h
        self.desc: dict[int, Desc] = {}

    def close(self):
        if getattr(self, "h", None):
            self.L.lh_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc: int, what: str):
        if rc != LH_OK:
            raise LHError(rc, f"{what}: {self.L.lh_batch_last_error(self.h).decode()}")

    @staticmethod
    def instance_bytes(desc: Desc) -> int:
        return lib().lh_instance_bytes(ctypes.byref(desc.c()))

    def add(self, desc: Desc, u1, u2, u3, p=None) -> int:
        bufs = [col_layout(x) for x in (u1, u2, u3)]
        pb = col_layout(p) if p is not None else None
        slot = ctypes.c_int()
        self._ck(self.L.lh_batch_add(self.h, ctypes.byref(desc.c()), *[_dp(b) for b in bufs], _dp(pb),
                                     ctypes.byref(slot)), "add")
        self.desc[slot.value] = desc
        return slot.value

    def remove(self, slot: int):
        self._ck(self.L.lh_batch_remove(self.h, slot), "remove")
        self.desc.pop(slot, None)

    def step(self, n: int = 1):
        self._ck(self.L.lh_batch_step(self.h, n), "step")

    def synchronize(self):
        self._ck(self.L.lh_batch_synchronize(self.h), "synchronize")

    def count(self) -> int:
        return self.L.lh_batch_count(self.h)

    def set_scalars(self, slot: int, t: float, it: int, mpgx: float):
        """Restore t, iter and mpgx of an instance (a snapshot or restart file)."""
        self._ck(self.L.lh_batch_set_scalars(self.h, slot, float(t), int(it), float(mpgx)), "set_scalars")

    def download(self, slot: int):
        d = self.desc[slot]
        u1 = np.zeros((d.ncols, d.nyu + 2), np.complex128)
        u2 = np.zeros((d.ncols, d.nyv + 2), np.complex128)
        u3 = np.zeros((d.ncols, d.nyu + 2), np.complex128)
        p = np.zeros((d.ncols, d.nyu), np.complex128)
        self._ck(self.L.lh_batch_download(self.h, slot, _dp(u1), _dp(u2), _dp(u3), _dp(p)), "download")
        return {"u1": u1, "u2": u2, "u3": u3, "p": p}

    def scalars(self, slot: int) -> dict:
        t, dt = ctypes.c_double(), ctypes.c_double()
        it = ctypes.c_int()
        self._ck(self.L.lh_batch_scalars(self.h, slot, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(it)),
                 "scalars")
        return {"t": t.value, "dt": dt.value, "iter": it.value}


_grid_cache: dict = {}


def host_grid(desc: Desc, which: int) -> np.ndarray:
    """Set-up arrays of a description computed on the host (no GPU needed);
    memoised on the fields the y grid depends on (sizes, box and grid
    stretching), a copy is returned."""
    key = (desc.Nx, desc.Nz, desc.ny, desc.alp, desc.bet, desc.grid_type, desc.dyq, desc.ppp, desc.gamma,
           desc.Re if which == 4 else None, which)
    hit = _grid_cache.get(key)
    if hit is None:
        L = lib()
        n = L.lh_host_grid(ctypes.byref(desc.c()), which, None, 0)
        if n < 0:
            raise LHError(n, f"set-up rejected for {desc}")
        hit = np.zeros(n)
        L.lh_host_grid(ctypes.byref(desc.c()), which, _dp(hit), n)
        if len(_grid_cache) > 256:
            _grid_cache.clear()
        _grid_cache[key] = hit
    return hit.copy()
