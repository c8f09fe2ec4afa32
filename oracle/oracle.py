"""TEST INFRASTRUCTURE -- ctypes front end of the parity oracle.

The oracle is a plain-C restatement of the reference's time-step path
(``lh_oracle.c``, ``lh_fftpack.c``).  This module loads it, builds it on
demand with ``make`` and exposes the reference-shaped arrays as numpy views.
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import it.

It also restates the reference's spectral file reader at one MPI rank
(``read_in``, start.f90:1545-1997, with ``buff_to_u`` FOU3D.f90:2297-2322):
planes 0..nyu of u1/u3, 0..nyv+1 of u2 and 1..nyu of p are read; the top
ghost plane nyu+1 of u1 and u3 is *not* read at np = 1 and stays zero.
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "build")

GRID_POLY, GRID_TANH = 0, 1
DT_CFL, DT_FIXED = 0, 1

F_U1, F_U2, F_U3, F_P, F_NU1, F_NU2, F_NU3, F_DIV, F_PSI = range(9)


class Params(ctypes.Structure):
    _fields_ = [
        ("Nx", ctypes.c_int), ("Nz", ctypes.c_int), ("ny", ctypes.c_int),
        ("Re", ctypes.c_double), ("alp", ctypes.c_double), ("bet", ctypes.c_double),
        ("mpgx", ctypes.c_double), ("flag_ctpress", ctypes.c_int),
        ("grid_type", ctypes.c_int), ("dyq", ctypes.c_double), ("ppp", ctypes.c_int),
        ("gamma", ctypes.c_double), ("dt_mode", ctypes.c_int), ("CFL", ctypes.c_double),
        ("dt_fixed", ctypes.c_double), ("nthreads", ctypes.c_int),
    ]


_libs: dict[bool, ctypes.CDLL] = {}


def build() -> None:
    """Compile the oracle shared libraries (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(threaded: bool = False) -> ctypes.CDLL:
    if threaded in _libs:
        return _libs[threaded]
    name = "liblh_oracle_omp.so" if threaded else "liblh_oracle.so"
    path = os.path.join(BUILD, name)
    if not os.path.exists(path):
        build()
    L = ctypes.CDLL(path)
    P = ctypes.POINTER
    d, i, v = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
    dp = P(ctypes.c_double)
    L.lho_create.restype = v
    L.lho_create.argtypes = [P(Params)]
    L.lho_destroy.argtypes = [v]
    L.lho_sizes.argtypes = [v, P(ctypes.c_int)]
    L.lho_get_array.restype = i
    L.lho_get_array.argtypes = [v, i, dp, i]
    L.lho_field_len.restype = i
    L.lho_field_len.argtypes = [v, i]
    L.lho_set_field.argtypes = [v, i, dp]
    L.lho_get_field.argtypes = [v, i, dp]
    L.lho_get_scalar.restype = d
    L.lho_get_scalar.argtypes = [v, i]
    L.lho_set_scalar.argtypes = [v, i, d]
    L.lho_substep.argtypes = [v, i]
    L.lho_step.argtypes = [v, i]
    L.lho_get_intermediate.restype = i
    L.lho_get_intermediate.argtypes = [v, i, dp, i]
    L.lho_four_to_phys.argtypes = [v, dp]
    L.lho_phys_to_four.argtypes = [v, dp]
    L.lho_der_x.argtypes = [v, dp, dp]
    L.lho_der_z.argtypes = [v, dp, dp]
    L.lho_lusolu.argtypes = [v, i, i, dp, dp]
    L.lho_lusolp.argtypes = [v, dp]
    L.lho_lu_factor.argtypes = [v, i, i, dp]
    L.lho_error_div.restype = d
    L.lho_error_div.argtypes = [v]
    L.lho_spectra.argtypes = [v, dp, dp, dp, dp, dp]
    L.lho_stats.argtypes = [v, dp]
    L.lho_pressure_snapshot.argtypes = [v]
    L.lho_omega_x.argtypes = [v, dp]
    L.lho_der_z_n.argtypes = [dp, dp, dp, i, i]
    L.lho_cfft_init.restype = i
    L.lho_rfft_init.restype = i
    _libs[threaded] = L
    return L


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@dataclass
class Config:
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
    dt_fixed: float = 1e-3
    nthreads: int = 0


class Oracle:
    """One channel instance advanced by the C restatement."""

    def __init__(self, cfg: Config, threaded: bool = False):
        self.cfg = cfg
        self.L = lib(threaded)
        p = Params(cfg.Nx, cfg.Nz, cfg.ny, cfg.Re, cfg.alp, cfg.bet, cfg.mpgx, cfg.flag_ctpress,
                   cfg.grid_type, cfg.dyq, cfg.ppp, cfg.gamma, cfg.dt_mode, cfg.CFL, cfg.dt_fixed,
                   cfg.nthreads)
        self.h = self.L.lho_create(ctypes.byref(p))
        if not self.h:
            raise ValueError(f"oracle rejected configuration {cfg}")
        s = (ctypes.c_int * 10)()
        self.L.lho_sizes(self.h, s)
        (self.Nx, self.Nz, self.Mx, self.Mz, self.nyu, self.nyv, self.nyp, self.ncols,
         self.igal, self.kgal) = list(s)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.L.lho_destroy(h)
            self.h = None

    # -- arrays ---------------------------------------------------------
    def array(self, which: int) -> np.ndarray:
        n = self.L.lho_get_array(self.h, which, None, 0)
        out = np.zeros(n, np.float64)
        self.L.lho_get_array(self.h, which, _dp(out), n)
        return out

    def field_shape(self, f: int) -> tuple[int, int]:
        n = self.L.lho_field_len(self.h, f) // 2
        return (self.ncols, n // self.ncols)

    def get(self, f: int) -> np.ndarray:
        """Field as complex array [column, j] (reference x(j, column))."""
        n = self.L.lho_field_len(self.h, f)
        out = np.zeros(n, np.float64)
        self.L.lho_get_field(self.h, f, _dp(out))
        nc = self.ncols
        return out.view(np.complex128).reshape(nc, -1)

    def set(self, f: int, a: np.ndarray) -> None:
        n = self.L.lho_field_len(self.h, f)
        buf = np.ascontiguousarray(np.asarray(a, np.complex128)).view(np.float64).ravel()
        assert buf.size == n, (buf.size, n)
        self.L.lho_set_field(self.h, f, _dp(buf))

    def intermediate(self, which: int) -> np.ndarray:
        n = self.L.lho_get_intermediate(self.h, which, None, 0)
        out = np.zeros(n, np.float64)
        self.L.lho_get_intermediate(self.h, which, _dp(out), n)
        return out.view(np.complex128).reshape(self.ncols, -1)

    def scalar(self, which: int) -> float:
        return self.L.lho_get_scalar(self.h, which)

    def set_scalar(self, which: int, v: float) -> None:
        self.L.lho_set_scalar(self.h, which, float(v))

    # -- stepping ---------------------------------------------------------
    def substep(self, kRK: int) -> None:
        self.L.lho_substep(self.h, kRK)

    def step(self, n: int = 1) -> None:
        self.L.lho_step(self.h, n)

    def load_state(self, u1, u2, u3, p) -> None:
        for f, a in ((F_U1, u1), (F_U2, u2), (F_U3, u3), (F_P, p)):
            self.set(f, a)

    def state(self) -> dict[str, np.ndarray]:
        return {"u1": self.get(F_U1), "u2": self.get(F_U2), "u3": self.get(F_U3), "p": self.get(F_P)}

    def error_div(self) -> float:
        return self.L.lho_error_div(self.h)

    STATS = ("Um", "U2m", "Vm", "V2m", "Wm", "W2m", "UVm", "UWm", "VWm", "Pm", "P2m", "wxm", "wx2m")

    def stats(self, acc: np.ndarray | None = None) -> np.ndarray:
        """stats() at a flagged output step: add into acc[13, nyu+2] (new zeros when None)."""
        if acc is None:
            acc = np.zeros((len(self.STATS), self.nyu + 2))
        self.L.lho_stats(self.h, _dp(acc))
        return acc

    def pressure_snapshot(self) -> None:
        """ppPL <- p, as nonlinear() does at output steps (FOU3D.f90:149-152)."""
        self.L.lho_pressure_snapshot(self.h)

    def omega_x(self) -> np.ndarray:
        """omega_x of the current state (FOU3D.f90:314-338): [nyu+2, Nz, Nx+2],
        physical values in [:, :, :Nx]."""
        wx = np.zeros((self.nyu + 2, self.Nz, self.Nx + 2))
        self.L.lho_omega_x(self.h, _dp(wx))
        return wx

    def spectra(self, acc: dict | None = None) -> dict:
        """spectra() at a flagged step: add the current state's terms into acc
        (new zero accumulators when None); arrays [column, j]."""
        nc, nyu, nyv = self.ncols, self.nyu, self.nyv
        if acc is None:
            acc = {"spU": np.zeros((nc, nyu + 2)), "spV": np.zeros((nc, nyv + 2)), "spW": np.zeros((nc, nyu + 2)),
                   "spUV": np.zeros((nc, nyu + 2)), "spP": np.zeros((nc, nyu))}
        self.L.lho_spectra(self.h, *(_dp(acc[k]) for k in ("spU", "spV", "spW", "spUV", "spP")))
        return acc

    # -- plane helpers ----------------------------------------------------
    def four_to_phys(self, plane: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(plane, np.float64).copy()
        self.L.lho_four_to_phys(self.h, _dp(a))
        return a

    def phys_to_four(self, plane: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(plane, np.float64).copy()
        self.L.lho_phys_to_four(self.h, _dp(a))
        return a

    def der_x(self, plane: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(plane, np.float64)
        out = np.full_like(a, np.nan)
        self.L.lho_der_x(self.h, _dp(a), _dp(out))
        return out

    def der_z(self, plane: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(plane, np.float64)
        out = np.full_like(a, np.nan)
        self.L.lho_der_z(self.h, _dp(a), _dp(out))
        return out


# -- FFTPACK-level helpers --------------------------------------------------
class _CFFT(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("dn1", ctypes.c_double), ("ifac", ctypes.c_int * 32),
                ("wa", ctypes.c_double * 2048)]


class _RFFT(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("dn1", ctypes.c_double), ("ifac", ctypes.c_int * 32),
                ("wa", ctypes.c_double * 1024)]


def cft(c: np.ndarray, ise: int, isa: int, m: int, iopt: int, n: int) -> np.ndarray:
    """Restated ``cft`` (cft_buff.f:1-65) on a flat real array (copy returned)."""
    L = lib()
    t = _CFFT()
    if L.lho_cfft_init(ctypes.byref(t), n) != 0:
        raise ValueError(f"unsupported length {n}")
    a = np.ascontiguousarray(c, np.float64).copy()
    w = np.zeros(4 * n + 8)
    L.lho_cft(_dp(a), ise, isa, m, iopt, ctypes.byref(t), _dp(w))
    return a


def rft(c: np.ndarray, isa: int, m: int, iopt: int, n: int) -> np.ndarray:
    """Restated ``rft`` (rft_buff.f:24-86) on a flat real array (copy returned)."""
    L = lib()
    t = _RFFT()
    if L.lho_rfft_init(ctypes.byref(t), n) != 0:
        raise ValueError(f"unsupported length {n}")
    a = np.ascontiguousarray(c, np.float64).copy()
    w = np.zeros(n + 8)
    L.lho_rft(_dp(a), isa, m, iopt, ctypes.byref(t), _dp(w))
    return a


def fft_factors(n: int, real: bool) -> list[int]:
    L = lib()
    t = _RFFT() if real else _CFFT()
    rc = (L.lho_rfft_init if real else L.lho_cfft_init)(ctypes.byref(t), n)
    if rc != 0:
        raise ValueError(f"unsupported length {n}")
    nf = t.ifac[1]
    return [t.ifac[2 + k] for k in range(nf)]


# -- reference spectral files ----------------------------------------------
def _records(path: str):
    with open(path, "rb") as f:
        data = f.read()
    off = 0
    while off < len(data):
        (n,) = struct.unpack_from("<i", data, off)
        rec = data[off + 4: off + 4 + n]
        (n2,) = struct.unpack_from("<i", data, off + 4 + n)
        if n2 != n:
            raise ValueError(f"{path}: broken record marker at {off}")
        off += 8 + n
        yield rec


@dataclass
class DatFile:
    t: float
    Re: float
    alp: float
    bet: float
    mpgx: float
    nband: int
    iter: int
    N: np.ndarray          # (4, 5)
    y: np.ndarray
    ddthetavi: float
    dthdy: np.ndarray
    planes: dict           # j -> (Nx+2, Nz) real, Fortran order


def read_dat(path: str) -> DatFile:
    """Parse one reference spectral file (record_out FOU3D.f90:2066-2078)."""
    recs = _records(path)
    r1 = next(recs)
    t, Re, alp, bet, mpgx = struct.unpack_from("<5d", r1, 0)
    nband, it = struct.unpack_from("<2i", r1, 40)
    N = np.frombuffer(next(recs), "<i4").reshape(5, 4).T.copy()
    r3 = np.frombuffer(next(recs), "<f8")
    ny = (r3.size - 1) // 2
    y, ddv, dthdy = r3[:ny], r3[ny], r3[ny + 1:]
    planes = {}
    for rec in recs:
        j, _id, nx, nz = struct.unpack_from("<4i", rec, 0)
        buf = np.frombuffer(rec, "<f8", offset=24).reshape(nz, nx).T.copy()
        planes[j] = buf
    return DatFile(t, Re, alp, bet, mpgx, nband, it, N, y, ddv, dthdy, planes)


def plane_to_columns(buf: np.ndarray, Nx: int, Nz: int) -> np.ndarray:
    """buff(Nx+2, Nz) spectral plane -> complex per column (k-major, i fast)."""
    re = buf[0::2, :]  # (Nx/2+1, Nz)
    im = buf[1::2, :]
    z = (re + 1j * im)  # [i, k]
    return z.T.reshape(-1)  # column index (k-1)*(Nx/2+1) + i


def read_in_np1(dirin: str, tag: str, Nx: int, Nz: int, nyu: int, nyv: int):
    """read_in at np = 1 (start.f90:1545-1997) -> u1, u2, u3, p [column, j]."""
    nc = (Nx // 2 + 1) * Nz
    u1 = np.zeros((nc, nyu + 2), np.complex128)
    u3 = np.zeros((nc, nyu + 2), np.complex128)
    u2 = np.zeros((nc, nyv + 2), np.complex128)
    p = np.zeros((nc, nyu), np.complex128)
    f1 = read_dat(os.path.join(dirin, "u1" + tag))
    f2 = read_dat(os.path.join(dirin, "u2" + tag))
    f3 = read_dat(os.path.join(dirin, "u3" + tag))
    fp = read_dat(os.path.join(dirin, "p" + tag))
    for j in range(0, nyu + 1):  # ju1 = jgal-1 = 0 .. ju2 = jgal(2,2) = nyu
        u1[:, j] = plane_to_columns(f1.planes[j], Nx, Nz)
        u3[:, j] = plane_to_columns(f3.planes[j], Nx, Nz)
    for j in range(0, nyv + 2):
        u2[:, j] = plane_to_columns(f2.planes[j], Nx, Nz)
    for j in range(1, nyu + 1):
        p[:, j - 1] = plane_to_columns(fp.planes[j], Nx, Nz)
    return u1, u2, u3, p, f1


def der_z_n(u: np.ndarray, kz_im, Nx: int, Nz: int, threaded: bool = False) -> np.ndarray:
    """der_z_N (FOU3D.f90:525-546) on an (Nx+2) x Nz real plane [k][i]: kz(k) u
    on every complex entry; kz_im are the imaginary parts of kz(1:Nz)."""
    L = lib(threaded)
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(Nz, Nx + 2)
    out = np.zeros_like(u)
    kz = np.ascontiguousarray(kz_im, dtype=np.float64)
    L.lho_der_z_n(_dp(u), _dp(out), _dp(kz), Nx, Nz)
    return out

