"""Initial conditions and the reference's spectral file format.

* :func:`perturbed_laminar` -- the synthetic initial state of the benchmark
  workloads: laminar u1(0,0)(y) = Re*mpgx*(y^2-1)/2 (the formula of the
  reference's commented parabolic start, start.f90:1501) plus seeded complex
  Gaussian perturbations 0.05*exp(-(kx^2+kz^2)/16)*(1-y^2)^2 on u1, u2, u3:
  one complex Gaussian coefficient per (field, kx, kz) times the smooth y
  envelope, drawn from a counter-based generator keyed by (seed, field, i,
  kz) so every run and every host gets the same bits.  (Independent draws
  per y row would put grid-scale noise in the divergence, and the first
  pressure projection of such a field is ill-conditioned: last-bit changes
  of the input move p by ~2e-12 relative.)  The kx = 0 column is made
  Hermitian so the field is real in physical space; the first pressure
  solve of the time step projects it divergence-free.
* :func:`read_state` / :func:`write_state` -- Fortran sequential unformatted
  files in the layout record_out writes (FOU3D.f90:2066-2165) and read_in
  reads (start.f90:1545-1997).  ``read_state(..., np1=True)`` reproduces
  read_in at one MPI rank, which does not read the top ghost plane nyu+1
  of u1 and u3 (it stays zero).
"""
from __future__ import annotations

import os
import struct

import numpy as np

from .capi import Desc

# SplitMix64 constants (a published 64-bit mixing function)
_G = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _mix(z: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = z + _G
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def _uniform(key: np.ndarray) -> np.ndarray:
    """(0, 1) doubles from 64-bit keys (53 high bits, never 0)."""
    return ((_mix(key) >> np.uint64(11)).astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)


def _gauss(seed: int, field: int, i, kz, j, stream: int) -> np.ndarray:
    with np.errstate(over="ignore"):
        base = np.uint64(seed) * np.uint64(0x100000001B3) + np.uint64(field * 4 + stream)
        key = (base * np.uint64(0xD6E8FEB86659FD93) + i.astype(np.uint64) * np.uint64(0x9E3779B1)
               + (kz.astype(np.int64) + 100000).astype(np.uint64) * np.uint64(0x85EBCA77)
               + j.astype(np.uint64) * np.uint64(0xC2B2AE3D))
    u1 = _uniform(key)
    u2 = _uniform(key ^ np.uint64(0x5851F42D4C957F2D))
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def re_from_retau(re_tau: float, mpgx: float = -3.0675e-3) -> float:
    """Bulk Re for a friction Reynolds number at fixed mean pressure gradient."""
    return re_tau / np.sqrt(-mpgx)


def grids(desc: Desc):
    """yu (0..nyu+1) and yv (0..nyv+1) from the engine's host set-up."""
    from .capi import host_grid
    return host_grid(desc, 0), host_grid(desc, 1)


def columns(desc: Desc):
    """(i, kz_signed) of every column in the reference order (start.f90:964-981)."""
    nxh = desc.Nx // 2 + 1
    kr = np.arange(desc.Nz)
    kzs = np.where(kr < desc.Nz // 2, kr, kr - desc.Nz)
    i = np.tile(np.arange(nxh), desc.Nz)
    kz = np.repeat(kzs, nxh)
    return i, kz


def perturbed_laminar(desc: Desc, seed: int, yu: np.ndarray, yv: np.ndarray, amp: float = 0.05,
                      np1_read_in: bool = True, white_in_y: bool = False):
    """Synthetic initial state in the reference column layout [column, j]."""
    i, kz = columns(desc)
    nc = i.size
    kx = desc.alp * i
    kzv = desc.bet * kz
    env = amp * np.exp(-(kx ** 2 + kzv ** 2) / 16.0)
    out = []
    for f, y in ((0, yu), (1, yv), (2, yu)):
        if white_in_y:
            J = np.arange(y.size)
            I2, J2 = np.meshgrid(i, J, indexing="ij")
            K2, _ = np.meshgrid(kz, J, indexing="ij")
            g = _gauss(seed, f, I2, K2, J2, 0) + 1j * _gauss(seed, f, I2, K2, J2, 1)
        else:  # one coefficient per column (counter j = 0), shared by every row
            j0 = np.zeros(nc, np.int64)
            g = (_gauss(seed, f, i, kz, j0, 0) + 1j * _gauss(seed, f, i, kz, j0, 1))[:, None]
        prof = (1.0 - np.clip(y, -1.0, 1.0) ** 2) ** 2
        a = env[:, None] * prof[None, :] * g
        a[0, :] = 0.0  # mode (0,0) carries the mean profile only
        # Hermitian kx = 0 column: u(0,-kz) = conj(u(0,kz)); kz = -Nz/2 real
        nxh = desc.Nx // 2 + 1
        for r in range(1, desc.Nz // 2):
            a[(desc.Nz - r) * nxh] = np.conj(a[r * nxh])
        a[(desc.Nz // 2) * nxh] = a[(desc.Nz // 2) * nxh].real
        out.append(a)
    u1, u2, u3 = out
    u1[0, :] += 0.5 * desc.Re * desc.mpgx * (yu ** 2 - 1.0)
    # ghost and wall rows by the reference boundary conditions (v_corr,
    # littleharsh.f90:935-984; weights start.f90:524-525)
    gwbc = (yu[0] - yv[0]) / (yu[1] - yv[0])
    for u in (u1, u3):
        u[:, 0] = gwbc * u[:, 1]
        u[:, -1] = gwbc * u[:, -2]
    u2[:, 0] = 0.0
    u2[:, -1] = 0.0
    if np1_read_in:
        u1[:, -1] = 0.0
        u3[:, -1] = 0.0
    p = np.zeros((nc, desc.nyu), np.complex128)
    return u1, u2, u3, p


# ---- reference file format ---------------------------------------------------
def _records(path: str):
    with open(path, "rb") as f:
        data = f.read()
    off = 0
    while off < len(data):
        (n,) = struct.unpack_from("<i", data, off)
        rec = data[off + 4: off + 4 + n]
        (n2,) = struct.unpack_from("<i", data, off + 4 + n)
        if n2 != n:
            raise ValueError(f"{path}: corrupt record at byte {off}")
        off += 8 + n
        yield rec


def _rec(b: bytes) -> bytes:
    return struct.pack("<i", len(b)) + b + struct.pack("<i", len(b))


def _plane_to_cols(buf: np.ndarray) -> np.ndarray:
    z = buf[0::2, :] + 1j * buf[1::2, :]
    return z.T.reshape(-1)


def _cols_to_plane(v: np.ndarray, Nx: int, Nz: int) -> np.ndarray:
    z = v.reshape(Nz, Nx // 2 + 1).T
    buf = np.zeros((Nx + 2, Nz))
    buf[0::2, :] = z.real
    buf[1::2, :] = z.imag
    return buf


def read_state(dirin: str, tag: str, desc: Desc, np1: bool = True):
    """u1, u2, u3, p (column layout) and the header of the u1 file."""
    nyu, nyv, nc = desc.nyu, desc.nyv, desc.ncols
    arrs = {}
    header = None
    for name, lo, hi in (("u1", 0, nyu + 1), ("u2", 0, nyv + 1), ("u3", 0, nyu + 1), ("p", 1, nyu)):
        path = os.path.join(dirin, name + tag)
        recs = _records(path)
        r1 = next(recs)
        t, Re, alp, bet, mpgx = struct.unpack_from("<5d", r1, 0)
        nband, it = struct.unpack_from("<2i", r1, 40)
        if name == "u1":
            header = {"t": t, "Re": Re, "alp": alp, "bet": bet, "mpgx": mpgx, "nband": nband, "iter": it}
        N = np.frombuffer(next(recs), "<i4").reshape(5, 4).T
        if N[0, 3] != desc.Nx or N[1, 3] != desc.Nz:
            raise ValueError(f"{path}: file has Nx={N[0, 3]} Nz={N[1, 3]}, expected {desc.Nx}x{desc.Nz}")
        next(recs)
        a = np.zeros((nc, hi - lo + 1), np.complex128)
        top = hi
        if np1 and name in ("u1", "u3"):
            top = nyu  # read_in at np=1 stops at jgal(2,2) = nyu
        for rec in recs:
            j, _id, nx, nz = struct.unpack_from("<4i", rec, 0)
            if lo <= j <= top:
                buf = np.frombuffer(rec, "<f8", offset=24).reshape(nz, nx).T
                a[:, j - lo] = _plane_to_cols(buf)
        arrs[name] = a
    return arrs["u1"], arrs["u2"], arrs["u3"], arrs["p"], header


def write_state(dirout: str, tag: str, desc: Desc, u1, u2, u3, p, yu, yv, dthdyu, dthdyv,
                t: float = 0.0, it: int = 0, mpgx: float | None = None) -> None:
    """Write the four spectral files the way record_out does (FOU3D.f90:2063-2165).
    The header carries t, iter and the current mpgx (which the constant flow
    rate mode changes; default: the description's)."""
    mp = desc.mpgx if mpgx is None else float(mpgx)
    N = np.zeros((4, 5), np.int32)
    N[0, 1:4] = desc.Nx
    N[0, 4] = -2
    N[1, 1:4] = desc.Nz
    N[2, 3] = desc.nyv
    N[3, 3] = desc.nyu
    for name, arr, lo, y, dth, ident in (("u1", u1, 0, yu, dthdyu, 1), ("u2", u2, 0, yv, dthdyv, 2),
                                         ("u3", u3, 0, yu, dthdyu, 3), ("p", p, 1, yu, dthdyu, 4)):
        with open(os.path.join(dirout, name + tag), "wb") as f:
            h = struct.pack("<5d", t, desc.Re, desc.alp, desc.bet, mp) + struct.pack("<2i", 3, it)
            h += np.zeros(88, np.int32).tobytes()
            f.write(_rec(h))
            f.write(_rec(N.T.astype("<i4").tobytes()))
            f.write(_rec(np.concatenate([y, [1.0], dth]).astype("<f8").tobytes()))
            for jj in range(arr.shape[1]):
                j = jj + lo
                buf = _cols_to_plane(arr[:, jj], desc.Nx, desc.Nz)
                rec = struct.pack("<4i", j, ident, desc.Nx + 2, desc.Nz) + struct.pack("<d", y[j])
                rec += np.asfortranarray(buf).T.astype("<f8").tobytes()
                f.write(_rec(rec))
