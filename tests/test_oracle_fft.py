"""Oracle FFTPACK restatement against numpy's FFT and the reference's rules.

Conventions checked (cft_buff.f:1-65, rft_buff.f:24-86):
* cft backward: unnormalised e^{+i}; forward: e^{-i} times 1/n;
* rft forward: half-complex cc(k) = X_k/n packed at (2k+1, 2k+2), with
  Im(cc(0)) = Im(cc(n/2)) = 0; inverse ignores both imaginary parts.
"""
import numpy as np
import pytest

import oracle as O

SIZES = [6, 12, 48, 96, 144, 192, 288, 384]


def test_factor_orders_follow_fftpack_rules():
    # cffti1 tries 3,4,2,5 and moves a factor 2 to the front (cft_buff.f:141-163)
    assert O.fft_factors(192, real=False) == [3, 4, 4, 4]
    assert O.fft_factors(96, real=False) == [2, 3, 4, 4]
    assert O.fft_factors(48, real=False) == [3, 4, 4]
    assert O.fft_factors(288, real=False) == [2, 3, 3, 4, 4]
    # rffti1 tries 4,2,3,5 (rft_buff.f:133-160)
    assert O.fft_factors(192, real=True) == [4, 4, 4, 3]
    assert O.fft_factors(96, real=True) == [2, 4, 4, 3]
    assert O.fft_factors(48, real=True) == [4, 4, 3]


def test_rejects_non_smooth_lengths():
    with pytest.raises(ValueError):
        O.fft_factors(80, real=True)     # factor 5: the reference's rfft stops
    with pytest.raises(ValueError):
        O.fft_factors(14, real=False)


@pytest.mark.parametrize("n", SIZES)
def test_cft_matches_numpy(n):
    rng = np.random.default_rng(n)
    m, ise = 5, 2 * 5 + 2      # 5 vectors, stride between elements in reals
    z = rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))
    c = np.zeros(ise * n)
    for k in range(m):
        c[2 * k::ise][:n] = z[:, k].real
        c[2 * k + 1::ise][:n] = z[:, k].imag
    back = O.cft(c, ise, 2, m, +1, n)
    fwd = O.cft(c, ise, 2, m, -1, n)
    for k in range(m):
        zb = back[2 * k::ise][:n] + 1j * back[2 * k + 1::ise][:n]
        zf = fwd[2 * k::ise][:n] + 1j * fwd[2 * k + 1::ise][:n]
        ref_b = np.fft.ifft(z[:, k]) * n
        ref_f = np.fft.fft(z[:, k]) / n
        assert np.max(np.abs(zb - ref_b)) <= 1e-13 * np.max(np.abs(ref_b))
        assert np.max(np.abs(zf - ref_f)) <= 1e-13 * np.max(np.abs(ref_f))


@pytest.mark.parametrize("n", [s for s in SIZES if s % 2 == 0])
def test_rft_matches_numpy(n):
    rng = np.random.default_rng(100 + n)
    m, isa = 4, n + 2
    x = rng.standard_normal((m, n))
    c = np.zeros(isa * m)
    for j in range(m):
        c[j * isa:j * isa + n] = x[j]
    f = O.rft(c, isa, m, -1, n)
    for j in range(m):
        row = f[j * isa:(j + 1) * isa]
        cc = row[0::2] + 1j * row[1::2]
        ref = np.fft.rfft(x[j]) / n
        ref[0] = ref[0].real
        ref[-1] = ref[-1].real
        assert np.max(np.abs(cc - ref)) <= 1e-14 * np.max(np.abs(ref))
        assert row[1] == 0.0 and row[n + 1] == 0.0
    # inverse: Hermitian synthesis, unnormalised, Im(0) and Im(n/2) ignored
    spec = rng.standard_normal((m, n // 2 + 1)) + 1j * rng.standard_normal((m, n // 2 + 1))
    c = np.zeros(isa * m)
    for j in range(m):
        c[j * isa:(j + 1) * isa:2] = spec[j].real
        c[j * isa + 1:(j + 1) * isa:2] = spec[j].imag
    b = O.rft(c, isa, m, +1, n)
    for j in range(m):
        s = spec[j].copy()
        s[0] = s[0].real
        s[-1] = s[-1].real
        ref = np.fft.irfft(s, n) * n
        got = b[j * isa:j * isa + n]
        assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_plane_round_trip():
    o = O.Oracle(O.Config(Nx=8, Nz=8, ny=9))
    rng = np.random.default_rng(7)
    plane = np.zeros((o.kgal, o.igal))
    # spectral content only where modes_to_planes puts columns
    for col in range(1, o.ncols + 1):
        pass
    nxh = o.Nx // 2 + 1
    rows = list(range(0, o.Nz // 2)) + list(range(o.Mz - o.Nz // 2, o.Mz))
    for r in rows:
        plane[r, :2 * nxh] = rng.standard_normal(2 * nxh)
    phys = o.four_to_phys(plane.ravel())
    back = o.phys_to_four(phys).reshape(o.kgal, o.igal)
    # the kx=0 imaginary part and the kx=Nx/2 column survive only in
    # Hermitian form; compare the modes the solver keeps (kz=-Nz/2 and the
    # Nyquist pair are not invariant under a real round trip)
    keep = [r for r in rows if r != o.Mz - o.Nz // 2]
    for r in keep:
        a, b = plane[r, 2:2 * (nxh - 1)], back[r, 2:2 * (nxh - 1)]
        assert np.max(np.abs(a - b)) < 1e-13
