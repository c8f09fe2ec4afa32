"""Oracle known-answer tests against the reference's own data and rules.

* ygrid (start.f90:665-806) reproduces the grid stored in the reference's
  input files bit for bit (tests/golden/grid_ny153_dyq10_p5.npz).
* der_x / der_z masks (FOU3D.f90:420-523), checked against an independent
  statement of the rule and a literal table for the fill pattern of
  test_der_x.f90:20-24 (u(i,k) = 100 k + i); der_z_N (FOU3D.f90:525-546)
  against the case of test_der_z.f90 (u(i,k) = 10 k + i, kz = i, 2i).
* After a full RK3 step from the reference's 32x32x153 initial condition the
  projected field is divergence-free to round-off (error(), littleharsh.f90:
  370-409) and the time step follows the CFL rule (FOU3D.f90:290-303).
* The spectra of flagged steps (spectra.f90:7-66) against a direct statement
  of buildsp/buildspUV with interp_v.
* The plane stats (stats.f90:1-97) and omega_x (FOU3D.f90:314-338) against a
  numpy statement with numpy's FFT in the reference's conventions.
"""
import os

import numpy as np
import pytest

import oracle as O


def test_grid_bit_exact(golden_dir):
    g = np.load(os.path.join(golden_dir, "grid_ny153_dyq10_p5.npz"))
    o = O.Oracle(O.Config())
    assert np.array_equal(o.array(0), g["yu"])
    assert np.array_equal(o.array(1), g["yv"])
    assert np.array_equal(o.array(2), g["dthdyu"])
    assert np.array_equal(o.array(3), g["dthdyv"])


def _rule_der(o, u, axis):
    """Independent statement of der_x/der_z on the complex plane view."""
    Nx, Nz, Mx, Mz, ig = o.Nx, o.Nz, o.Mx, o.Mz, o.igal
    kx = o.array(7)
    kz = o.array(8)
    out = np.zeros_like(u)
    uc = u.reshape(Mz, ig)
    oc = out.reshape(Mz, ig)
    for k in range(1, Mz + 1):
        if k <= Nz // 2:
            kidx = k
        elif k >= Mz - Nz // 2 + 2:
            kidx = k + Nz - Mz
        else:
            continue  # rows Nz/2+1 .. Mz-Nz/2+1 are zero (includes kz=-Nz/2)
        for i in range(0, Nx // 2 + 1):
            w = kx[i] if axis == "x" else kz[kidx - 1]
            re, im = uc[k - 1, 2 * i], uc[k - 1, 2 * i + 1]
            oc[k - 1, 2 * i] = 0.0 * re - w * im
            oc[k - 1, 2 * i + 1] = 0.0 * im + w * re
    return out


@pytest.mark.parametrize("N", [4, 8, 32])
def test_der_masks_match_rule(N):
    o = O.Oracle(O.Config(Nx=N, Nz=N, ny=9, alp=1.0, bet=1.0))
    u = np.zeros((o.kgal, o.igal))
    for k in range(1, o.kgal + 1):
        for i in range(0, o.igal):
            u[k - 1, i] = 100.0 * k + i
    u = u.ravel()
    dx = o.der_x(u)
    dz = o.der_z(u)
    # der_x/der_z write the complex view (0:Mx/2); slots Mx+1..Mx+2 are the
    # last complex entry and are written as well
    assert np.array_equal(dx, _rule_der(o, u, "x"))
    assert np.array_equal(dz, _rule_der(o, u, "z"))


def test_der_x_literal_table():
    # Nx=Nz=4 -> Mx=Mz=6, kx = i (alp = 1), u(i,k) = 100k + i packed real
    o = O.Oracle(O.Config(Nx=4, Nz=4, ny=9, alp=1.0, bet=1.0))
    u = np.array([[100.0 * k + i for i in range(o.igal)] for k in range(1, o.kgal + 1)]).ravel()
    d = o.der_x(u).reshape(o.kgal, o.igal)
    # rows 1,2 (kz = 0, 1) and row 6 (kz = -1) keep i = 0..2; rows 3..5 zero
    expect = np.zeros((6, 8))
    for k in (1, 2, 6):
        for i in range(3):
            re, im = 100.0 * k + 2 * i, 100.0 * k + 2 * i + 1
            expect[k - 1, 2 * i] = -i * im
            expect[k - 1, 2 * i + 1] = i * re
    assert np.array_equal(d, expect)
    assert d[1, 2:4].tolist() == [-203.0, 202.0]       # row 2, i = 1
    assert d[4].tolist() == [0.0] * 8                   # row 5: kz = -Nz/2 zeroed


def test_der_z_n_literal_table():
    """test_der_z.f90: Nspec_x = 4, Nspec_z = 2, u(i,k) = 10k + i packed real,
    kz = (0,1), (0,2): dudz = kz u on every complex entry (der_z_N,
    FOU3D.f90:525-546, no masking)."""
    u = np.array([[10.0 * k + i for i in range(1, 7)] for k in (1, 2)])
    d = O.der_z_n(u, [1.0, 2.0], 4, 2)
    expect = np.array([[-12.0, 11.0, -14.0, 13.0, -16.0, 15.0],
                       [-44.0, 42.0, -48.0, 46.0, -52.0, 50.0]])
    assert np.array_equal(d, expect)


def test_one_step_from_reference_ic(golden_dir):
    ic = np.load(os.path.join(golden_dir, "ref_ic_0032x0032x0153.npz"))
    o = O.Oracle(O.Config())
    o.load_state(ic["u1"], ic["u2"], ic["u3"], ic["p"])
    o.step(1)
    assert o.error_div() < 1e-12
    # CFL rule: dt = min(2.5 dtv, CFL * dtc)
    dtv = o.array(6)[6]
    assert o.scalar(1) == min(2.5 * dtv, 0.7 * o.scalar(7))
    s = o.state()
    assert np.all(np.isfinite(s["u1"])) and abs(s["u2"][:, 0]).max() == 0.0


def test_oracle_spectra_follow_spectra_f90():
    """lho_spectra adds, per (y row, column), |u1|^2, |u2|^2, |u3|^2, |p|^2 and
    Re(u1) Re(u2i) + Im(u1) Im(u2i) with u2i = interp_v(u2) (spectra.f90:7-66,
    FOU3D.f90:394-418); two accumulations of one state give twice the terms."""
    from lh_b200 import Desc, grids, perturbed_laminar
    d = Desc(Nx=16, Nz=16, ny=33, dt_mode=1, dt=1e-3)
    yu, yv = grids(d)
    o = O.Oracle(O.Config(Nx=16, Nz=16, ny=33, dt_mode=O.DT_FIXED, dt_fixed=1e-3))
    o.load_state(*perturbed_laminar(d, 3, yu, yv))
    o.step(1)
    st = o.state()
    acc = o.spectra(o.spectra())
    u1, u2, u3, p = st["u1"], st["u2"], st["u3"], st["p"]
    nyu = d.nyu
    ui = np.zeros_like(u1)
    for j in range(1, nyu + 1):
        ui[:, j] = ((yu[j] - yv[j - 1]) * u2[:, j] + (yv[j] - yu[j]) * u2[:, j - 1]) / (yv[j] - yv[j - 1])
    g1 = (yu[0] - yu[1]) / (yv[0] - yu[1])
    g2 = (yu[nyu + 1] - yu[nyu]) / (yv[nyu] - yu[nyu])
    ui[:, 0] = g1 * (u2[:, 0] - ui[:, 1]) + ui[:, 1]
    ui[:, -1] = g2 * (u2[:, -1] - ui[:, -2]) + ui[:, -2]
    ref = {"spU": 2 * abs(u1) ** 2, "spV": 2 * abs(u2) ** 2, "spW": 2 * abs(u3) ** 2,
           "spUV": 2 * (u1.real * ui.real + u1.imag * ui.imag), "spP": 2 * abs(p) ** 2}
    for k, r in ref.items():
        assert acc[k].shape == r.shape, k
        assert np.max(abs(acc[k] - r)) <= 1e-14 * np.max(abs(r)), k


def _ngal_planes(o, x):
    """columns [col, j] -> spectral planes [j, Mz, Nx/2+1] in the dealiased row
    order of modes_to_planes_UVP (start.f90:1031-1040)."""
    nxh = o.Nx // 2 + 1
    X = x.T.reshape(x.shape[1], o.Nz, nxh)
    P = np.zeros((x.shape[1], o.Mz, nxh), complex)
    P[:, :o.Nz // 2] = X[:, :o.Nz // 2]
    P[:, o.Mz - o.Nz // 2:] = X[:, o.Nz // 2:]
    return P


def _to_phys(P, M):
    """cft backward (unscaled) along z, then rft backward along x, which
    ignores the imaginary parts of modes 0 and M/2 (rft_buff.f:78-81)."""
    c = np.fft.ifft(P, axis=1) * P.shape[1]
    full = np.zeros(P.shape[:2] + (M // 2 + 1,), complex)
    full[..., :P.shape[2]] = c
    return np.fft.irfft(full, n=M, axis=2) * M


def test_oracle_stats_follow_stats_f90():
    """lho_stats against a numpy statement of stats() as nonlinear() calls it
    (FOU3D.f90:240, 307-341): planes 1..nyu in physical space after
    four_to_phys_u, wall planes over the spectral coefficients (Re + Im
    entries), Pm/P2m over the pressure snapshot's coefficients, wxm/wx2m over
    omega_x = -d(u2)/dz + d(u3)/dy at the faces in physical space of the
    Nspec grid (FOU3D.f90:314-338)."""
    from lh_b200 import Desc, grids, perturbed_laminar
    N, ny = 16, 33
    d = Desc(Nx=N, Nz=N, ny=ny, dt_mode=1, dt=1e-3)
    yu, yv = grids(d)
    o = O.Oracle(O.Config(Nx=N, Nz=N, ny=ny, dt_mode=O.DT_FIXED, dt_fixed=1e-3))
    o.load_state(*perturbed_laminar(d, 3, yu, yv))
    o.step(1)
    o.pressure_snapshot()
    pp = o.state()["p"]
    o.step(1)
    acc = o.stats()
    st = o.state()
    u1, u2, u3 = st["u1"], st["u2"], st["u3"]
    nyu, nyv, Mx, Mz = d.nyu, d.nyv, o.Mx, o.Mz
    # interpolations (interp_v, interp_u; FOU3D.f90:373-418)
    u2i = np.zeros_like(u1)
    for j in range(1, nyu + 1):
        u2i[:, j] = ((yu[j] - yv[j - 1]) * u2[:, j] + (yv[j] - yu[j]) * u2[:, j - 1]) / (yv[j] - yv[j - 1])
    g1 = (yu[0] - yu[1]) / (yv[0] - yu[1])
    g2 = (yu[nyu + 1] - yu[nyu]) / (yv[nyu] - yu[nyu])
    u2i[:, 0] = g1 * (u2[:, 0] - u2i[:, 1]) + u2i[:, 1]
    u2i[:, -1] = g2 * (u2[:, -1] - u2i[:, -2]) + u2i[:, -2]
    u3i = np.zeros_like(u2)
    for j in range(nyv + 2):
        u3i[:, j] = ((yv[j] - yu[j]) * u3[:, j + 1] + (yu[j + 1] - yv[j]) * u3[:, j]) / (yu[j + 1] - yu[j])
    pad = lambda a: np.concatenate([a, np.zeros((a.shape[0], nyu + 2 - a.shape[1]), complex)], axis=1)
    F = {k: _ngal_planes(o, v) for k, v in
         (("a", u1), ("w", u3), ("vi", u2i), ("v", pad(u2)), ("wi", pad(u3i)))}
    ph = {k: _to_phys(v[1:nyu + 1], Mx) for k, v in F.items()}
    ref = np.zeros((13, nyu + 2))
    lin = lambda z: (z.real + z.imag).sum()
    dot = lambda x, y: (x.real * y.real + x.imag * y.imag).sum()
    for j in (0, nyu + 1):   # wall planes keep their spectral coefficients
        a, w, vi, v, wi = (F[k][j] for k in ("a", "w", "vi", "v", "wi"))
        ref[:9, j] = [lin(a), dot(a, a), lin(v), dot(v, v), lin(w), dot(w, w), dot(a, vi), dot(a, w), dot(v, wi)]
    a, w, vi, v, wi = (ph[k] for k in ("a", "w", "vi", "v", "wi"))
    S = lambda x: x.sum(axis=(1, 2))
    ref[:9, 1:nyu + 1] = [S(a), S(a * a), S(v), S(v * v), S(w), S(w * w), S(a * vi), S(a * w), S(v * wi)]
    for j in range(1, nyu + 1):
        ref[9, j], ref[10, j] = lin(pp[:, j - 1]), dot(pp[:, j - 1], pp[:, j - 1])
    # omega_x spectral (der_z_N, der_yv_h_wx), then four_to_phys_N on the Nspec grid
    dthdyv = o.array(3)
    kz = d.bet * np.repeat(np.where(np.arange(N) < N // 2, np.arange(N), np.arange(N) - N), N // 2 + 1)
    wxh = np.zeros((u1.shape[0], nyu + 2), complex)
    for j in range(nyv + 2):
        wxh[:, j] = -(1j * kz * u2[:, j]) + (u3[:, j + 1] - u3[:, j]) * dthdyv[j]
    wxp = _to_phys(wxh.T.reshape(nyu + 2, N, N // 2 + 1), N)
    ref[11], ref[12] = S(wxp), S(wxp * wxp)
    fmax = max(np.max(abs(x)) for x in ph.values())
    n = Mx * Mz
    for q, name in enumerate(O.Oracle.STATS):
        if name.startswith("wx"):
            scale = N * N * np.max(abs(wxp)) ** (2 if name == "wx2m" else 1)
        else:
            scale = n * fmax ** (1 if name in ("Um", "Vm", "Wm", "Pm") else 2)
        assert np.max(abs(acc[q] - ref[q])) <= 1e-13 * scale, (name, np.max(abs(acc[q] - ref[q])), scale)
    # the wall planes and the pressure rows are plain sums of coefficients
    assert np.allclose(acc[9:11], ref[9:11], rtol=1e-13, atol=0)
    assert acc[9, 0] == 0.0 and acc[9, nyu + 1] == 0.0


def test_oracle_omega_x_is_the_curl_on_the_nspec_grid():
    """lho_omega_x equals the x vorticity of the state evaluated by numpy on
    the Nx x Nz grid: -d(u2)/dz from the spectral derivative and
    d(u3)/dy from the face difference, planes 0..nyv+1, zero above."""
    from lh_b200 import Desc, grids, perturbed_laminar
    N, ny = 16, 33
    d = Desc(Nx=N, Nz=N, ny=ny, dt_mode=1, dt=1e-3)
    yu, yv = grids(d)
    o = O.Oracle(O.Config(Nx=N, Nz=N, ny=ny, dt_mode=O.DT_FIXED, dt_fixed=1e-3))
    o.load_state(*perturbed_laminar(d, 5, yu, yv))
    wx = o.omega_x()
    st = o.state()
    u2, u3 = st["u2"], st["u3"]
    dthdyv = o.array(3)
    kz = d.bet * np.repeat(np.where(np.arange(N) < N // 2, np.arange(N), np.arange(N) - N), N // 2 + 1)
    wxh = np.zeros((u2.shape[0], d.nyu + 2), complex)
    for j in range(d.nyv + 2):
        wxh[:, j] = -(1j * kz * u2[:, j]) + (u3[:, j + 1] - u3[:, j]) * dthdyv[j]
    ref = _to_phys(wxh.T.reshape(d.nyu + 2, N, N // 2 + 1), N)
    assert wx.shape == (d.nyu + 2, N, N + 2)
    assert np.max(abs(wx[:, :, :N] - ref)) <= 1e-13 * np.max(abs(ref))
    assert not np.any(wx[d.nyu + 1])
