"""GPU parity of the sm_100a engine against the C oracle, through the C ABI.

Bars (per field, relative L2 over all stored complex entries):
* plane transforms (cft/rft restated) and tridiagonal solves: <= 1e-13;
* one RK3 step from the same initial fields: <= 1e-12 for u1, u2, u3, p;
* ten RK3 steps: <= 1e-9.
Index maps and masks are checked bit for bit on the nonlinear-term
intermediates (zero rows/columns exactly zero).
"""
import numpy as np
import pytest

import oracle as O
from helpers import golden_ic, oracle_cfg, rel_l2

pytestmark = pytest.mark.gpu

FIELDS = ("u1", "u2", "u3", "p")


def _engine(desc):
    from lh_b200 import Engine
    return Engine(desc)


def _random_spectral_planes(o, nplanes, seed, full=False):
    rng = np.random.default_rng(seed)
    pl = np.zeros((nplanes, o.kgal, o.igal))
    nxh = o.Nx // 2 + 1
    rows = list(range(o.Nz // 2)) + list(range(o.Mz - o.Nz // 2, o.Mz))
    for n in range(nplanes):
        if full:
            pl[n] = rng.standard_normal((o.kgal, o.igal))
        else:
            for r in rows:
                pl[n, r, :2 * nxh] = rng.standard_normal(2 * nxh)
    return pl


@pytest.mark.parametrize("N", [8, 32, 64, 128])
def test_four_to_phys_matches_oracle(N):
    from lh_b200 import Desc
    d = Desc(Nx=N, Nz=N, ny=17)
    e = _engine(d)
    o = O.Oracle(oracle_cfg(d))
    for full in (False, True):
        pl = _random_spectral_planes(o, 3, 11 + N, full)
        got = e.four_to_phys(pl).reshape(pl.shape)
        for n in range(pl.shape[0]):
            ref = o.four_to_phys(pl[n].ravel()).reshape(o.kgal, o.igal)
            assert rel_l2(got[n], ref) <= 1e-13, (N, full, n)


@pytest.mark.parametrize("N", [8, 32, 64, 128])
def test_phys_to_four_matches_oracle(N):
    from lh_b200 import Desc
    d = Desc(Nx=N, Nz=N, ny=17)
    e = _engine(d)
    o = O.Oracle(oracle_cfg(d))
    rng = np.random.default_rng(5 + N)
    pl = rng.standard_normal((3, o.kgal, o.igal))
    got = e.phys_to_four(pl).reshape(pl.shape)
    for n in range(3):
        ref = o.phys_to_four(pl[n].ravel()).reshape(o.kgal, o.igal)
        assert rel_l2(got[n], ref) <= 1e-13
        # the oddball row Mz/2+1 is exactly zero (FOU3D.f90:1670)
        assert np.all(got[n, o.Mz // 2] == 0.0)


@pytest.mark.parametrize("grid,kRK", [(2, 1), (2, 3), (1, 2)])
def test_lusolu_matches_oracle(grid, kRK):
    from lh_b200 import Desc
    d = Desc(Nx=16, Nz=16, ny=65, dt_mode=1, dt=2e-3)
    e = _engine(d)
    o = O.Oracle(oracle_cfg(d))
    o.set_scalar(1, d.dt)
    n = (d.nyu + 2) if grid == 2 else (d.nyv + 2)
    rng = np.random.default_rng(kRK)
    rhs = rng.standard_normal((d.ncols, n)) + 1j * rng.standard_normal((d.ncols, n))
    got = e.lusolu(grid, kRK, d.dt, rhs)
    ref = np.zeros_like(rhs)
    rb = np.ascontiguousarray(rhs).view(np.float64).ravel()
    ub = np.zeros_like(rb)
    o.L.lho_lusolu(o.h, grid, kRK, O._dp(rb), O._dp(ub))
    ref = ub.view(np.complex128).reshape(d.ncols, n)
    assert rel_l2(got, ref) <= 1e-13


def test_lusolp_matches_oracle():
    from lh_b200 import Desc
    d = Desc(Nx=16, Nz=16, ny=65)
    e = _engine(d)
    o = O.Oracle(oracle_cfg(d))
    rng = np.random.default_rng(3)
    x = rng.standard_normal((d.ncols, d.nyu)) + 1j * rng.standard_normal((d.ncols, d.nyu))
    got = e.lusolp(x)
    xb = np.ascontiguousarray(x).view(np.float64).ravel().copy()
    o.L.lho_lusolp(o.h, O._dp(xb))
    ref = xb.view(np.complex128).reshape(d.ncols, d.nyu)
    assert rel_l2(got, ref) <= 1e-12


def _run_both(desc, ic, nsteps, threaded=False):
    e = _engine(desc)
    e.upload(*ic)
    e.step(nsteps)
    e.synchronize()
    g = e.download()
    o = O.Oracle(oracle_cfg(desc), threaded=threaded)
    o.load_state(*ic)
    o.step(nsteps)
    r = o.state()
    return e, g, o, r


def test_substep_intermediates_bitexact_masks():
    from lh_b200 import Desc
    d = Desc()  # reference input.in: 32x32x153, CFL 0.7
    ic = golden_ic()
    e = _engine(d)
    e.upload(*ic)
    e.substep(1)
    e.synchronize()
    o = O.Oracle(oracle_cfg(d))
    o.load_state(*ic)
    o.substep(1)
    # Nu x/z parts, y-flux spectra
    for w in range(6):
        g = e.intermediate(w)
        r = o.intermediate(w)
        assert g.shape == r.shape, (w, g.shape, r.shape)
        assert rel_l2(g, r) <= 1e-12, (w, rel_l2(g, r))
        # zeros where the reference writes zeros, bit for bit
        assert np.array_equal(g == 0, r == 0) or w >= 3, w
    nxh = d.Nx // 2 + 1
    nu1 = e.intermediate(0)
    assert np.all(nu1[(d.Nz // 2) * nxh:(d.Nz // 2 + 1) * nxh] == 0.0)  # kz = -Nz/2 row
    uvf = e.intermediate(3)
    assert np.all(uvf[:, 0] == 0.0)  # plane 0 never computed (reads as zero)
    vvc = e.intermediate(4)
    assert np.all(vvc[:, 0] == 0.0) and np.all(vvc[:, -1] == 0.0)
    g = e.download()
    r = o.state()
    for f in FIELDS:
        assert rel_l2(g[f], r[f]) <= 1e-12, (f, rel_l2(g[f], r[f]))
    s = e.scalars()
    assert abs(s["dt"] - o.scalar(1)) <= 1e-14 * o.scalar(1)


def test_one_and_ten_steps_reference_ic_cfl():
    from lh_b200 import Desc
    d = Desc()
    ic = golden_ic()
    e, g, o, r = _run_both(d, ic, 1)
    errs = {f: rel_l2(g[f], r[f]) for f in FIELDS}
    print("1 step errors", errs)
    assert all(v <= 1e-12 for v in errs.values()), errs
    assert abs(e.scalars()["t"] - o.scalar(0)) <= 1e-13 * o.scalar(0)
    assert e.error_div() < 1e-11
    e.step(9)
    e.synchronize()
    o.step(9)
    g, r = e.download(), o.state()
    errs = {f: rel_l2(g[f], r[f]) for f in FIELDS}
    print("10 step errors", errs)
    assert all(v <= 1e-9 for v in errs.values()), errs
    assert e.scalars()["iter"] == 10


@pytest.mark.parametrize("grid_type,ctpress", [(0, 1), (1, 1), (0, 0)])
def test_fixed_dt_synthetic_ic(grid_type, ctpress):
    from lh_b200 import Desc, grids, perturbed_laminar
    d = Desc(Nx=32, Nz=32, ny=97, grid_type=grid_type, flag_ctpress=ctpress, dt_mode=1, dt=1e-3)
    yu, yv = grids(d)
    ic = perturbed_laminar(d, 20260001, yu, yv)
    e, g, o, r = _run_both(d, ic, 1)
    errs = {f: rel_l2(g[f], r[f]) for f in FIELDS}
    assert all(v <= 1e-12 for v in errs.values()), errs
    e.step(9)
    e.synchronize()
    o.step(9)
    g, r = e.download(), o.state()
    errs = {f: rel_l2(g[f], r[f]) for f in FIELDS}
    assert all(v <= 1e-9 for v in errs.values()), errs
    if ctpress == 0:
        # mpgx accumulates g = (QxT - Qx0)/Qx1, a difference of nearly equal
        # flow rates, so its relative error is larger than the fields'
        assert abs(e.scalars()["mpgx"] - o.scalar(3)) <= 1e-8 * abs(o.scalar(3))


def test_one_step_128():
    from lh_b200 import Desc, grids, perturbed_laminar
    d = Desc(Nx=128, Nz=128, ny=153, dt_mode=1, dt=5e-4)
    yu, yv = grids(d)
    ic = perturbed_laminar(d, 20260002, yu, yv)
    e, g, o, r = _run_both(d, ic, 1, threaded=True)
    errs = {f: rel_l2(g[f], r[f]) for f in FIELDS}
    print("128^2 one step", errs)
    assert all(v <= 1e-12 for v in errs.values()), errs


def test_step_host_matches_device_path():
    from lh_b200 import Desc
    d = Desc()
    ic = golden_ic()
    e = _engine(d)
    e.upload(*ic)
    e.step(2)
    e.synchronize()
    ref = e.download()
    bufs = [np.ascontiguousarray(x).copy() for x in ic]
    e2 = _engine(d)
    e2.step_host(bufs, 2)
    for f, b in zip(FIELDS, bufs):
        assert np.array_equal(b, ref[f]), f


@pytest.mark.parametrize("N", [32, 64, 128, 192, 256])
def test_fast_and_generic_fft_paths_agree(N, monkeypatch):
    """The compile-time-sized plane kernels and the generic ones give the
    same step to round-off (both are checked against the oracle above), at
    every Ngal size of the fast path the configs use (48 ... 384).  The
    velocities agree to 1e-13; p, whose (0,0) Poisson solve amplifies
    last-bit differences of its right-hand side, to 1e-12."""
    from lh_b200 import Desc, grids, perturbed_laminar
    d = Desc(Nx=N, Nz=N, ny=65, dt_mode=1, dt=1e-3)
    yu, yv = grids(d)
    ic = perturbed_laminar(d, 5, yu, yv)
    out = []
    for gen in ("0", "1"):
        monkeypatch.setenv("LH_GENERIC_FFT", gen)
        e = _engine(d)
        e.upload(*ic)
        e.step(2)
        e.synchronize()
        out.append(e.download())
    for f in FIELDS:
        assert rel_l2(out[0][f], out[1][f]) <= (1e-12 if f == "p" else 1e-13), f


@pytest.mark.parametrize("N,ctpress,ny", [(16, 1, 97), (32, 0, 97), (64, 1, 97), (128, 1, 97), (32, 1, 257)])
def test_small_and_sequential_column_passes_agree(N, ctpress, ny, monkeypatch):
    """The one-CTA-per-column pass (warp scans over the y rows) and the
    32-columns-per-CTA sequential pass give the same steps: only the values
    entering each lane's block of rows are formed in a different order.  Both
    are forced through LH_SMALL_COLUMNS, whichever the size would pick."""
    from lh_b200 import Desc, grids, perturbed_laminar
    d = Desc(Nx=N, Nz=N, ny=ny, flag_ctpress=ctpress, dt_mode=1, dt=1e-3)
    yu, yv = grids(d)
    ic = perturbed_laminar(d, 7, yu, yv)
    out = []
    for limit in ("0", "1000000000"):
        monkeypatch.setenv("LH_SMALL_COLUMNS", limit)
        e = _engine(d)
        e.upload(*ic)
        e.step(3)
        e.synchronize()
        out.append((e.download(), e.scalars()))
    for f in FIELDS:
        assert rel_l2(out[0][0][f], out[1][0][f]) <= (1e-12 if f == "p" else 1e-13), f
    if ctpress == 0:
        assert abs(out[0][1]["mpgx"] - out[1][1]["mpgx"]) <= 1e-10 * abs(out[0][1]["mpgx"])
