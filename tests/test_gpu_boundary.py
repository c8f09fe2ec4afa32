"""The tridiagonal factor entries and the continued-run entry of the C ABI.

* lh_tridiag_factor equals the oracle's LU_build + LU_dec (tridLU_3D.f90:
  163-221, 327-364) bit for bit on both velocity grids, and returns the
  DG factors of LU_buildP + LU_decP (:224-297, 366-407) bit for bit;
* lh_tridiag_solve with those factors equals lh_lusolu / lh_lusolp (the
  solves of LUsolU / LUsolP) bit for bit;
* lh_set_dg installs a caller's DG: the engine's own DG leaves a step
  unchanged, a different one is what lh_lusolp then solves with, and a DG
  whose lower diagonal varies by column is rejected;
* lh_set_scalars continues a run from a restart file (getini with
  flag_init = 2, start.f90:1268-1282): N steps, record_out's file format
  written and read back, N more steps equal 2N uninterrupted steps bit for
  bit.
"""
import numpy as np
import pytest

import oracle as O
from helpers import oracle_cfg

pytestmark = pytest.mark.gpu

FIELDS = ("u1", "u2", "u3", "p")


@pytest.mark.parametrize("grid,kRK,dt", [(2, 1, 1e-3), (2, 3, 2e-3), (1, 2, 5e-4)])
def test_tridiag_factor_matches_oracle(grid, kRK, dt):
    from lh_b200 import Desc, Engine
    d = Desc(Nx=32, Nz=16, ny=97, dt_mode=1, dt=dt)
    e = Engine(d)
    got = e.tridiag_factor(grid, kRK, dt)
    o = O.Oracle(oracle_cfg(d))
    o.set_scalar(1, dt)
    rows = d.nyu + 2 if grid == 2 else d.nyv + 2
    ref = np.zeros(3 * rows * d.ncols)
    o.L.lho_lu_factor(o.h, grid, kRK, O._dp(ref))
    assert np.array_equal(got.ravel(), ref)


def test_dg_matches_oracle_and_solves():
    from lh_b200 import Desc, Engine
    d = Desc(Nx=32, Nz=16, ny=97)
    e = Engine(d)
    dg = e.tridiag_factor(3)
    o = O.Oracle(oracle_cfg(d))
    assert np.array_equal(dg.ravel(), o.array(11))
    rng = np.random.default_rng(2)
    x = rng.standard_normal((d.ncols, d.nyu)) + 1j * rng.standard_normal((d.ncols, d.nyu))
    assert np.array_equal(e.tridiag_solve(3, dg, x), e.lusolp(x))


@pytest.mark.parametrize("grid,kRK", [(2, 2), (1, 3)])
def test_tridiag_solve_matches_lusolu(grid, kRK):
    from lh_b200 import Desc, Engine
    d = Desc(Nx=32, Nz=16, ny=97, dt_mode=1, dt=1e-3)
    e = Engine(d)
    a = e.tridiag_factor(grid, kRK, d.dt)
    n = d.nyu + 2 if grid == 2 else d.nyv + 2
    rng = np.random.default_rng(grid + kRK)
    x = rng.standard_normal((d.ncols, n)) + 1j * rng.standard_normal((d.ncols, n))
    assert np.array_equal(e.tridiag_solve(grid, a, x), e.lusolu(grid, kRK, d.dt, x))


def test_set_dg():
    from lh_b200 import Desc, Engine, LHError, grids, perturbed_laminar
    d = Desc(Nx=32, Nz=32, ny=97, dt_mode=1, dt=1e-3)
    ic = perturbed_laminar(d, 3, *grids(d))
    runs = []
    for install in (False, True):
        e = Engine(d)
        if install:
            e.set_dg(e.tridiag_factor(3))
        e.upload(*ic)
        e.step(2)
        e.synchronize()
        runs.append(e.download())
    for f in FIELDS:
        assert np.array_equal(runs[0][f], runs[1][f]), f
    # another DG (pivots scaled by 2) is the one the Poisson solve then uses
    e = Engine(d)
    dg = e.tridiag_factor(3).copy()
    dg[:, :, 1] *= 2.0
    e.set_dg(dg)
    assert np.array_equal(e.tridiag_factor(3), dg)
    rng = np.random.default_rng(4)
    x = rng.standard_normal((d.ncols, d.nyu)) + 1j * rng.standard_normal((d.ncols, d.nyu))
    assert np.array_equal(e.lusolp(x), e.tridiag_solve(3, dg, x))
    bad = dg.copy()
    bad[5, 10, 0] += 1.0
    with pytest.raises(LHError):
        e.set_dg(bad)


@pytest.mark.parametrize("ctpress,cfl", [(1, False), (1, True), (0, False)])
def test_continue_from_restart_file(tmp_path, ctpress, cfl):
    from lh_b200 import Desc, Engine, grids, perturbed_laminar
    from lh_b200.state import read_state, write_state
    d = Desc(Nx=32, Nz=32, ny=97, flag_ctpress=ctpress, dt_mode=0 if cfl else 1, dt=1e-3)
    yu, yv = grids(d)
    ic = perturbed_laminar(d, 9, yu, yv)
    n = 3
    a = Engine(d)
    a.upload(*ic)
    a.step(2 * n)
    a.synchronize()
    ref, ref_sc = a.download(), a.scalars()
    b = Engine(d)
    b.upload(*ic)
    b.step(n)
    b.synchronize()
    st, sc = b.download(), b.scalars()
    write_state(str(tmp_path), "_restart.dat", d, st["u1"], st["u2"], st["u3"], st["p"], yu, yv,
                b.grid(2), b.grid(3), t=sc["t"], it=sc["iter"], mpgx=sc["mpgx"])
    u1, u2, u3, p, hdr = read_state(str(tmp_path), "_restart.dat", d, np1=False)
    for f, x in zip(FIELDS, (u1, u2, u3, p)):
        assert np.array_equal(x, st[f]), f
    c = Engine(d)
    c.upload(u1, u2, u3, p)
    c.set_scalars(hdr["t"], hdr["iter"], hdr["mpgx"])
    c.step(n)
    c.synchronize()
    got, got_sc = c.download(), c.scalars()
    assert got_sc["iter"] == ref_sc["iter"] == 2 * n
    if ctpress == 1:
        # Nu of the previous substep enters with c_1 = 0 at kRK = 1, so a step
        # boundary carries no state besides the fields and the scalars
        for f in FIELDS:
            assert np.array_equal(got[f], ref[f]), f
        assert got_sc["t"] == ref_sc["t"] and got_sc["dt"] == ref_sc["dt"]
    else:
        # getini sets the target flow rate QxT to the restart state's Qx,
        # which the uninterrupted run only matches to round-off
        for f in FIELDS:
            assert np.linalg.norm(got[f] - ref[f]) <= 1e-12 * np.linalg.norm(ref[f]), f
        assert abs(got_sc["mpgx"] - ref_sc["mpgx"]) <= 1e-9 * abs(ref_sc["mpgx"])
