"""On-device diagnostics of flagged steps through the C ABI: the spectra
(spectra.f90:7-66), the plane stats (stats.f90:1-97) and omega_x
(FOU3D.f90:314-338).

The engine's accumulators, added to between steps as the reference's
nonlinear() does at its flagged steps, are compared with the oracle's
restatement applied to the same (downloaded) states.  Sums over spectral
coefficients (the spectra; the stats of the wall planes and of the pressure
snapshot) match bit for bit: both round every product and sum separately in
the reference's order.  Sums over physical values (the stats of planes
1..nyu and of omega_x) go through the device's FFTs and a tree reduction,
so they agree to 1e-12 of the row's magnitude."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,ny", [(32, 65), (128, 153)])
def test_spectra_match_oracle_on_the_same_states(N, ny):
    from lh_b200 import Desc, Engine, grids, perturbed_laminar
    d = Desc(Nx=N, Nz=N, ny=ny, dt_mode=1, dt=5e-4)
    yu, yv = grids(d)
    e = Engine(d)
    e.upload(*perturbed_laminar(d, 11, yu, yv))
    o = O.Oracle(O.Config(Nx=N, Nz=N, ny=ny, dt_mode=O.DT_FIXED, dt_fixed=5e-4))
    acc = None
    for k in range(3):
        e.step(1)
        e.spectra_accumulate()
        st = e.download()
        o.load_state(st["u1"], st["u2"], st["u3"], st["p"])
        acc = o.spectra(acc)
    got, count = e.spectra()
    assert count == 3
    for name in Engine.SPECTRA:
        assert got[name].shape == acc[name].shape, name
        assert np.array_equal(got[name], acc[name]), (name, float(np.max(abs(got[name] - acc[name]))))
    e.spectra_reset()
    got, count = e.spectra()
    assert count == 0 and all(not np.any(a) for a in got.values())


@pytest.mark.parametrize("N,ny", [(16, 33), (32, 65), (64, 97), (256, 65)])
def test_stats_match_oracle_on_the_same_states(N, ny):
    from lh_b200 import Desc, Engine, grids, perturbed_laminar
    d = Desc(Nx=N, Nz=N, ny=ny, dt_mode=1, dt=5e-4)
    yu, yv = grids(d)
    e = Engine(d)
    e.upload(*perturbed_laminar(d, 12, yu, yv))
    o = O.Oracle(O.Config(Nx=N, Nz=N, ny=ny, dt_mode=O.DT_FIXED, dt_fixed=5e-4))
    acc = None
    for k in range(3):
        e.step(2)
        st = e.download()
        o.load_state(st["u1"], st["u2"], st["u3"], st["p"])
        if k != 1:   # output steps refresh the pressure planes; k = 1 reads the older ones
            e.pressure_snapshot()
            o.pressure_snapshot()
        e.stats_accumulate()
        acc = o.stats(acc)
    got, count = e.stats()
    assert count == 3 and got.shape == acc.shape == (13, d.nyu + 2)
    assert Engine.STATS == O.Oracle.STATS
    q = {name: k for k, name in enumerate(Engine.STATS)}
    # spectral sums: the wall planes of the velocity rows, the pressure rows
    for name in Engine.STATS[:9]:
        for j in (0, d.nyu + 1):
            assert got[q[name], j] == acc[q[name], j], (name, j)
    for name in ("Pm", "P2m"):
        assert np.array_equal(got[q[name]], acc[q[name]]), name
    # physical sums: interior planes and omega_x, against the row's scale
    n = 3 * o.Mx * o.Mz
    scale = {"U2m": acc[q["U2m"]], "V2m": acc[q["V2m"]], "W2m": acc[q["W2m"]],
             "wx2m": acc[q["wx2m"]]}
    scale.update(Um=np.sqrt(n * scale["U2m"]), Vm=np.sqrt(n * scale["V2m"]), Wm=np.sqrt(n * scale["W2m"]),
                 wxm=np.sqrt(3 * N * N * scale["wx2m"]), UVm=np.sqrt(scale["U2m"] * scale["V2m"]),
                 UWm=np.sqrt(scale["U2m"] * scale["W2m"]), VWm=np.sqrt(scale["V2m"] * scale["W2m"]))
    for name, sc in scale.items():
        rows = slice(1, d.nyu + 1) if not name.startswith("wx") else slice(None)
        err = np.max(abs(got[q[name], rows] - acc[q[name], rows]))
        assert err <= 1e-12 * np.max(sc), (name, err, np.max(sc))
    e.stats_reset()
    got, count = e.stats()
    assert count == 0 and not np.any(got)


@pytest.mark.parametrize("N,ny", [(16, 33), (64, 97)])
def test_omega_x_matches_oracle(N, ny):
    from lh_b200 import Desc, Engine, grids, perturbed_laminar
    d = Desc(Nx=N, Nz=N, ny=ny, dt_mode=1, dt=5e-4)
    yu, yv = grids(d)
    e = Engine(d)
    e.upload(*perturbed_laminar(d, 13, yu, yv))
    e.step(2)
    got = e.omega_x()
    st = e.download()
    o = O.Oracle(O.Config(Nx=N, Nz=N, ny=ny, dt_mode=O.DT_FIXED, dt_fixed=5e-4))
    o.load_state(st["u1"], st["u2"], st["u3"], st["p"])
    ref = o.omega_x()
    assert got.shape == ref.shape
    assert np.max(abs(got[:, :, :N] - ref[:, :, :N])) <= 1e-13 * np.max(abs(ref[:, :, :N]))
    assert not np.any(got[d.nyu + 1])
