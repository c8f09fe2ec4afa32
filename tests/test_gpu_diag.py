"""On-device diagnostics of flagged steps through the C ABI: the spectra
(spectra.f90:7-66) and the plane stats (stats.f90:1-97).

The engine's accumulators, added to between steps as the reference's
nonlinear() does at its flagged steps, equal the oracle's restatement applied
to the same (downloaded) states bit for bit: both round every product and sum
separately in the reference's order."""
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


@pytest.mark.parametrize("N,ny", [(16, 33), (32, 65), (64, 97)])
def test_stats_match_oracle_on_the_same_states(N, ny):
    from lh_b200 import Desc, Engine, grids, perturbed_laminar
    d = Desc(Nx=N, Nz=N, ny=ny, dt_mode=1, dt=5e-4)
    yu, yv = grids(d)
    e = Engine(d)
    e.upload(*perturbed_laminar(d, 12, yu, yv))
    o = O.Oracle(O.Config(Nx=N, Nz=N, ny=ny, dt_mode=O.DT_FIXED, dt_fixed=5e-4))
    acc = None
    for k in range(2):
        e.step(2)
        e.stats_accumulate()
        st = e.download()
        o.load_state(st["u1"], st["u2"], st["u3"], st["p"])
        acc = o.stats(acc)
    got, count = e.stats()
    assert count == 2 and got.shape == acc.shape
    for q, name in enumerate(Engine.STATS):
        assert np.array_equal(got[q], acc[q]), (name, float(np.max(abs(got[q] - acc[q]))))
    e.stats_reset()
    got, count = e.stats()
    assert count == 0 and not np.any(got)
