"""The launch-shape autotuner (lh_autotune): it measures a size on first use,
writes the cache file keyed by GPU name and sizes, reads it back instead of
measuring again, and the tuned plan -- single instance and batch -- steps to
bit-identical states."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("u1", "u2", "u3", "p")


def test_autotune_measures_caches_and_keeps_states(tmp_path, monkeypatch):
    from lh_b200 import Batch, Desc, Engine, grids, perturbed_laminar
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("LH_TUNE_CACHE", str(cache))
    d = Desc(Nx=64, Nz=64, ny=97, dt_mode=1, dt=1e-3)
    ic = perturbed_laminar(d, 11, *grids(d))
    ref = Engine(d)  # default plan (built before any tuning in this process)
    ref.upload(*ic)
    ref.step(3)
    ref.synchronize()
    want = ref.download()

    e = Engine(d)
    e.upload(*ic)
    p = e.autotune()
    assert p["source"] == "measured", p
    lines = cache.read_text().splitlines()
    assert len(lines) == 1 and "|96|96|96 " in lines[0], lines
    assert all(p[k] > 0 for k in ("cbz", "rbx", "cbf", "staging_mb", "col_waves")), p
    e.step(3)
    e.synchronize()
    got = e.download()
    for f in FIELDS:
        assert np.array_equal(got[f], want[f]), f

    # a second context of the size reads the cache
    e2 = Engine(d)
    q = e2.autotune()
    assert q["source"] == "cache" and {k: q[k] for k in p if k != "source"} == {k: p[k] for k in p if k != "source"}
    assert len(cache.read_text().splitlines()) == 1

    # a batch plan of the tuned size uses the table too; still the same states
    b = Batch()
    b.add(d, *ic)
    b.step(3)
    b.synchronize()
    got_b = b.download(0)
    for f in FIELDS:
        assert np.array_equal(got_b[f], want[f]), f
    b.close()
