"""Serving with continuous batching on the GPU: requests of different sizes
that arrive while others run are admitted under an HBM budget, and every
request's final state equals the same request run alone through the
single-instance engine (same kernels, same arithmetic per instance)."""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _one_column_kernel(monkeypatch):
    """A mixed batch and a lone small request would otherwise run different
    column-pass kernels (which agree to round-off, tested in
    test_gpu_parity.py); the serving equivalence is checked with the same one."""
    monkeypatch.setenv("LH_SMALL_COLUMNS", "0")


def test_each_result_same_alone_and_in_the_mix():
    from lh_b200 import Batch, Desc
    from lh_b200.serve import Request, run_plain, serve
    descs = [Desc(Nx=16, Nz=16, ny=33, dt_mode=1, dt=1e-3), Desc(Nx=32, Nz=32, ny=65, dt_mode=1, dt=1e-3),
             Desc(Nx=32, Nz=16, ny=41, dt_mode=0, CFL=0.5), Desc(Nx=64, Nz=64, ny=97, dt_mode=1, dt=5e-4)]
    rng = np.random.default_rng(11)
    reqs = []
    t = 0.0
    for k in range(10):
        t += rng.exponential(0.02)
        reqs.append(Request(k, descs[k % 4], 500 + k, int(rng.integers(3, 15)), t))
    # budget for about three of the largest instances at once
    budget = 3 * Batch.instance_bytes(descs[3])
    st = serve(reqs, hbm_budget=budget, max_chunk=4)
    assert st.requests == 10 and st.max_live >= 2
    mixed = {r.rid: r.result for r in reqs}
    alone = [Request(r.rid, r.desc, r.seed, r.nsteps) for r in reqs]
    run_plain(alone)
    for r in alone:
        for f in ("u1", "u2", "u3", "p"):
            assert rel_l2(mixed[r.rid][f], r.result[f]) <= 1e-14, (r.rid, f)
    assert st.p99 >= st.p50 > 0
