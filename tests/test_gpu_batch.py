"""Batched engine: instances of uneven size advanced in shared launches give
the same result as each instance alone (same kernels, same arithmetic per
instance), and admission respects the HBM budget."""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _one_column_kernel(monkeypatch):
    """A batch of many columns and a lone small instance would otherwise run
    different column-pass kernels (which agree to round-off, tested in
    test_gpu_parity.py); batching equivalence is checked with the same one."""
    monkeypatch.setenv("LH_SMALL_COLUMNS", "0")


def _ic(desc, seed):
    from lh_b200 import grids, perturbed_laminar
    yu, yv = grids(desc)
    return perturbed_laminar(desc, seed, yu, yv)


def test_batch_equals_single_instances():
    from lh_b200 import Batch, Desc, Engine, re_from_retau
    descs = [
        Desc(Nx=32, Nz=32, ny=153, Re=re_from_retau(180), dt_mode=1, dt=1e-3),
        Desc(Nx=64, Nz=64, ny=97, Re=re_from_retau(300), dt_mode=1, dt=5e-4),
        Desc(Nx=32, Nz=16, ny=65, Re=re_from_retau(120), dt_mode=0, CFL=0.5),
        Desc(Nx=16, Nz=32, ny=41, Re=re_from_retau(250), dt_mode=1, dt=2e-3, grid_type=1),
    ]
    b = Batch()
    slots = []
    ics = []
    for k, d in enumerate(descs):
        ic = _ic(d, 1000 + k)
        ics.append(ic)
        slots.append(b.add(d, *ic))
    assert b.count() == 4
    b.step(3)
    b.synchronize()
    for d, s, ic in zip(descs, slots, ics):
        e = Engine(d)
        e.upload(*ic)
        e.step(3)
        e.synchronize()
        ref = e.download()
        got = b.download(s)
        for f in ("u1", "u2", "u3", "p"):
            assert rel_l2(got[f], ref[f]) <= 1e-14, (d, f, rel_l2(got[f], ref[f]))
        assert b.scalars(s)["iter"] == 3


def test_batch_membership_changes_between_steps():
    from lh_b200 import Batch, Desc, Engine
    d1 = Desc(Nx=16, Nz=16, ny=33, dt_mode=1, dt=1e-3)
    d2 = Desc(Nx=32, Nz=32, ny=65, dt_mode=1, dt=1e-3)
    ic1, ic2 = _ic(d1, 1), _ic(d2, 2)
    b = Batch()
    s1 = b.add(d1, *ic1)
    b.step(2)
    s2 = b.add(d2, *ic2)  # joins while s1 is in flight
    b.step(2)
    b.remove(s1)
    b.step(1)
    b.synchronize()
    e = Engine(d2)
    e.upload(*ic2)
    e.step(3)
    e.synchronize()
    ref = e.download()
    got = b.download(s2)
    for f in ("u1", "u2", "u3", "p"):
        assert rel_l2(got[f], ref[f]) <= 1e-14
    assert b.count() == 1


def test_budget_rejects_admission():
    from lh_b200 import Batch, Desc, LHError
    d = Desc(Nx=32, Nz=32, ny=65, dt_mode=1, dt=1e-3)
    need = Batch.instance_bytes(d)
    b = Batch(hbm_budget=int(need * 1.5))
    b.add(d, *_ic(d, 1))
    with pytest.raises(LHError) as ei:
        b.add(d, *_ic(d, 2))
    assert ei.value.code == -3
    assert b.count() == 1


def test_isolated_plans_equal_the_shared_plan(monkeypatch):
    """Instances of 128^2 modes and more get a launch plan of their own
    (LH_BATCH_ISOLATE sets the threshold); the states do not depend on how
    the instances are grouped into plans."""
    from lh_b200 import Batch, Desc
    descs = [Desc(Nx=32, Nz=32, ny=33, dt_mode=1, dt=1e-3), Desc(Nx=128, Nz=128, ny=33, dt_mode=1, dt=5e-4),
             Desc(Nx=16, Nz=32, ny=41, dt_mode=0, CFL=0.5)]
    out = []
    for iso in ("1", "1000000000"):
        monkeypatch.setenv("LH_BATCH_ISOLATE", iso)
        b = Batch()
        slots = [b.add(d, *_ic(d, 300 + k)) for k, d in enumerate(descs)]
        b.step(3)
        b.synchronize()
        out.append([b.download(s) for s in slots])
        b.close()
    for k in range(len(descs)):
        for f in ("u1", "u2", "u3", "p"):
            assert rel_l2(out[0][k][f], out[1][k][f]) <= 1e-14, (k, f)


def test_batch_of_small_instances_uses_the_per_column_pass(monkeypatch):
    """Plans of few columns run the one-CTA-per-column column pass, batches
    included: two small instances in one batch give each instance's states
    as it gives them alone (the per-column pass does not depend on the other
    columns of the launch)."""
    from lh_b200 import Batch, Desc, Engine
    monkeypatch.setenv("LH_SMALL_COLUMNS", "1000000000")
    descs = [Desc(Nx=16, Nz=16, ny=33, dt_mode=1, dt=1e-3), Desc(Nx=32, Nz=16, ny=65, dt_mode=0, CFL=0.5)]
    ics = [_ic(d, 400 + k) for k, d in enumerate(descs)]
    b = Batch()
    slots = [b.add(d, *ic) for d, ic in zip(descs, ics)]
    b.step(3)
    b.synchronize()
    for d, s, ic in zip(descs, slots, ics):
        e = Engine(d)
        e.upload(*ic)
        e.step(3)
        e.synchronize()
        ref = e.download()
        got = b.download(s)
        for f in ("u1", "u2", "u3", "p"):
            assert rel_l2(got[f], ref[f]) <= 1e-14, (d, f, rel_l2(got[f], ref[f]))


def test_batch_snapshot_restore_continues_bit_for_bit():
    """A live instance's snapshot (download + scalars) re-admitted into another
    batch with its t and iter restored continues exactly as the instance does
    where it was left (ct. pressure gradient: Nu of the previous substep
    enters with c_1 = 0 at kRK = 1, so a step boundary carries no other state)."""
    import numpy as np
    from lh_b200 import Batch, Desc
    d1 = Desc(Nx=32, Nz=32, ny=97, dt_mode=1, dt=1e-3)
    d2 = Desc(Nx=64, Nz=32, ny=65, dt_mode=0, CFL=0.5)
    a = Batch()
    s1 = a.add(d1, *_ic(d1, 21))
    a.add(d2, *_ic(d2, 22))
    a.step(3)
    a.synchronize()
    snap, sc = a.download(s1), a.scalars(s1)
    a.step(3)
    a.synchronize()
    want, want_sc = a.download(s1), a.scalars(s1)
    b = Batch()
    s = b.add(d1, snap["u1"], snap["u2"], snap["u3"], snap["p"])
    b.set_scalars(s, sc["t"], sc["iter"], d1.mpgx)
    b.step(3)
    b.synchronize()
    got, got_sc = b.download(s), b.scalars(s)
    for f in ("u1", "u2", "u3", "p"):
        assert np.array_equal(got[f], want[f]), f
    assert got_sc == want_sc
    a.close()
    b.close()


def test_uneven_batch_with_a_256x257_instance_equals_alone():
    """The largest instance of the uneven configuration (256x256x257, tanh(2)
    grid) in a batch with small ones gets a launch plan of its own and steps
    exactly as it does alone (its single-instance step is checked against the
    oracle in test_gpu_parity.py)."""
    import numpy as np
    from lh_b200 import Batch, Desc, Engine, re_from_retau
    big = Desc(Nx=256, Nz=256, ny=257, grid_type=1, Re=re_from_retau(550), dt_mode=1, dt=2.5e-4)
    small = Desc(Nx=32, Nz=32, ny=153, grid_type=1, Re=re_from_retau(180), dt_mode=1, dt=5e-4)
    ics = [_ic(big, 31), _ic(small, 32), _ic(small, 33)]
    b = Batch()
    slots = [b.add(d, *ic) for d, ic in zip((big, small, small), ics)]
    b.step(1)
    b.synchronize()
    for d, s, ic in zip((big, small, small), slots, ics):
        e = Engine(d)
        e.upload(*ic)
        e.step(1)
        e.synchronize()
        ref = e.download()
        got = b.download(s)
        for f in ("u1", "u2", "u3", "p"):
            assert np.array_equal(got[f], ref[f]), (d.Nx, f)
        e.close()
    b.close()
