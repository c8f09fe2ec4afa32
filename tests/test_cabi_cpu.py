"""C-ABI checks that need no GPU: the library loads, exports every function
include/lh_gpu.h declares, and its host set-up (the start() restatement)
reproduces the reference grid and the oracle's operators."""
import os
import re

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "lh_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lh_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from lh_b200 import capi
    L = capi.lib()
    declared = _declared()
    assert declared, "no declarations parsed"
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(capi.EXPORTS) == declared


def test_host_setup_matches_reference_grid(golden_dir):
    from lh_b200 import Desc, host_grid
    g = np.load(os.path.join(golden_dir, "grid_ny153_dyq10_p5.npz"))
    d = Desc()
    assert np.array_equal(host_grid(d, 0), g["yu"])
    assert np.array_equal(host_grid(d, 1), g["yv"])
    assert np.array_equal(host_grid(d, 2), g["dthdyu"])
    assert np.array_equal(host_grid(d, 3), g["dthdyv"])


@pytest.mark.parametrize("grid_type", [O.GRID_POLY, O.GRID_TANH])
def test_host_setup_matches_oracle(grid_type):
    from lh_b200 import Desc, host_grid
    d = Desc(Nx=16, Nz=8, ny=41, grid_type=grid_type)
    o = O.Oracle(O.Config(Nx=16, Nz=8, ny=41, grid_type=grid_type))
    for w in range(4):
        assert np.array_equal(host_grid(d, w), o.array(w))
    sc = o.array(6)
    hs = host_grid(d, 4)
    # gw1, gw2, gw_bc, gwi1, gwi2, dtv
    assert np.array_equal(hs, [sc[0], sc[1], sc[2], sc[4], sc[5], sc[6]])


def test_rejects_unsupported_sizes():
    from lh_b200 import Desc, LHError, host_grid
    with pytest.raises(LHError):
        host_grid(Desc(Nx=40, Nz=32), 0)   # Ngal_x = 60 has a factor 5
    with pytest.raises(LHError):
        host_grid(Desc(Nx=31, Nz=32), 0)   # odd
    with pytest.raises(LHError):
        host_grid(Desc(ny=3), 0)


def test_ic_generator_is_deterministic_and_hermitian():
    from lh_b200 import Desc, grids, perturbed_laminar
    d = Desc(Nx=16, Nz=16, ny=33)
    yu, yv = grids(d)
    a = perturbed_laminar(d, 7, yu, yv)
    b = perturbed_laminar(d, 7, yu, yv)
    c = perturbed_laminar(d, 8, yu, yv)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert not np.array_equal(a[0], c[0])
    nxh = d.Nx // 2 + 1
    u1 = a[0]
    for r in range(1, d.Nz // 2):
        assert np.array_equal(u1[(d.Nz - r) * nxh], np.conj(u1[r * nxh]))
    assert np.all(a[1][:, 0] == 0) and np.all(a[1][:, -1] == 0)
    # read_in at np=1 leaves the top ghost of u1/u3 unread (zero)
    assert np.all(u1[:, -1] == 0)


def test_state_file_round_trip(tmp_path):
    from lh_b200 import Desc, grids, host_grid, perturbed_laminar, read_state, write_state
    d = Desc(Nx=8, Nz=8, ny=17)
    yu, yv = grids(d)
    u1, u2, u3, p = perturbed_laminar(d, 3, yu, yv, np1_read_in=False)
    p = p + 0.25
    write_state(str(tmp_path), "_t.dat", d, u1, u2, u3, p, yu, yv, host_grid(d, 2), host_grid(d, 3), t=1.5, it=7)
    r1, r2, r3, rp, hdr = read_state(str(tmp_path), "_t.dat", d, np1=False)
    assert np.array_equal(r1, u1) and np.array_equal(r2, u2) and np.array_equal(r3, u3) and np.array_equal(rp, p)
    assert hdr["t"] == 1.5 and hdr["iter"] == 7
    # the oracle's independent reader agrees, including the np=1 ghost rule
    o1, o2, o3, op, _ = O.read_in_np1(str(tmp_path), "_t.dat", 8, 8, d.nyu, d.nyv)
    s1, _, s3, _, _ = read_state(str(tmp_path), "_t.dat", d, np1=True)
    assert np.array_equal(o1, s1) and np.array_equal(o3, s3) and np.array_equal(o2, r2) and np.array_equal(op, p)
