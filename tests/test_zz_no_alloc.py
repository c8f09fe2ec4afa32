"""The allocation-free LUsolU entry point, lh_lusolu_noalloc.

It exists for callers that cannot allocate device memory per call (a loop
captured into a CUDA graph, a serving loop that must not pay the device
synchronisation of cudaMalloc/cudaFree, a host program whose device memory
belongs to another allocator).  The test drives it through the C ABI with
device arrays it owns and checks it against the allocating entry point
lh_lusolu on the same right-hand sides, on two calls in a row (the shared
scratch keeps the previous call's contents).  This file is collected last.
"""
import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu


def _device(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


@pytest.mark.parametrize("grid,kRK", [(2, 1), (1, 3)])
def test_noalloc_matches_allocating_lusolu_twice(grid, kRK):
    import torch
    from lh_b200 import Desc, Engine, capi
    d = Desc(Nx=16, Nz=16, ny=65, dt_mode=1, dt=2e-3)
    e = Engine(d)
    L = capi.lib()
    n = (d.nyu + 2) if grid == 2 else (d.nyv + 2)
    rng = np.random.default_rng(100 + grid)
    for call in range(2):
        rhs = rng.standard_normal((d.ncols, n)) + 1j * rng.standard_normal((d.ncols, n))
        ref = e.lusolu(grid, kRK, d.dt, rhs)  # allocating entry, column layout
        rhs_dev = _device(rhs.T)              # engine layout: row j, then column
        u_dev = torch.empty_like(rhs_dev)
        torch.cuda.synchronize()
        rc = L.lh_lusolu_noalloc(e.h, grid, kRK, d.dt, rhs_dev.data_ptr(), u_dev.data_ptr())
        assert rc == 0, L.lh_last_error(e.h).decode()
        e.synchronize()
        got = u_dev.cpu().numpy().T
        assert rel_l2(got, ref) <= 1e-13, (call, rel_l2(got, ref))


def test_noalloc_in_place_and_size_limit():
    import torch
    from lh_b200 import Desc, Engine, capi
    d = Desc(Nx=16, Nz=16, ny=65, dt_mode=1, dt=1e-3)
    e = Engine(d)
    L = capi.lib()
    rng = np.random.default_rng(7)
    n = d.nyu + 2
    rhs = rng.standard_normal((d.ncols, n)) + 1j * rng.standard_normal((d.ncols, n))
    ref = e.lusolu(2, 2, d.dt, rhs)
    x = _device(rhs.T)
    torch.cuda.synchronize()
    assert L.lh_lusolu_noalloc(e.h, 2, 2, d.dt, x.data_ptr(), x.data_ptr()) == 0
    e.synchronize()
    assert rel_l2(x.cpu().numpy().T, ref) <= 1e-13
    # 258 rows x 8256 columns exceed the 2^21-entry scratch: rejected, no launch
    big = Engine(Desc(Nx=256, Nz=64, ny=257, dt_mode=1, dt=1e-3))
    rc = L.lh_lusolu_noalloc(big.h, 2, 1, 1e-3, x.data_ptr(), x.data_ptr())
    assert rc == -1
    assert "exceed" in L.lh_last_error(big.h).decode()
