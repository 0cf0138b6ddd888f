"""The allocation-free spreading entry point, through the C ABI.

Callers that cannot allocate device memory (graph capture in global mode, hosts owning
all memory through their own arena, latency-bound callers) use rmd_spread_charges_noalloc,
whose scratch grid is a static device array. Its output must equal the engine's own
spreading (rmd_debug_charge_grid) on the same positions, on two calls in a row (the second
call must not see the first call's accumulation), for both spline orders. Sizes beyond the
static array are refused before anything is launched, including sizes whose product
overflows 64 bits. This file is collected last.
"""
import ctypes

import numpy as np
import pytest

from goldens import system_for

ALPHA = 2.6282608939112584


def _call(lib, posq_ptr, n, box, grid, order, out_ptr):
    g = np.ascontiguousarray(grid, dtype=np.int32)
    return lib.rmd_spread_charges_noalloc(
        ctypes.c_void_p(posq_ptr), n, box.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        g.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), order, ctypes.c_void_p(out_ptr), None)


@pytest.mark.parametrize("grid", [[2 ** 21, 2 ** 21, 2 ** 22], [2 ** 30, 2 ** 30, 16], [65, 64, 64],
                                  [2 ** 31 - 1, 1, 1], [4, 4, 2 ** 20]])
def test_noalloc_refuses_oversized_grids_before_launching(grid):
    """Each size is bounded before the product is formed: a product that would overflow (and
    could wrap to a small value) and one just above 64^3 points are both refused. The
    pointers are placeholders the entry point must never reach, so this runs only where no
    GPU is visible: a missed refusal then fails at cudaGetDevice instead of launching."""
    import torch

    from rainmd_b200 import _lib

    if torch.cuda.is_available():
        pytest.skip("host-side refusal test; placeholder pointers are only safe without a GPU")

    lib = _lib.load()
    box = np.diag([2.0, 2.0, 2.0]).reshape(-1).astype(np.float64)
    status = _call(lib, 0x1000, 10, box, grid, 4, 0x2000)
    assert status == _lib.RMD_ERR_INVALID


@pytest.mark.gpu
@pytest.mark.parametrize("order", [4, 5])
def test_noalloc_spread_matches_engine_twice(order):
    import torch

    from rainmd_b200 import _lib
    from rainmd_b200.simulation import GpuSimulation

    s, pos, _ = system_for("ala-wat")
    grid = [24, 24, 24]
    sim = GpuSimulation(s, {"alpha": ALPHA, "grid": grid, "skin": 0.1, "dispersionCorrection": False,
                            "pmeOrder": order})
    sim.setState(pos)
    sim.initialise()
    expect = sim.debugChargeGrid(points=int(np.prod(grid)))

    n = s["topology"]["atomCount"]
    posq = np.zeros((n, 4), dtype=np.float32)
    posq[:, :3] = pos.reshape(-1, 3).astype(np.float32)
    posq[:, 3] = s["topology"]["charges"].astype(np.float32)
    d_posq = torch.from_numpy(posq).cuda()
    d_out = torch.zeros(int(np.prod(grid)), dtype=torch.float64, device="cuda")
    box = np.ascontiguousarray(s["boxVectors"], dtype=np.float64)
    lib = _lib.load()
    for call in range(2):
        d_out.fill_(float("nan"))
        status = _call(lib, d_posq.data_ptr(), n, box, grid, order, d_out.data_ptr())
        assert status == 0, call
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - expect)) <= 1e-12, call

    # sizes beyond the static scratch are refused, and nothing is written
    d_out.fill_(-7.0)
    status = _call(lib, d_posq.data_ptr(), n, box, [128, 128, 128], order, d_out.data_ptr())
    assert status == _lib.RMD_ERR_INVALID
    torch.cuda.synchronize()
    assert bool(torch.all(d_out == -7.0))
    sim.release()
