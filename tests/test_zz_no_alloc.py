"""The allocation-free spreading entry point, through the C ABI.

Callers that cannot allocate device memory (graph capture in global mode, hosts owning
all memory through their own arena, latency-bound callers) use rmd_spread_charges_noalloc,
whose scratch grid is a static device array. Its output must equal the engine's own
spreading (rmd_debug_charge_grid) on the same positions, on two calls in a row (the second
call must not see the first call's accumulation). This file is collected last.
"""
import ctypes

import numpy as np
import pytest

from goldens import system_for

pytestmark = pytest.mark.gpu

ALPHA = 2.6282608939112584


def test_noalloc_spread_matches_engine_twice():
    import torch

    from rainmd_b200 import _lib
    from rainmd_b200.simulation import GpuSimulation

    s, pos, _ = system_for("ala-wat")
    grid = [24, 24, 24]
    sim = GpuSimulation(s, {"alpha": ALPHA, "grid": grid, "skin": 0.1, "dispersionCorrection": False})
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
    g = np.ascontiguousarray(grid, dtype=np.int32)
    lib = _lib.load()
    for call in range(2):
        d_out.fill_(float("nan"))
        status = lib.rmd_spread_charges_noalloc(
            ctypes.c_void_p(d_posq.data_ptr()), n, box.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            g.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), 5, ctypes.c_void_p(d_out.data_ptr()), None)
        assert status == 0, call
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert np.max(np.abs(got - expect)) <= 1e-12, call

    # sizes beyond the static scratch are refused, and nothing is written
    big = np.ascontiguousarray([128, 128, 128], dtype=np.int32)
    status = lib.rmd_spread_charges_noalloc(
        ctypes.c_void_p(d_posq.data_ptr()), n, box.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        big.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), 5, ctypes.c_void_p(d_out.data_ptr()), None)
    assert status == _lib.RMD_ERR_INVALID
    sim.release()
