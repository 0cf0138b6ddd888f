"""`GpuSimulation`: the Python mirror of RainMD's `class GpuSimulation`
(webgpu/simulation.js:82-1341) over the C ABI in include/rmd.h.

Same constructor inputs (a `system` from `build_system`, RainMD's option names), same
methods (setState, setNoise, initialise, run, minimise, attemptVolumeChange, scaleVolume,
energy, readPositions, readState, diagnostics, release) and the same error classes, so a
test written against the reference's interface reads the same here. `BatchSimulation`
advances many independent systems of uneven size in one set of launches.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class RainMDError(RuntimeError):
    pass


class NeighbourOverflowError(RainMDError):
    """webgpu/kernels/neighbours.js:172-183"""


class NonFiniteStateError(RainMDError):
    """shared/finite.js:63-95"""


class SimulationStopped(RainMDError):
    """webgpu/runtime/yield.js:44-50"""


class GpuBudgetError(RainMDError):
    """webgpu/runtime/allocator.js:141-154"""


_ERRORS = {
    L.RMD_ERR_INVALID: ValueError,
    L.RMD_ERR_NEIGHBOUR_OVERFLOW: NeighbourOverflowError,
    L.RMD_ERR_NON_FINITE: NonFiniteStateError,
    L.RMD_ERR_BUDGET: GpuBudgetError,
    L.RMD_ERR_STOPPED: SimulationStopped,
    L.RMD_ERR_CUDA: RainMDError,
    L.RMD_ERR_CONSTRAINTS: RainMDError,
}

_OPTION_NAMES = {
    "timestep": "timestep", "temperature": "temperature", "friction": "friction", "seed": "seed",
    "tolerance": "tolerance", "maxConstraintIterations": "max_constraint_iterations",
    "rebuildInterval": "rebuild_interval", "adaptiveRebuild": "adaptive_rebuild",
    "barostatInterval": "barostat_interval", "dispersionCorrection": "dispersion_correction",
    "restraintForce": "restraint_force", "skin": "skin", "neighbourSlack": "neighbour_slack",
    "maxNeighbours": "max_neighbours", "ewaldTolerance": "ewald_tolerance", "alpha": "alpha",
    "pmeOrder": "pme_order", "waterSolver": "water_solver", "learnedBarostat": "learned_barostat",
    "forceAccumulation": "force_accumulation", "neighbourGroupAtoms": "neighbour_group_atoms",
    "nonbondedLanes": "nonbonded_lanes", "spreadAtomsPerBlock": "spread_atoms_per_block",
    "learnedWarmupMoves": "learned_warmup_moves", "learnedStepsPerMove": "learned_steps_per_move",
    "learnedRate": "learned_rate", "rebuildOnDemand": "rebuild_on_demand", "pairList": "pair_list",
}


def _arr(values, dtype, keep):
    a = np.ascontiguousarray(values if values is not None and len(values) else np.zeros(1), dtype=dtype)
    keep.append(a)
    return a


def pack_system(system: dict, keep: list) -> L.RmdSystem:
    """Flatten a build_system() dictionary into the rmd_system struct."""
    t = system["topology"]
    ip = lambda v: _arr(v, np.int32, keep).ctypes.data_as(C.POINTER(C.c_int32))  # noqa: E731
    dp = lambda v: _arr(v, np.float64, keep).ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    hb, an, di = system["harmonicBonds"], t["angles"], t["dihedrals"]
    ex, co = system["exceptions"], system["constraints"]
    s = L.RmdSystem()
    s.atom_count = t["atomCount"]
    s.charges, s.masses = dp(t["charges"]), dp(t["masses"])
    s.atom_types, s.type_count = ip(t["atomTypes"]), t["typeCount"]
    s.lj_a, s.lj_b = dp(t["ljA"]), dp(t["ljB"])
    s.exclusion_start = ip(t["exclusions"]["start"])
    s.exclusion_partners = ip(t["exclusions"]["partners"])
    s.bond_count = hb["count"]
    s.bond_atoms = ip(np.stack([hb["atomA"], hb["atomB"]], 1).reshape(-1) if hb["count"] else [])
    s.bond_k, s.bond_r0 = dp(hb["k"]), dp(hb["r0"])
    s.angle_count = an["count"]
    s.angle_atoms = ip(np.stack([an["atomA"], an["atomB"], an["atomC"]], 1).reshape(-1) if an["count"] else [])
    s.angle_k, s.angle_theta0 = dp(an["k"]), dp(an["theta0"])
    s.torsion_count = di["count"]
    s.torsion_atoms = ip(np.stack([di["atomA"], di["atomB"], di["atomC"], di["atomD"]], 1).reshape(-1)
                         if di["count"] else [])
    s.torsion_k, s.torsion_periodicity, s.torsion_phase = dp(di["k"]), dp(di["periodicity"]), dp(di["phase"])
    s.constraint_count = co["count"]
    s.constraint_atoms = ip(np.stack([co["atomA"], co["atomB"]], 1).reshape(-1) if co["count"] else [])
    s.constraint_distance = dp(co["distance"])
    s.exception_count = ex["count"]
    s.exception_atoms = ip(np.stack([ex["atomA"], ex["atomB"]], 1).reshape(-1) if ex["count"] else [])
    s.exception_charge_product, s.exception_lj_a, s.exception_lj_b = (
        dp(ex["chargeProduct"]), dp(ex["ljA"]), dp(ex["ljB"]))
    s.molecule_count = system["molecules"]["count"]
    s.molecule_of_atom = ip(t["moleculeOfAtom"])
    s.box_vectors = dp(system["boxVectors"]) if system["boxVectors"] is not None else None
    s.degrees_of_freedom = system["degreesOfFreedom"]
    s.cutoff = system["options"]["cutoff"]
    return s


def pack_options(options: dict, keep: list) -> L.RmdOptions:
    lib = L.load()
    o = L.RmdOptions()
    lib.rmd_default_options(C.byref(o))
    for key, value in (options or {}).items():
        if value is None:
            continue
        if key in _OPTION_NAMES:
            field = _OPTION_NAMES[key]
            current = getattr(o, field)
            setattr(o, field, type(current)(value) if not isinstance(current, float) else float(value))
        elif key == "pressure":
            o.pressure = float(value)
        elif key == "grid":
            o.grid[0], o.grid[1], o.grid[2] = (int(v) for v in value)
        elif key in ("restraintAtoms", "restraintReference"):
            continue
        else:
            raise ValueError(f"unknown option {key!r}")
    atoms = options.get("restraintAtoms") if options else None
    if atoms is not None and len(atoms) and (options.get("restraintForce") or 0) > 0:
        o.restraint_count = len(atoms)
        o.restraint_atoms = _arr(atoms, np.int32, keep).ctypes.data_as(C.POINTER(C.c_int32))
        o.restraint_reference = _arr(options["restraintReference"], np.float64, keep).ctypes.data_as(
            C.POINTER(C.c_double))
    return o


def _struct_dict(obj) -> dict:
    out = {}
    for name, _ in obj._fields_:
        value = getattr(obj, name)
        if isinstance(value, C.Array):
            value = list(value)
        out[name] = value
    return out


SURROGATE_PARAMS = 4801  # W1[64][8], b1[64], W2[64][64], b2[64], W3[64], b3


def surrogate_evaluate(params, inputs, targets=None, gradients=False):
    """The learned barostat's device forward pass (and MSE gradient) on given data:
    (outputs, gradients or None, loss or None). At most 64 samples of 8 inputs."""
    lib = L.load()
    p = np.ascontiguousarray(params, np.float32)
    x = np.ascontiguousarray(inputs, np.float32).reshape(-1, 8)
    count = x.shape[0]
    t = None if targets is None else np.ascontiguousarray(targets, np.float32)
    out = np.zeros(count, np.float32)
    grads = np.zeros(SURROGATE_PARAMS, np.float32) if gradients else None
    loss = C.c_double(0)
    fp = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    status = lib.rmd_surrogate_evaluate(fp(p), fp(x), fp(t), count, fp(out), fp(grads), C.byref(loss))
    if status != L.RMD_OK:
        raise _ERRORS.get(status, RainMDError)(lib.rmd_last_error(None).decode())
    return out, grads, (loss.value if gradients else None)


def planSystem(system: dict, options: dict | None = None) -> dict:
    """The cell plan, skin and PME parameters the engine uses for `system`, computed on the host
    (no GPU needed): skinFor, planCellList (shared/topology/cells.js:67-171) and pmeParameters
    (shared/pme/parameters.js:227-252), the fields GpuSimulation exposes as plan.counts,
    pme.grid and pme.alpha."""
    lib = L.load()
    keep: list = []
    out = L.RmdPlan()
    status = lib.rmd_plan_system(C.byref(pack_system(system, keep)), C.byref(pack_options(options or {}, keep)),
                                 C.byref(out))
    if status != L.RMD_OK:
        raise _ERRORS.get(status, RainMDError)(lib.rmd_last_error(None).decode())
    return _struct_dict(out)


def grownCapacity(capacity: int, required: int) -> int:
    """grownPlan (cells.js:282-288) as the engine applies it to its neighbour rows."""
    return int(L.load().rmd_grown_capacity(int(capacity), int(required)))


def deviceDraws(seed: int, atom0: int, count: int, step: int):
    """The thermostat's counter-based draws computed on the device: (uniforms [count, 4],
    normals [count, 3]) for atoms atom0 .. atom0 + count - 1 at `step`."""
    lib = L.load()
    u = np.zeros((count, 4), np.float32)
    g = np.zeros((count, 3), np.float32)
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    status = lib.rmd_debug_draws(seed & 0xffffffff, atom0, count, step & 0xffffffff, fp(u), fp(g))
    if status != L.RMD_OK:
        raise _ERRORS.get(status, RainMDError)(lib.rmd_last_error(None).decode())
    return u, g


class BatchSimulation:
    """Many independent systems advanced together; every call takes a system index."""

    def __init__(self, systems: list, options):
        self._lib = L.load()
        self._keep: list = []
        opts = options if isinstance(options, (list, tuple)) else [options] * len(systems)
        self.systems = systems
        self.atom_counts = [s["topology"]["atomCount"] for s in systems]
        structs = (L.RmdSystem * len(systems))(*[pack_system(s, self._keep) for s in systems])
        ostructs = (L.RmdOptions * len(systems))(*[pack_options(o, self._keep) for o in opts])
        handle = C.c_void_p()
        status = self._lib.rmd_create_batch(len(systems), structs, ostructs, C.byref(handle))
        if status != L.RMD_OK:
            raise _ERRORS.get(status, RainMDError)(self._lib.rmd_last_error(None).decode())
        self._h = handle
        self.step = 0
        self.timestep = float(ostructs[0].timestep)  # ps, for the restart's time

    # -- plumbing --
    def _check(self, status):
        if status != L.RMD_OK:
            message = self._lib.rmd_last_error(self._h).decode()
            raise _ERRORS.get(status, RainMDError)(message)

    @property
    def count(self) -> int:
        return self._lib.rmd_system_count(self._h)

    def setState(self, index, positions, velocities=None, step=0, suppliedNoise=False):
        pos = np.ascontiguousarray(positions, dtype=np.float64)
        vel = None if velocities is None else np.ascontiguousarray(velocities, dtype=np.float64)
        self._check(self._lib.rmd_set_state_at(
            self._h, index, pos.ctypes.data_as(C.POINTER(C.c_double)),
            None if vel is None else vel.ctypes.data_as(C.POINTER(C.c_double)), int(step),
            1 if suppliedNoise else 0))
        self.step = int(step)

    def setNoise(self, index, noise):
        n = np.ascontiguousarray(noise, dtype=np.float32)
        self._check(self._lib.rmd_set_noise_at(self._h, index, n.ctypes.data_as(C.POINTER(C.c_float))))

    def initialise(self):
        self._check(self._lib.rmd_initialise(self._h))

    def run(self, count, blockSize=None, stopSignal=None):
        step = C.c_int64(0)
        flag = None
        if stopSignal is not None:
            flag = stopSignal if isinstance(stopSignal, C.c_int32) else C.c_int32(int(bool(stopSignal)))
        self._check(self._lib.rmd_run(self._h, int(count), int(blockSize or 0),
                                      None if flag is None else C.pointer(flag), C.byref(step)))
        self.step = step.value
        return self.step

    def energy(self, index=0) -> dict:
        out = L.RmdEnergyReport()
        self._check(self._lib.rmd_energy_at(self._h, index, C.byref(out)))
        e = _struct_dict(out)
        return {
            "step": e["step"], "time": e["time"], "bonded": e["bonded"],
            "harmonicBond": e["harmonic_bond"], "harmonicAngle": e["harmonic_angle"],
            "periodicTorsion": e["periodic_torsion"], "lennardJones": e["lennard_jones"],
            "dispersion": e["dispersion"], "coulombDirect": e["coulomb_direct"],
            "coulombReciprocal": e["coulomb_reciprocal"], "coulombSelf": e["coulomb_self"],
            "coulomb": e["coulomb"], "potential": e["potential"], "kinetic": e["kinetic"],
            "total": e["total"], "positionRestraint": e["position_restraint"],
            "restrainedAtoms": e["restrained_atoms"], "temperature": e["temperature"],
            "kineticForTemperature": e["kinetic_for_temperature"],
            "kineticSampledAt": ("before the closing half kick"
                                 if e["kinetic_sampled_before_closing_kick"] else "after the step"),
            "volume": e["volume"], "boxVectors": np.array(e["box_vectors"]),
            "volumeDerivative": e["volume_derivative"],
        }

    def readState(self, index=0) -> dict:
        n = self.atom_counts[index]
        pos = np.zeros(3 * n, np.float32)
        vel = np.zeros(3 * n, np.float32)
        frc = np.zeros(3 * n, np.float32)
        box = np.zeros(9)
        vol = C.c_double(0)
        f = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
        self._check(self._lib.rmd_read_state_at(self._h, index, f(pos), f(vel), f(frc),
                                                box.ctypes.data_as(C.POINTER(C.c_double)), C.byref(vol)))
        return {"positions": pos, "velocities": vel, "forces": frc, "boxVectors": box, "volume": vol.value}

    def readPositions(self, index=0):
        return self.readState(index)["positions"]

    def diagnostics(self, index=0) -> dict:
        out = L.RmdDiagnostics()
        self._check(self._lib.rmd_diagnostics_at(self._h, index, C.byref(out)))
        return _struct_dict(out)

    def attemptVolumeChange(self):
        out = L.RmdVolumeMove()
        self._check(self._lib.rmd_attempt_volume_change(self._h, C.byref(out)))
        return _struct_dict(out) if out.attempted else None

    def lastVolumeMove(self, index=0):
        out = L.RmdVolumeMove()
        self._check(self._lib.rmd_last_volume_move_at(self._h, index, C.byref(out)))
        return _struct_dict(out) if out.attempted else None

    def minimise(self, maxIterations=200, forceTolerance=500.0, maxStep=0.002, maxDisplacement=0.05):
        out = L.RmdMinimiseResult()
        self._check(self._lib.rmd_minimise(self._h, int(maxIterations), float(forceTolerance),
                                           float(maxStep), float(maxDisplacement), C.byref(out)))
        return _struct_dict(out)

    # -- inspection used by the parity tests --
    def debugCells(self, index=0):
        counts = (C.c_int32 * 3)()
        self._check(self._lib.rmd_debug_cells(self._h, index, counts, None, None))
        cells = counts[0] * counts[1] * counts[2]
        start = np.zeros(cells + 1, np.int32)
        atoms = np.zeros(self.atom_counts[index], np.int32)
        self._check(self._lib.rmd_debug_cells(self._h, index, counts,
                                              start.ctypes.data_as(C.POINTER(C.c_int32)),
                                              atoms.ctypes.data_as(C.POINTER(C.c_int32))))
        return list(counts), start, atoms

    def debugNeighbours(self, index=0):
        cap = C.c_int32(0)
        self._check(self._lib.rmd_debug_neighbours(self._h, index, C.byref(cap), None, None, None))
        n = self.atom_counts[index]
        counts = np.zeros(n, np.int32)
        rows = np.zeros(n * cap.value, np.int32)
        req = C.c_int32(0)
        p = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))  # noqa: E731
        self._check(self._lib.rmd_debug_neighbours(self._h, index, C.byref(cap), p(counts), p(rows),
                                                   C.byref(req)))
        return cap.value, counts, rows.reshape(n, cap.value), req.value

    def debugGroupRows(self, index=0) -> dict:
        """The group-pair rows: atoms [groups, 4] (-1 = none), counts [groups], and per entry
        [groups, capacity] partner, image code and skip mask, in the system's atom indices."""
        groups, cap = C.c_int32(0), C.c_int32(0)
        self._check(self._lib.rmd_debug_group_rows(self._h, index, C.byref(groups), C.byref(cap), None, None,
                                                   None, None, None))
        g, c = groups.value, cap.value
        atoms = np.zeros((g, 4), np.int32)
        counts = np.zeros(g, np.int32)
        partners, codes, masks = (np.zeros((g, c), np.int32) for _ in range(3))
        p = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))  # noqa: E731
        self._check(self._lib.rmd_debug_group_rows(self._h, index, C.byref(groups), C.byref(cap), p(atoms),
                                                   p(counts), p(partners), p(codes), p(masks)))
        return {"atoms": atoms, "counts": counts, "partners": partners, "codes": codes, "masks": masks,
                "capacity": c}

    def debugEvaluate(self, index=0):
        out = L.RmdEnergyReport()
        forces = np.zeros(3 * self.atom_counts[index])
        self._check(self._lib.rmd_debug_evaluate(self._h, index, C.byref(out),
                                                 forces.ctypes.data_as(C.POINTER(C.c_double))))
        return _struct_dict(out), forces

    def debugForceTerm(self, term: str, index=0):
        code = {"direct": 0, "bonded": 1, "reciprocal": 2}[term]
        forces = np.zeros(3 * self.atom_counts[index])
        self._check(self._lib.rmd_debug_force_term(self._h, index, code,
                                                   forces.ctypes.data_as(C.POINTER(C.c_double))))
        return forces

    def debugRead(self, which: str, count: int, index=0):
        code = {"real_grid": 0, "half": 1, "list_origin": 2}[which]
        out = np.zeros(count)
        self._check(self._lib.rmd_debug_read(self._h, index, code, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def debugChargeGrid(self, index=0, points=None):
        grid = np.zeros(points)
        self._check(self._lib.rmd_debug_charge_grid(self._h, index, grid.ctypes.data_as(C.POINTER(C.c_double))))
        return grid

    def debugFft(self, data, half_points, index=0):
        d = np.ascontiguousarray(data, dtype=np.float64)
        half = np.zeros(2 * half_points)
        back = np.zeros(d.size)
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        self._check(self._lib.rmd_debug_fft(self._h, index, dp(d), dp(half), dp(back)))
        return half[0::2] + 1j * half[1::2], back

    def timeKernel(self, which: str, reps: int = 20) -> float:
        """Average ms per launch of a kernel group, CUDA events on the engine's stream."""
        code = {"nonbonded": 0, "pme": 1, "integrate": 2, "bonded": 3, "rebuild": 4,
                "nonbonded_energy": 5}[which]
        ms = C.c_double(0)
        self._check(self._lib.rmd_debug_time_kernel(self._h, code, int(reps), C.byref(ms)))
        return ms.value

    def benchRun(self, count: int, blockSize: int, flushL2: bool = True) -> float:
        """run() timed on the device: summed CUDA-event milliseconds of the step blocks."""
        ms = C.c_double(0)
        self._check(self._lib.rmd_bench_run(self._h, int(count), int(blockSize), 1 if flushL2 else 0,
                                             C.byref(ms)))
        self.step += int(count)
        return ms.value

    def kernelLaunches(self) -> int:
        return int(self._lib.rmd_debug_kernel_launches(self._h))

    def setNonbonded(self, lanes: int = 32, pairFixed: bool = True):
        self._check(self._lib.rmd_debug_set_nonbonded(self._h, int(lanes), 1 if pairFixed else 0))

    def kernelShapes(self) -> dict:
        """The launch shapes in use and, for those the autotuner chose, its timings (ms)."""
        shapes = np.zeros(3, np.int32)
        ms = np.zeros(9)
        self._check(self._lib.rmd_kernel_shapes(self._h, shapes.ctypes.data_as(C.POINTER(C.c_int32)),
                                                ms.ctypes.data_as(C.POINTER(C.c_double))))

        def table(row, keys):
            return {k: float(v) for k, v in zip(keys, row) if v >= 0}

        lanes = (8, 16, 32) if self.diagnostics()["pair_list"] == 1 else (32, 64, 128)
        return {"neighbourGroupAtoms": int(shapes[0]), "nonbondedLanes": int(shapes[1]),
                "spreadAtomsPerBlock": int(shapes[2]),
                "tuned": {"neighbourGroupAtoms": table(ms[0:3], (4, 8, 16)),
                          "nonbondedLanes": table(ms[3:6], lanes),
                          "spreadAtomsPerBlock": table(ms[6:9], (4, 8, 16))}}

    def surrogateReport(self, index=0) -> dict:
        out = L.RmdSurrogateReport()
        self._check(self._lib.rmd_surrogate_report_at(self._h, index, C.byref(out)))
        return _struct_dict(out)

    def surrogateWeights(self, index=0) -> np.ndarray:
        w = np.zeros(SURROGATE_PARAMS, np.float32)
        self._check(self._lib.rmd_surrogate_weights(self._h, index, w.ctypes.data_as(C.POINTER(C.c_float))))
        return w

    def setKernelShapes(self, neighbourGroupAtoms: int = 0, nonbondedLanes: int = 0,
                        spreadAtomsPerBlock: int = 0):
        self._check(self._lib.rmd_set_kernel_shapes(self._h, int(neighbourGroupAtoms), int(nonbondedLanes),
                                                    int(spreadAtomsPerBlock)))

    def release(self):
        if getattr(self, "_h", None):
            self._lib.rmd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class GpuSimulation(BatchSimulation):
    """One system; the signatures of webgpu/simulation.js's GpuSimulation."""

    def __init__(self, system: dict, options: dict | None = None):
        super().__init__([system], [options or {}])
        self.system = system

    def setState(self, positions, velocities=None, step=0, suppliedNoise=False):
        super().setState(0, positions, velocities, step, suppliedNoise)

    def setNoise(self, noise):
        super().setNoise(0, noise)

    def scaleVolume(self, lengthScale):
        out = C.c_double(0)
        self._check(self._lib.rmd_scale_volume(self._h, float(lengthScale), C.byref(out)))
        return out.value
