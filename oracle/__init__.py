"""CPU oracle for the RainMD MD step — TEST INFRASTRUCTURE ONLY.

Only tests/, `__graft_entry__.smoke()` and the CPU-baseline leg of bench.py may import
this package. It is the checker the CUDA path is compared against, never part of the
product: the engine in `rainmd_b200` has no import of it and no CPU fallback.

`liboracle.so` is compiled from `rmd_oracle.c` (an FP64 restatement of RainMD's
`cpu/` and `shared/` reference code, plus an f32 restatement of the WGSL cell and
neighbour search for bit-exact checks) by `build()`.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
SOURCE = os.path.join(HERE, "rmd_oracle.c")
SOURCES = [SOURCE, os.path.join(HERE, "raster.c")]

_i = C.POINTER(C.c_int)
_d = C.POINTER(C.c_double)
_f = C.POINTER(C.c_float)


class OrcSystem(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("charges", _d), ("masses", _d), ("types", _i), ("ntypes", C.c_int),
        ("lj_a", _d), ("lj_b", _d),
        ("nbonds", C.c_int), ("bond_a", _i), ("bond_b", _i), ("bond_k", _d), ("bond_r0", _d),
        ("nangles", C.c_int), ("angle_a", _i), ("angle_b", _i), ("angle_c", _i),
        ("angle_k", _d), ("angle_theta0", _d),
        ("ntorsions", C.c_int), ("tor_a", _i), ("tor_b", _i), ("tor_c", _i), ("tor_d", _i),
        ("tor_k", _d), ("tor_n", _d), ("tor_phase", _d),
        ("nexceptions", C.c_int), ("exc_a", _i), ("exc_b", _i), ("exc_q", _d),
        ("exc_lja", _d), ("exc_ljb", _d),
        ("nconstraints", C.c_int), ("con_a", _i), ("con_b", _i), ("con_d", _d),
        ("nmolecules", C.c_int), ("mol_start", _i), ("mol_atoms", _i),
        ("box", _d), ("cutoff", C.c_double), ("degrees_of_freedom", C.c_int),
    ]


class OrcIntegrator(C.Structure):
    _fields_ = [("timestep", C.c_double), ("temperature", C.c_double),
                ("friction", C.c_double), ("seed", C.c_uint32), ("tolerance", C.c_double),
                ("max_iterations", C.c_int)]


def build(force: bool = False) -> str:
    """Compile liboracle.so with gcc (OpenMP, no floating-point contraction)."""
    if not force and os.path.exists(LIB_PATH) and all(
            os.path.getmtime(LIB_PATH) >= os.path.getmtime(s) for s in SOURCES):
        return LIB_PATH
    cmd = ["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC",
           "-o", LIB_PATH, *SOURCES, "-lm"]
    subprocess.run(cmd, check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _bind(_lib)
        _bind_render(_lib)
    return _lib


def _bind_render(L):
    f = C.POINTER(C.c_float)
    L.orc_render.argtypes = [f, C.c_int, f, f, f, C.c_int, C.POINTER(C.c_uint), C.c_int, C.c_int, C.c_int,
                             C.c_int, C.c_int, C.POINTER(C.c_ubyte)]
    L.orc_render.restype = None


def render(positions, camera, styles, guides=None, segments=None, spheres=True, ribbon=True,
           width=64, height=48):
    """The renderer's oracle (raster.c): an RGBA8 image [height, width, 4]."""
    L = lib()
    f = C.POINTER(C.c_float)
    pos = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1)
    cam = np.ascontiguousarray(camera, dtype=np.float32).reshape(-1)
    sty = np.ascontiguousarray(styles if styles is not None else np.zeros(4), dtype=np.float32).reshape(-1)
    gui = np.ascontiguousarray(guides if guides is not None else np.zeros(12), dtype=np.float32).reshape(-1)
    seg = np.ascontiguousarray(segments if segments is not None else np.zeros(4), dtype=np.uint32).reshape(-1)
    nseg = 0 if segments is None else len(seg) // 4
    out = np.zeros((height, width, 4), np.uint8)
    L.orc_render(pos.ctypes.data_as(f), len(pos) // 3, cam.ctypes.data_as(f), sty.ctypes.data_as(f),
                 gui.ctypes.data_as(f), len(gui) // 12, seg.ctypes.data_as(C.POINTER(C.c_uint)), nseg,
                 1 if spheres else 0, 1 if ribbon else 0, width, height,
                 out.ctypes.data_as(C.POINTER(C.c_ubyte)))
    return out


def _bind(L):
    S = C.POINTER(OrcSystem)
    I = C.POINTER(OrcIntegrator)
    L.orc_erfc.restype = C.c_double
    L.orc_erfc.argtypes = [C.c_double]
    L.orc_erf.restype = C.c_double
    L.orc_erf.argtypes = [C.c_double]
    L.orc_uniform_at.restype = C.c_double
    L.orc_uniform_at.argtypes = [C.c_uint32] * 4
    L.orc_gaussian_triple.argtypes = [_d, C.c_uint32, C.c_uint32, C.c_uint32]
    L.orc_set_threads.argtypes = [C.c_int]
    L.orc_get_threads.restype = C.c_int
    L.orc_alpha_from_tolerance.restype = C.c_double
    L.orc_alpha_from_tolerance.argtypes = [C.c_double, C.c_double]
    L.orc_grid_size_for.argtypes = [_d, C.c_double, C.c_double, _i]
    L.orc_bspline.argtypes = [C.c_double, C.c_int, _d, _d]
    L.orc_bspline_moduli.restype = C.c_int
    L.orc_bspline_moduli.argtypes = [C.c_int, C.c_int, _d]
    L.orc_dft_axis.argtypes = [_d, _i, C.c_int, C.c_int]
    L.orc_reciprocal.restype = C.c_double
    L.orc_reciprocal.argtypes = [S, _d, C.c_double, _i, C.c_int, _d, _d]
    L.orc_ewald_self.argtypes = [S, C.c_double, _d]
    L.orc_dispersion_coefficients.argtypes = [S, _d]
    L.orc_dispersion_energy.restype = C.c_double
    L.orc_dispersion_energy.argtypes = [_d, C.c_double, C.c_double]
    L.orc_direct_space.argtypes = [S, _d, C.c_double, C.c_double, _d, _d, _d]
    L.orc_exceptions.argtypes = [S, _d, C.c_double, _d, _d, _d]
    for name in ("orc_bonds", "orc_angles", "orc_torsions"):
        getattr(L, name).restype = C.c_double
        getattr(L, name).argtypes = [S, _d, _d]
    L.orc_restraint.restype = C.c_double
    L.orc_restraint.argtypes = [S, C.c_int, _i, _d, C.c_double, _d, _d]
    L.orc_potential.argtypes = [S, _d, C.c_int, C.c_double, _i, C.c_int, C.c_int, _i, _d,
                                C.c_double, _d, _d]
    L.orc_constrain_positions.restype = C.c_int
    L.orc_constrain_positions.argtypes = [S, _d, _d, C.c_double, C.c_int, _d]
    L.orc_constrain_velocities.restype = C.c_int
    L.orc_constrain_velocities.argtypes = [S, _d, _d, C.c_double, C.c_int]
    L.orc_langevin_step.restype = C.c_int
    L.orc_langevin_step.argtypes = [S, _d, _d, _d, I, C.c_uint32, _d]
    L.orc_finish_step.restype = C.c_int
    L.orc_finish_step.argtypes = [S, _d, _d, _d, I]
    L.orc_kinetic.restype = C.c_double
    L.orc_kinetic.argtypes = [S, _d]
    L.orc_run_dynamics.restype = C.c_double
    L.orc_run_dynamics.argtypes = [S, _d, _d, C.c_int, C.c_uint32, I, C.c_double, _i, C.c_int, _d]
    L.orc_metropolis_weight.restype = C.c_double
    L.orc_metropolis_weight.argtypes = [C.c_double] * 5 + [C.c_int]
    L.orc_scale_molecules.argtypes = [S, _d, C.c_double]
    L.orc_cell_list_f32.argtypes = [C.c_int, _f, _f, _i, _i, _i, _i]
    L.orc_neighbour_list_f32.restype = C.c_int
    L.orc_neighbour_list_f32.argtypes = [C.c_int, _f, _f, _i, _i, _i, _i, _i, C.c_int, _i, _i]
    L.orc_reciprocal_box.argtypes = [_d, _d]


def _p(array, ctype):
    return array.ctypes.data_as(C.POINTER(ctype))


class Oracle:
    """Holds a ctypes view of one built system (the arrays stay alive with it)."""

    def __init__(self, system: dict):
        lib()
        t = system["topology"]
        self.system = system
        keep = []

        def arr(values, dtype):
            a = np.ascontiguousarray(values, dtype=dtype)
            if a.size == 0:
                a = np.zeros(1, dtype=dtype)
            keep.append(a)
            return a

        def ip(values):
            return _p(arr(values, np.int32), C.c_int)

        def dp(values):
            return _p(arr(values, np.float64), C.c_double)

        hb, an, di = system["harmonicBonds"], t["angles"], t["dihedrals"]
        ex, co, mo = system["exceptions"], system["constraints"], system["molecules"]
        s = OrcSystem()
        s.n = t["atomCount"]
        s.charges, s.masses = dp(t["charges"]), dp(t["masses"])
        s.types, s.ntypes = ip(t["atomTypes"]), t["typeCount"]
        s.lj_a, s.lj_b = dp(t["ljA"]), dp(t["ljB"])
        s.nbonds = hb["count"]
        s.bond_a, s.bond_b, s.bond_k, s.bond_r0 = ip(hb["atomA"]), ip(hb["atomB"]), dp(hb["k"]), dp(hb["r0"])
        s.nangles = an["count"]
        s.angle_a, s.angle_b, s.angle_c = ip(an["atomA"]), ip(an["atomB"]), ip(an["atomC"])
        s.angle_k, s.angle_theta0 = dp(an["k"]), dp(an["theta0"])
        s.ntorsions = di["count"]
        s.tor_a, s.tor_b, s.tor_c, s.tor_d = ip(di["atomA"]), ip(di["atomB"]), ip(di["atomC"]), ip(di["atomD"])
        s.tor_k, s.tor_n, s.tor_phase = dp(di["k"]), dp(di["periodicity"]), dp(di["phase"])
        s.nexceptions = ex["count"]
        s.exc_a, s.exc_b = ip(ex["atomA"]), ip(ex["atomB"])
        s.exc_q, s.exc_lja, s.exc_ljb = dp(ex["chargeProduct"]), dp(ex["ljA"]), dp(ex["ljB"])
        s.nconstraints = co["count"]
        s.con_a, s.con_b, s.con_d = ip(co["atomA"]), ip(co["atomB"]), dp(co["distance"])
        s.nmolecules = mo["count"]
        s.mol_start, s.mol_atoms = ip(mo["start"]), ip(mo["atoms"])
        s.box = dp(system["boxVectors"]) if system["boxVectors"] is not None else None
        s.cutoff = system["options"]["cutoff"]
        s.degrees_of_freedom = system["degreesOfFreedom"]
        self._keep = keep
        self.struct = s
        self.ref = C.byref(s)
        self.n = s.n

    # -- whole potential (cpu/energy.js) --
    def potential(self, positions, method="PME", alpha=None, grid=None, order=5,
                  restraint=None):
        L = lib()
        pos = np.ascontiguousarray(positions, dtype=np.float64)
        forces = np.zeros(3 * self.n)
        terms = np.zeros(10)
        g = np.ascontiguousarray(grid if grid is not None else [1, 1, 1], dtype=np.int32)
        if restraint is not None:
            ra = np.ascontiguousarray(restraint["atoms"], dtype=np.int32)
            rr = np.ascontiguousarray(restraint["reference"], dtype=np.float64)
            rk = float(restraint["force"])
            rcount = len(ra)
        else:
            ra, rr, rk, rcount = np.zeros(1, np.int32), np.zeros(3), 0.0, 0
        L.orc_potential(self.ref, _p(pos, C.c_double), 1 if method == "PME" else 0,
                        float(alpha or 0.0), _p(g, C.c_int), int(order), rcount,
                        _p(ra, C.c_int), _p(rr, C.c_double), rk, _p(forces, C.c_double),
                        _p(terms, C.c_double))
        names = ["harmonicBond", "harmonicAngle", "periodicTorsion", "lennardJones",
                 "coulombDirect", "coulombReciprocal", "coulombSelf", "coulombNetCharge",
                 "positionRestraint", "total"]
        energy = dict(zip(names, terms.tolist()))
        energy["bonded"] = terms[0] + terms[1] + terms[2]
        energy["coulomb"] = terms[4] + terms[5] + terms[6] + terms[7]
        return energy, forces

    def term_forces(self, positions, term, alpha=None, grid=None, order=5):
        """Forces of one term: "direct" (direct space + exceptions), "bonded", "reciprocal"."""
        L = lib()
        pos = np.ascontiguousarray(positions, dtype=np.float64)
        f = np.zeros(3 * self.n)
        a, b = C.c_double(0), C.c_double(0)
        if term == "direct":
            L.orc_direct_space(self.ref, _p(pos, C.c_double), float(alpha), float(self.struct.cutoff),
                               _p(f, C.c_double), C.byref(a), C.byref(b))
            L.orc_exceptions(self.ref, _p(pos, C.c_double), float(alpha), _p(f, C.c_double),
                             C.byref(a), C.byref(b))
        elif term == "bonded":
            for name in ("orc_bonds", "orc_angles", "orc_torsions"):
                getattr(L, name)(self.ref, _p(pos, C.c_double), _p(f, C.c_double))
        else:
            g = np.ascontiguousarray(grid, dtype=np.int32)
            L.orc_reciprocal(self.ref, _p(pos, C.c_double), float(alpha), _p(g, C.c_int), int(order),
                             _p(f, C.c_double), None)
        return f

    def reciprocal(self, positions, alpha, grid, order, want_grid=False):
        L = lib()
        pos = np.ascontiguousarray(positions, dtype=np.float64)
        forces = np.zeros(3 * self.n)
        g = np.ascontiguousarray(grid, dtype=np.int32)
        q = np.zeros(int(np.prod(grid))) if want_grid else None
        e = L.orc_reciprocal(self.ref, _p(pos, C.c_double), float(alpha), _p(g, C.c_int),
                             int(order), _p(forces, C.c_double),
                             _p(q, C.c_double) if q is not None else None)
        return (e, forces, q) if want_grid else (e, forces)

    def self_energy(self, alpha):
        out = np.zeros(2)
        lib().orc_ewald_self(self.ref, float(alpha), _p(out, C.c_double))
        return out

    def dispersion(self, volume, cutoff):
        ab = np.zeros(2)
        lib().orc_dispersion_coefficients(self.ref, _p(ab, C.c_double))
        return lib().orc_dispersion_energy(_p(ab, C.c_double), float(volume), float(cutoff))

    def scale_molecules(self, positions, scale):
        pos = np.ascontiguousarray(positions, dtype=np.float64).copy()
        lib().orc_scale_molecules(self.ref, _p(pos, C.c_double), float(scale))
        return pos

    def integrator(self, timestep=0.002, temperature=300.0, friction=1.0, seed=0,
                   tolerance=1e-5, max_iterations=150):
        o = OrcIntegrator()
        o.timestep, o.temperature, o.friction = timestep, temperature, friction
        o.seed, o.tolerance, o.max_iterations = seed, tolerance, max_iterations
        return o

    def langevin_step(self, positions, velocities, forces, integ, step, noise=None):
        pos = np.ascontiguousarray(positions, dtype=np.float64).copy()
        vel = np.ascontiguousarray(velocities, dtype=np.float64).copy()
        f = np.ascontiguousarray(forces, dtype=np.float64)
        nz = np.ascontiguousarray(noise, dtype=np.float64) if noise is not None else None
        status = lib().orc_langevin_step(self.ref, _p(pos, C.c_double), _p(vel, C.c_double),
                                         _p(f, C.c_double), C.byref(integ), int(step),
                                         _p(nz, C.c_double) if nz is not None else None)
        return pos, vel, status

    def finish_step(self, positions, velocities, forces, integ):
        pos = np.ascontiguousarray(positions, dtype=np.float64)
        vel = np.ascontiguousarray(velocities, dtype=np.float64).copy()
        f = np.ascontiguousarray(forces, dtype=np.float64)
        lib().orc_finish_step(self.ref, _p(pos, C.c_double), _p(vel, C.c_double),
                              _p(f, C.c_double), C.byref(integ))
        return vel

    def kinetic(self, velocities):
        v = np.ascontiguousarray(velocities, dtype=np.float64)
        return lib().orc_kinetic(self.ref, _p(v, C.c_double))

    def run_dynamics(self, positions, velocities, steps, first_step, integ, alpha, grid, order):
        pos = np.ascontiguousarray(positions, dtype=np.float64).copy()
        vel = np.ascontiguousarray(velocities, dtype=np.float64).copy()
        g = np.ascontiguousarray(grid, dtype=np.int32)
        kin = C.c_double(0)
        e = lib().orc_run_dynamics(self.ref, _p(pos, C.c_double), _p(vel, C.c_double), int(steps),
                                   int(first_step), C.byref(integ), float(alpha),
                                   _p(g, C.c_int), int(order), C.byref(kin))
        return pos, vel, e, kin.value

    def constrain_positions(self, positions, reference, tolerance, max_iterations=150):
        pos = np.ascontiguousarray(positions, dtype=np.float64).copy()
        ref = np.ascontiguousarray(reference, dtype=np.float64)
        it = lib().orc_constrain_positions(self.ref, _p(pos, C.c_double), _p(ref, C.c_double),
                                           float(tolerance), int(max_iterations), None)
        return pos, it

    # -- steepest descent (webgpu/simulation.js:880-979, integrate.js:589-688) --
    def minimise(self, positions, max_iterations=200, force_tolerance=500.0, max_step=0.002,
                 max_displacement=0.05, constraint_tolerance=1e-7, **potential_args):
        """The reference's line search in FP64: at the accepted structure, stop when the
        largest per-atom force is within tolerance; otherwise try up to 14 steps that move the
        largest force `max_step` nm (every displacement capped at `max_displacement`),
        projected onto the constraints against the pre-move structure. A lower potential is
        accepted and grows the step by 1.3; a rejection halves it, and 14 rejections or a step
        below 1e-9 stall the search. As on the device, a rejected trial leaves the accepted
        structure AND its forces in place."""
        pos = np.asarray(positions, dtype=np.float64).reshape(-1, 3).copy()

        def evaluate(p):
            e, f = self.potential(p.reshape(-1), **potential_args)
            return e["total"], f.reshape(-1, 3)

        potential, forces = evaluate(pos)
        iterations = rejected = 0
        stalled = False
        for iteration in range(max_iterations):
            iterations = iteration + 1
            worst = float(np.max(np.linalg.norm(forces, axis=1)))
            if worst <= force_tolerance:
                break
            accepted = False
            for _ in range(14):
                d = forces * (max_step / max(worst, 1e-6))
                norm = np.linalg.norm(d, axis=1)
                over = norm > max_displacement
                d[over] *= (max_displacement / norm[over])[:, None]
                trial, _ = self.constrain_positions((pos + d).reshape(-1), pos.reshape(-1),
                                                    constraint_tolerance)
                trial = trial.reshape(-1, 3)
                e, f = evaluate(trial)
                if e < potential:
                    potential, pos, forces = e, trial, f
                    max_step *= 1.3
                    accepted = True
                    break
                rejected += 1
                max_step *= 0.5
                if max_step < 1e-9:
                    break
            if not accepted:
                stalled = True
                break
        worst = float(np.max(np.linalg.norm(forces, axis=1)))
        return {"positions": pos.reshape(-1), "iterations": iterations, "rejected": rejected,
                "stalled": stalled, "converged": worst <= force_tolerance, "potential": potential,
                "max_force": worst, "max_step": max_step}


def erfc(x: float) -> float:
    return lib().orc_erfc(float(x))


def erf(x: float) -> float:
    return lib().orc_erf(float(x))


def uniform_at(seed, a, b, c) -> float:
    return lib().orc_uniform_at(seed & 0xFFFFFFFF, a & 0xFFFFFFFF, b & 0xFFFFFFFF, c & 0xFFFFFFFF)


def gaussian_triple(seed, atom, step):
    out = np.zeros(3)
    lib().orc_gaussian_triple(_p(out, C.c_double), seed, atom, step)
    return out


def bspline(offset, order):
    w = np.zeros(order)
    d = np.zeros(order)
    lib().orc_bspline(float(offset), int(order), _p(w, C.c_double), _p(d, C.c_double))
    return w, d


def bspline_moduli(size, order):
    out = np.zeros(size)
    ok = lib().orc_bspline_moduli(int(size), int(order), _p(out, C.c_double))
    if not ok:
        raise ValueError("B-spline modulus still zero after patching")
    return out


def alpha_from_tolerance(cutoff, tolerance):
    return lib().orc_alpha_from_tolerance(float(cutoff), float(tolerance))


def grid_size_for(box, alpha, tolerance):
    b = np.ascontiguousarray(box, dtype=np.float64)
    g = np.zeros(3, dtype=np.int32)
    lib().orc_grid_size_for(_p(b, C.c_double), float(alpha), float(tolerance), _p(g, C.c_int))
    return g.tolist()


def dft_axis(data, grid, axis, sign):
    d = np.ascontiguousarray(data, dtype=np.float64).copy()
    g = np.ascontiguousarray(grid, dtype=np.int32)
    lib().orc_dft_axis(_p(d, C.c_double), _p(g, C.c_int), int(axis), int(sign))
    return d


def metropolis_weight(delta_energy, delta_volume, volume_ratio, pressure, kT, molecules):
    return lib().orc_metropolis_weight(float(delta_energy), float(delta_volume),
                                       float(volume_ratio), float(pressure), float(kT),
                                       int(molecules))


def set_threads(count: int):
    lib().orc_set_threads(int(count))


def get_threads() -> int:
    return lib().orc_get_threads()


def pack_params(box, cutoff, list_cutoff, alpha, coulomb=138.935456):
    """The 28-float uniform of the reference's wgsl-common.js:24-64, as f32."""
    b = np.asarray(box, dtype=np.float64)
    r = np.zeros(9)
    lib().orc_reciprocal_box(_p(np.ascontiguousarray(b), C.c_double), _p(r, C.c_double))
    P = np.zeros(28, dtype=np.float32)
    for row in range(3):
        P[row * 4: row * 4 + 3] = b[row * 3: row * 3 + 3]
        P[12 + row * 4: 12 + row * 4 + 3] = r[row * 3: row * 3 + 3]
    P[24], P[25], P[26], P[27] = cutoff, list_cutoff, alpha, coulomb
    return P


def cell_list_f32(positions32, params, counts):
    n = len(positions32) // 3
    pos = np.ascontiguousarray(positions32, dtype=np.float32)
    P = np.ascontiguousarray(params, dtype=np.float32)
    cnt = np.ascontiguousarray(counts, dtype=np.int32)
    cells = int(np.prod(counts))
    coa = np.zeros(n, np.int32)
    cs = np.zeros(cells + 1, np.int32)
    ca = np.zeros(n, np.int32)
    lib().orc_cell_list_f32(n, _p(pos, C.c_float), _p(P, C.c_float), _p(cnt, C.c_int),
                            _p(coa, C.c_int), _p(cs, C.c_int), _p(ca, C.c_int))
    return coa, cs, ca


def neighbour_list_f32(positions32, params, counts, cell_start, cell_atoms, excl_start,
                       excl_partners, capacity):
    n = len(positions32) // 3
    pos = np.ascontiguousarray(positions32, dtype=np.float32)
    P = np.ascontiguousarray(params, dtype=np.float32)
    cnt = np.ascontiguousarray(counts, dtype=np.int32)
    cs = np.ascontiguousarray(cell_start, dtype=np.int32)
    ca = np.ascontiguousarray(cell_atoms, dtype=np.int32)
    es = np.ascontiguousarray(excl_start, dtype=np.int32)
    ep = np.ascontiguousarray(excl_partners if len(excl_partners) else np.zeros(1), dtype=np.int32)
    nb = np.zeros(n * capacity, np.int32)
    nc = np.zeros(n, np.int32)
    req = lib().orc_neighbour_list_f32(n, _p(pos, C.c_float), _p(P, C.c_float), _p(cnt, C.c_int),
                                       _p(cs, C.c_int), _p(ca, C.c_int), _p(es, C.c_int),
                                       _p(ep, C.c_int), int(capacity), _p(nb, C.c_int),
                                       _p(nc, C.c_int))
    return nb.reshape(n, capacity), nc, req


# ---------------------------------------------------------------------------- cell plan
# shared/topology/cells.js restated in Python floats (the JavaScript Number): the stencil's
# per-axis offsets, skinFor, planCellList and grownPlan. Test infrastructure only.

def axis_offsets(cell_count: int):
    """cells.js:25-29: three cells or more visit {-1, 0, 1}; two visit {0, 1}; one {0}."""
    if cell_count >= 3:
        return [-1, 0, 1]
    if cell_count == 2:
        return [0, 1]
    return [0]


def skin_for(masses, box, cutoff, timestep=0.002, temperature=298.0):
    """cells.js:67-91 (lightestMovingMass :35-41, halfSmallestWidth :93-97): the 0.40 nm anchor
    scaled linearly by the timestep and by sqrt(T/298 * 1.008/m) of the lightest moving atom,
    capped at 0.9 of the room between the cutoff and half the smallest box width."""
    lightest = math.inf
    for m in masses:
        if m > 0 and m < lightest:
            lightest = float(m)
    if not math.isfinite(lightest):
        lightest = 1.008
    speed_ratio = math.sqrt((temperature / 298) * (1.008 / lightest))
    scaled = 0.40 * (timestep / 0.002) * speed_ratio
    widest = None if box is None else min(abs(box[0]), abs(box[4]), abs(box[8])) / 2
    room = math.inf if widest is None else widest - cutoff
    return max(0.1, min(scaled, room * 0.9 if room > 0 else 0.1))


def plan_cell_list(atom_count, box, cutoff, skin=0.1, neighbour_slack=2.0, max_neighbours=None):
    """cells.js:101-171: cells per axis floor(|w| / (cutoff + skin)) (at least one), the
    deduplicated stencil, and the capacity max(32, ceil(density * 4/3 pi (rc+skin)^3 * slack))."""
    list_cutoff = cutoff + skin
    widths = [box[0], box[4], box[8]]
    counts = [max(1, math.floor(abs(w) / list_cutoff)) for w in widths]
    offsets = [axis_offsets(c) for c in counts]
    stencil = [(dx, dy, dz) for dx in offsets[0] for dy in offsets[1] for dz in offsets[2]]
    volume = abs(box[0] * box[4] * box[8])
    density = atom_count / volume
    estimated = density * ((4 / 3) * math.pi * list_cutoff ** 3)
    capacity = max_neighbours if max_neighbours is not None else max(32, math.ceil(estimated * neighbour_slack))
    return {"skin": skin, "cutoff": cutoff, "listCutoff": list_cutoff, "counts": counts,
            "cellCount": counts[0] * counts[1] * counts[2], "stencil": stencil,
            "maxNeighbours": capacity, "estimatedNeighbours": estimated,
            "meanOccupancy": atom_count / (counts[0] * counts[1] * counts[2])}


def grown_plan(max_neighbours, required):
    """cells.js:282-288: max(maxNeighbours + 32, ceil(required * 1.25))."""
    return max(max_neighbours + 32, math.ceil(required * 1.25))


# ------------------------------------------------------------------------ volume move
BAR_TO_KJ_PER_MOL_NM3 = 0.06022140857   # shared/units.js:53
BOLTZMANN = 0.008314462618              # shared/units.js:50


def volume_move(system, positions, velocities, attempt, volume_scale, *, seed, temperature, pressure,
                alpha, grid, order, dispersion=True):
    """One Monte Carlo volume move, attemptVolumeChange (webgpu/simulation.js:995-1070) restated in
    FP64 on the oracle: the potential at the current state, a volume change drawn from
    uniformAt(seed ^ 0x5a17, attempt, 0, 0), molecule centroids scaled with the box, the
    potential of the scaled state, metropolisWeight (barostat.js:158-162) and the second draw;
    a rejected move restores the state and evaluates it again, as the reference does. The PME
    grid stays fixed. Returns (accepted, positions, box, weight, delta_volume)."""
    box = np.asarray(system["boxVectors"], dtype=np.float64)
    volume = abs(box[0] * box[4] * box[8])
    kT = BOLTZMANN * temperature
    p = pressure * BAR_TO_KJ_PER_MOL_NM3

    def total(sys_, pos, vol):
        e, _ = Oracle(sys_).potential(pos, method="PME", alpha=alpha, grid=grid, order=order)
        if dispersion:
            e["total"] += Oracle(sys_).dispersion(vol, sys_["options"]["cutoff"])
        return e["total"]

    old = total(system, positions, volume)
    draw = uniform_at((seed ^ 0x5A17) & 0xFFFFFFFF, attempt, 0, 0)
    delta = volume_scale * 2 * (draw - 0.5)
    new_volume = volume + delta
    if not new_volume > 0:
        return False, positions, box, 0.0, delta
    scale = float(np.cbrt(new_volume / volume))
    if system["options"]["cutoff"] > 0.5 * scale * min(abs(box[0]), abs(box[4]), abs(box[8])):
        return False, positions, box, 0.0, delta
    scaled_system = dict(system)
    scaled_system["boxVectors"] = box * scale
    scaled = Oracle(system).scale_molecules(positions, scale)
    new = total(scaled_system, scaled, new_volume)
    weight = metropolis_weight(new - old, delta, new_volume / volume, p, kT, system["molecules"]["count"])
    accept = weight <= 0 or uniform_at((seed ^ 0x5A17) & 0xFFFFFFFF, attempt, 1, 0) < math.exp(-weight / kT)
    if accept:
        return True, scaled, box * scale, weight, delta
    total(system, positions, volume)
    return False, positions, box, weight, delta
