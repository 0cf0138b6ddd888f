"""ctypes binding of librmd.so (include/rmd.h). Fails loudly when the library is missing:
there is no CPU fallback for the engine."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librmd.so")

_i32p = C.POINTER(C.c_int32)
_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)

RMD_OK = 0
RMD_ERR_INVALID = 1
RMD_ERR_NEIGHBOUR_OVERFLOW = 2
RMD_ERR_NON_FINITE = 3
RMD_ERR_BUDGET = 4
RMD_ERR_STOPPED = 5
RMD_ERR_CUDA = 6
RMD_ERR_CONSTRAINTS = 7
RMD_NO_PRESSURE = -1.0e300


class RmdSystem(C.Structure):
    _fields_ = [
        ("atom_count", C.c_int32), ("charges", _dp), ("masses", _dp), ("atom_types", _i32p),
        ("type_count", C.c_int32), ("lj_a", _dp), ("lj_b", _dp),
        ("exclusion_start", _i32p), ("exclusion_partners", _i32p),
        ("bond_count", C.c_int32), ("bond_atoms", _i32p), ("bond_k", _dp), ("bond_r0", _dp),
        ("angle_count", C.c_int32), ("angle_atoms", _i32p), ("angle_k", _dp), ("angle_theta0", _dp),
        ("torsion_count", C.c_int32), ("torsion_atoms", _i32p), ("torsion_k", _dp),
        ("torsion_periodicity", _dp), ("torsion_phase", _dp),
        ("constraint_count", C.c_int32), ("constraint_atoms", _i32p), ("constraint_distance", _dp),
        ("exception_count", C.c_int32), ("exception_atoms", _i32p),
        ("exception_charge_product", _dp), ("exception_lj_a", _dp), ("exception_lj_b", _dp),
        ("molecule_count", C.c_int32), ("molecule_of_atom", _i32p),
        ("box_vectors", _dp), ("degrees_of_freedom", C.c_int32), ("cutoff", C.c_double),
    ]


class RmdOptions(C.Structure):
    _fields_ = [
        ("timestep", C.c_double), ("temperature", C.c_double), ("friction", C.c_double),
        ("seed", C.c_uint32), ("tolerance", C.c_double), ("max_constraint_iterations", C.c_int32),
        ("rebuild_interval", C.c_int32), ("adaptive_rebuild", C.c_int32), ("pressure", C.c_double),
        ("barostat_interval", C.c_int32), ("dispersion_correction", C.c_int32),
        ("restraint_force", C.c_double), ("restraint_count", C.c_int32),
        ("restraint_atoms", _i32p), ("restraint_reference", _dp),
        ("skin", C.c_double), ("neighbour_slack", C.c_double), ("max_neighbours", C.c_int32),
        ("ewald_tolerance", C.c_double), ("alpha", C.c_double), ("grid", C.c_int32 * 3),
        ("pme_order", C.c_int32), ("water_solver", C.c_int32), ("learned_barostat", C.c_int32),
        ("force_accumulation", C.c_int32), ("neighbour_group_atoms", C.c_int32),
        ("nonbonded_lanes", C.c_int32), ("spread_atoms_per_block", C.c_int32),
        ("learned_warmup_moves", C.c_int32), ("learned_steps_per_move", C.c_int32),
        ("learned_rate", C.c_double), ("rebuild_on_demand", C.c_int32), ("pair_list", C.c_int32),
    ]


class RmdSurrogateReport(C.Structure):
    _fields_ = [
        ("samples", C.c_int64), ("train_steps", C.c_int64), ("loss", C.c_double),
        ("prediction_error_kT", C.c_double), ("screening", C.c_int32), ("attempts", C.c_int64),
        ("exact_evaluations", C.c_int64), ("screened", C.c_int64), ("accepted", C.c_int64),
        ("exact_passes", C.c_int64), ("skipped_passes", C.c_int64),
    ]


class RmdEnergyReport(C.Structure):
    _fields_ = [
        ("step", C.c_int64), ("time", C.c_double),
        ("bonded", C.c_double), ("harmonic_bond", C.c_double), ("harmonic_angle", C.c_double),
        ("periodic_torsion", C.c_double), ("lennard_jones", C.c_double), ("dispersion", C.c_double),
        ("coulomb_direct", C.c_double), ("coulomb_reciprocal", C.c_double),
        ("coulomb_self", C.c_double), ("coulomb", C.c_double), ("position_restraint", C.c_double),
        ("restrained_atoms", C.c_int32), ("potential", C.c_double), ("kinetic", C.c_double),
        ("total", C.c_double), ("temperature", C.c_double), ("kinetic_for_temperature", C.c_double),
        ("kinetic_sampled_before_closing_kick", C.c_int32), ("volume", C.c_double),
        ("box_vectors", C.c_double * 9), ("volume_derivative", C.c_double),
    ]


class RmdVolumeMove(C.Structure):
    _fields_ = [
        ("attempted", C.c_int32), ("accepted", C.c_int32), ("refused", C.c_int32),
        ("screened", C.c_int32), ("weight", C.c_double), ("delta_volume", C.c_double),
        ("length_scale", C.c_double), ("old_potential", C.c_double), ("new_potential", C.c_double),
        ("volume", C.c_double), ("volume_scale", C.c_double), ("acceptance_rate", C.c_double),
    ]


class RmdMinimiseResult(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32), ("rejected", C.c_int32), ("stalled", C.c_int32),
        ("converged", C.c_int32), ("potential", C.c_double), ("max_force", C.c_double),
        ("max_step", C.c_double),
    ]


class RmdDiagnostics(C.Structure):
    _fields_ = [
        ("max_shake_iterations", C.c_int32), ("shake_hit_iteration_cap", C.c_int32),
        ("rattle_hit_iteration_cap", C.c_int32), ("worst_stalled_residual", C.c_double),
        ("neighbour_required", C.c_int32), ("neighbour_capacity", C.c_int32),
        ("worst_neighbour_required", C.c_int32), ("neighbour_growths", C.c_int32),
        ("skin", C.c_double), ("worst_displacement", C.c_double), ("worst_skin_ratio", C.c_double),
        ("skin_violations", C.c_int32), ("steps_with_stale_list", C.c_int64),
        ("rebuild_interval", C.c_int32), ("requested_rebuild_interval", C.c_int32),
        ("rebuild_shrinks", C.c_int32), ("rebuild_growths", C.c_int32),
        ("worst_skin_usage", C.c_double), ("adaptive_rebuild", C.c_int32), ("volume", C.c_double),
        ("barostat_attempts", C.c_int32), ("barostat_accepted", C.c_int32),
        ("barostat_refused", C.c_int32), ("barostat_screened", C.c_int32),
        ("barostat_exact_evaluations", C.c_int32), ("volume_scale", C.c_double),
        ("constraint_tolerance", C.c_double), ("requested_tolerance", C.c_double),
        ("tolerance_floor", C.c_double), ("cell_counts", C.c_int32 * 3),
        ("pme_grid", C.c_int32 * 3), ("pme_alpha", C.c_double), ("pme_order", C.c_int32),
        ("cluster_count", C.c_int32), ("settle_count", C.c_int32), ("device_bytes", C.c_int64),
        ("list_builds", C.c_int64), ("rebuild_on_demand", C.c_int32), ("pair_list", C.c_int32),
    ]


class RmdPlan(C.Structure):
    _fields_ = [
        ("skin", C.c_double), ("cutoff", C.c_double), ("list_cutoff", C.c_double),
        ("counts", C.c_int32 * 3), ("cell_count", C.c_int32), ("stencil_cells", C.c_int32),
        ("estimated_neighbours", C.c_double), ("max_neighbours", C.c_int32), ("capacity", C.c_int32),
        ("mean_occupancy", C.c_double), ("alpha", C.c_double), ("grid", C.c_int32 * 3), ("order", C.c_int32),
    ]


EXPORTS = [
    "rmd_default_options", "rmd_create", "rmd_create_batch", "rmd_system_count", "rmd_set_state",
    "rmd_set_state_at", "rmd_set_noise", "rmd_set_noise_at", "rmd_initialise", "rmd_run",
    "rmd_minimise", "rmd_attempt_volume_change", "rmd_last_volume_move_at", "rmd_scale_volume",
    "rmd_energy", "rmd_energy_at", "rmd_read_positions", "rmd_read_state", "rmd_read_state_at",
    "rmd_diagnostics", "rmd_diagnostics_at", "rmd_destroy", "rmd_last_error", "rmd_debug_cells",
    "rmd_debug_neighbours", "rmd_debug_evaluate", "rmd_debug_charge_grid", "rmd_debug_fft",
    "rmd_debug_time_kernel", "rmd_debug_kernel_launches", "rmd_debug_set_nonbonded", "rmd_debug_plane_pass",
    "rmd_bench_run", "rmd_debug_force_term", "rmd_debug_read", "rmd_spread_charges_noalloc",
    "rmd_kernel_shapes", "rmd_set_kernel_shapes", "rmd_surrogate_report_at", "rmd_surrogate_weights",
    "rmd_surrogate_evaluate", "rmd_image_molecules_at", "rmd_dcd_frame_bytes", "rmd_dcd_frame_at",
    "rmd_dcd_header", "rmd_restart_at", "rmd_render_at", "rmd_render_positions", "rmd_plan_system",
    "rmd_grown_capacity", "rmd_debug_draws", "rmd_debug_group_rows",
]

_lib = None


def load():
    """Load librmd.so (building it first if this tree has nvcc and it is stale)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        try:
            from .build import build
            build()
        except Exception as error:  # pragma: no cover - surfaced below
            raise RuntimeError(f"librmd.so is missing and could not be built: {error}") from error
    lib = C.CDLL(LIB_PATH)
    S = C.POINTER(C.c_void_p)
    sim = C.c_void_p
    lib.rmd_default_options.argtypes = [C.POINTER(RmdOptions)]
    lib.rmd_default_options.restype = None
    lib.rmd_create.argtypes = [C.POINTER(RmdSystem), C.POINTER(RmdOptions), S]
    lib.rmd_create_batch.argtypes = [C.c_int32, C.POINTER(RmdSystem), C.POINTER(RmdOptions), S]
    lib.rmd_system_count.argtypes = [sim]
    lib.rmd_system_count.restype = C.c_int32
    lib.rmd_set_state.argtypes = [sim, _dp, _dp, C.c_int64, C.c_int32]
    lib.rmd_set_state_at.argtypes = [sim, C.c_int32, _dp, _dp, C.c_int64, C.c_int32]
    lib.rmd_set_noise.argtypes = [sim, _fp]
    lib.rmd_set_noise_at.argtypes = [sim, C.c_int32, _fp]
    lib.rmd_initialise.argtypes = [sim]
    lib.rmd_run.argtypes = [sim, C.c_int64, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    lib.rmd_minimise.argtypes = [sim, C.c_int32, C.c_double, C.c_double, C.c_double,
                                 C.POINTER(RmdMinimiseResult)]
    lib.rmd_attempt_volume_change.argtypes = [sim, C.POINTER(RmdVolumeMove)]
    lib.rmd_last_volume_move_at.argtypes = [sim, C.c_int32, C.POINTER(RmdVolumeMove)]
    lib.rmd_scale_volume.argtypes = [sim, C.c_double, _dp]
    lib.rmd_energy.argtypes = [sim, C.POINTER(RmdEnergyReport)]
    lib.rmd_energy_at.argtypes = [sim, C.c_int32, C.POINTER(RmdEnergyReport)]
    lib.rmd_read_positions.argtypes = [sim, _fp]
    lib.rmd_read_state.argtypes = [sim, _fp, _fp, _fp, _dp, _dp]
    lib.rmd_read_state_at.argtypes = [sim, C.c_int32, _fp, _fp, _fp, _dp, _dp]
    lib.rmd_diagnostics.argtypes = [sim, C.POINTER(RmdDiagnostics)]
    lib.rmd_diagnostics_at.argtypes = [sim, C.c_int32, C.POINTER(RmdDiagnostics)]
    lib.rmd_destroy.argtypes = [sim]
    lib.rmd_destroy.restype = None
    lib.rmd_last_error.argtypes = [sim]
    lib.rmd_last_error.restype = C.c_char_p
    lib.rmd_debug_cells.argtypes = [sim, C.c_int32, _i32p, _i32p, _i32p]
    lib.rmd_debug_neighbours.argtypes = [sim, C.c_int32, _i32p, _i32p, _i32p, _i32p]
    lib.rmd_debug_evaluate.argtypes = [sim, C.c_int32, C.POINTER(RmdEnergyReport), _dp]
    lib.rmd_debug_charge_grid.argtypes = [sim, C.c_int32, _dp]
    lib.rmd_debug_fft.argtypes = [sim, C.c_int32, _dp, _dp, _dp]
    lib.rmd_debug_time_kernel.argtypes = [sim, C.c_int32, C.c_int32, _dp]
    lib.rmd_debug_kernel_launches.argtypes = [sim]
    lib.rmd_debug_kernel_launches.restype = C.c_int64
    lib.rmd_debug_plane_pass.argtypes = [C.c_int32, C.c_int32]
    lib.rmd_debug_plane_pass.restype = C.c_int32
    lib.rmd_debug_set_nonbonded.argtypes = [sim, C.c_int32, C.c_int32]
    lib.rmd_kernel_shapes.argtypes = [sim, _i32p, _dp]
    lib.rmd_set_kernel_shapes.argtypes = [sim, C.c_int32, C.c_int32, C.c_int32]
    lib.rmd_surrogate_report_at.argtypes = [sim, C.c_int32, C.POINTER(RmdSurrogateReport)]
    lib.rmd_surrogate_weights.argtypes = [sim, C.c_int32, _fp]
    lib.rmd_surrogate_evaluate.argtypes = [_fp, _fp, _fp, C.c_int32, _fp, _fp, _dp]
    lib.rmd_bench_run.argtypes = [sim, C.c_int64, C.c_int32, C.c_int32, _dp]
    lib.rmd_debug_force_term.argtypes = [sim, C.c_int32, C.c_int32, _dp]
    lib.rmd_debug_read.argtypes = [sim, C.c_int32, C.c_int32, _dp]
    lib.rmd_spread_charges_noalloc.argtypes = [C.c_void_p, C.c_int32, _dp, _i32p, C.c_int32, C.c_void_p,
                                               C.c_void_p]
    lib.rmd_image_molecules_at.argtypes = [sim, C.c_int32, _dp]
    lib.rmd_dcd_frame_bytes.argtypes = [C.c_int32, C.c_int32]
    lib.rmd_dcd_frame_bytes.restype = C.c_int64
    lib.rmd_dcd_frame_at.argtypes = [sim, C.c_int32, C.c_int32, C.c_int32, C.c_void_p]
    lib.rmd_dcd_header.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_int32,
                                   C.c_char_p, C.c_char_p, C.c_void_p]
    lib.rmd_restart_at.argtypes = [sim, C.c_int32, C.c_char_p, C.c_double, C.c_int32, C.c_int32, C.c_void_p,
                                   C.c_int64, C.POINTER(C.c_int64)]
    render_args = [C.c_void_p, _fp, _fp, C.c_int32, C.POINTER(C.c_uint32), C.c_int32, C.c_int32, C.c_int32,
                   C.c_int32, C.c_int32, C.POINTER(C.c_uint8)]
    lib.rmd_render_at.argtypes = [sim, C.c_int32, *render_args]
    lib.rmd_render_positions.argtypes = [_fp, C.c_int32, *render_args]
    lib.rmd_plan_system.argtypes = [C.POINTER(RmdSystem), C.POINTER(RmdOptions), C.POINTER(RmdPlan)]
    lib.rmd_grown_capacity.argtypes = [C.c_int32, C.c_int32]
    lib.rmd_grown_capacity.restype = C.c_int32
    lib.rmd_debug_draws.argtypes = [C.c_uint32, C.c_uint32, C.c_int32, C.c_uint32, _fp, _fp]
    lib.rmd_debug_group_rows.argtypes = [sim, C.c_int32, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p]
    for name in EXPORTS:
        fn = getattr(lib, name)
        if fn.restype is C.c_int and name not in ("rmd_system_count",):
            fn.restype = C.c_int32
    _lib = lib
    return lib
