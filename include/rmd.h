/*
 * rmd.h — C ABI of the B200 RainMD step engine.
 *
 * Every entry point replaces one member of RainMD's `class GpuSimulation`
 * (webgpu/simulation.js:82-1341); the comment on each names the member and its line.
 * A Node N-API addon binds these 1:1; Python binds them with ctypes (rainmd_b200/_lib.py).
 *
 * Conventions
 *   - Units are RainMD's (shared/units.js): nm, ps, kJ/mol, amu, elementary charge, K, bar.
 *   - Inputs are caller-owned host arrays, copied at the call; outputs are written into
 *     caller-owned host buffers. No pointer is retained after a call returns.
 *   - Every call returns an rmd_status (0 = ok). rmd_last_error() gives the message of the
 *     last failure on that handle; the N-API shim maps codes to RainMD's error classes.
 *   - A handle holds one or more independent systems advanced together ("batch"); system
 *     index 0 is the only one for a handle made by rmd_create. Calls on one handle must not
 *     overlap; different handles are independent.
 */
#ifndef RMD_H
#define RMD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  RMD_OK = 0,
  RMD_ERR_INVALID = 1,            /* refused input: RangeError/Error from buildSystem, pmeParameters */
  RMD_ERR_NEIGHBOUR_OVERFLOW = 2, /* NeighbourOverflowError (webgpu/kernels/neighbours.js:172-183) */
  RMD_ERR_NON_FINITE = 3,         /* NonFiniteStateError (shared/finite.js:63-95) */
  RMD_ERR_BUDGET = 4,             /* GpuBudgetError (webgpu/runtime/allocator.js:141-154) */
  RMD_ERR_STOPPED = 5,            /* SimulationStopped (webgpu/runtime/yield.js:44-50) */
  RMD_ERR_CUDA = 6,               /* device or driver failure */
  RMD_ERR_CONSTRAINTS = 7         /* constraint solver hit its iteration cap */
} rmd_status;

typedef struct rmd_sim rmd_sim;

/* The `system` object of shared/topology/system.js:205-235 (the output of buildSystem),
 * flattened. Index arrays are 0-based. */
typedef struct {
  int32_t atom_count;
  const double *charges;        /* [N] e */
  const double *masses;         /* [N] amu; <= 0 marks a massless site */
  const int32_t *atom_types;    /* [N] */
  int32_t type_count;
  const double *lj_a;           /* [T*T] kJ/mol nm^12, A/r^12 - B/r^6 */
  const double *lj_b;           /* [T*T] kJ/mol nm^6 */
  const int32_t *exclusion_start;    /* [N+1] AMBER one-sided exclusion CSR (topology.exclusions) */
  const int32_t *exclusion_partners; /* [exclusion_start[N]] */
  int32_t bond_count;           /* harmonic (unconstrained) bonds: 1/2 k (r - r0)^2 */
  const int32_t *bond_atoms;    /* [2*B] */
  const double *bond_k, *bond_r0;
  int32_t angle_count;          /* 1/2 k (theta - theta0)^2 */
  const int32_t *angle_atoms;   /* [3*A] */
  const double *angle_k, *angle_theta0;
  int32_t torsion_count;        /* k (1 + cos(n phi - phase)) */
  const int32_t *torsion_atoms; /* [4*D] */
  const double *torsion_k, *torsion_periodicity, *torsion_phase;
  int32_t constraint_count;
  const int32_t *constraint_atoms; /* [2*C] */
  const double *constraint_distance;
  int32_t exception_count;      /* every excluded pair; 1-4 pairs carry scaled parameters */
  const int32_t *exception_atoms;  /* [2*E] */
  const double *exception_charge_product, *exception_lj_a, *exception_lj_b;
  int32_t molecule_count;
  const int32_t *molecule_of_atom; /* [N] */
  const double *box_vectors;    /* [9] reduced, row-major (a, b, c); NULL = not periodic */
  int32_t degrees_of_freedom;
  double cutoff;                /* nm */
} rmd_system;

/* Constructor options of GpuSimulation (webgpu/simulation.js:93-188). A field set to its
 * "derive" value takes the reference's default. rmd_default_options() fills them. */
typedef struct {
  double timestep;              /* ps, default 0.002 */
  double temperature;           /* K, default 298 */
  double friction;              /* 1/ps, default 1.0 */
  uint32_t seed;                /* default 0 */
  double tolerance;             /* constraint tolerance, default 1e-5 (floored as clusters.js:136) */
  int32_t max_constraint_iterations; /* default 150 */
  int32_t rebuild_interval;     /* default 20 */
  int32_t adaptive_rebuild;     /* default 1 */
  double pressure;              /* bar; <= -1e30 (RMD_NO_PRESSURE) = NVT */
  int32_t barostat_interval;    /* steps, default 25 */
  int32_t dispersion_correction;/* default 1 */
  double restraint_force;       /* kJ/mol/nm^2 in k*d^2, default 0 */
  int32_t restraint_count;
  const int32_t *restraint_atoms;      /* [R] */
  const double *restraint_reference;   /* [3N] positions to restrain towards (only restrained atoms read) */
  double skin;                  /* nm; <= 0 derives it (cells.js:67 skinFor) */
  double neighbour_slack;       /* default 2.0 */
  int32_t max_neighbours;       /* <= 0 derives it */
  double ewald_tolerance;       /* default 5e-4 */
  double alpha;                 /* 1/nm; <= 0 derives it */
  int32_t grid[3];              /* <= 0 derives it */
  /* B200 engine options (no counterpart in the reference) */
  int32_t pme_order;            /* B-spline order, 4 or 5; default 5 (the reference's PME_ORDER) */
  int32_t water_solver;         /* 0 = SHAKE/RATTLE per cluster (reference); 1 = SETTLE for rigid 3-site water */
  int32_t learned_barostat;     /* 0 = exact Metropolis test; 1 = two-stage delayed acceptance with the MLP */
  int32_t force_accumulation;   /* 0 = each pair force quantised to 64-bit fixed point before summing
                                   (order-independent, bitwise reproducible; default);
                                   1 = per-lane f32 partial sums, converted once per lane */
  /* kernel shapes; 0 = chosen by the engine's autotuner at initialise() */
  int32_t neighbour_group_atoms; /* atoms per neighbour-search warp: 4, 8, 16 or 32 (per-atom rows;
                                    group-pair rows always search 4-atom groups) */
  int32_t nonbonded_lanes;       /* pair-loop lanes: per atom on per-atom rows (8, 16 or 32); per
                                    group row on group-pair rows (32, 64 or 128: one partner a
                                    lane, the row shared by 1, 2 or 4 warps) */
  int32_t spread_atoms_per_block; /* atoms per PME charge-spreading block: 4, 8 or 16 */
  /* learned barostat (learned_barostat = 1) */
  int32_t learned_warmup_moves;  /* exact moves that train the surrogate before it screens; <= 0: 2000 */
  int32_t learned_steps_per_move; /* Adam steps after each exact move; <= 0: 4 */
  double learned_rate;           /* Adam learning rate; <= 0: 1e-3 */
  /* 1 (default): the device checks every step whether some atom has moved more than half the
   * skin since the last build and rebuilds the lists exactly then (an IF node of the step
   * graph), so no step uses a stale list and no rebuild is early; rebuild_interval and
   * adaptive_rebuild are then unused. 0: the reference's host-side schedule (a rebuild every
   * rebuild_interval steps, adapted between blocks when adaptive_rebuild is set,
   * simulation.js:544-623). No reference counterpart. */
  int32_t rebuild_on_demand;
  /* Which neighbour structure the pair loop walks. 0 (default): per 4-atom group of
   * spatially close atoms, the half list of partner atoms within cutoff + skin of the group's
   * bounding box, each pair evaluated once and its force added to both atoms (64-bit
   * fixed-point atomics for the partner); needs force_accumulation 0 and at most 2^23 atoms
   * in the handle, else 1 is used. 1: the reference's full per-atom rows (neighbours.js:46-151),
   * each pair evaluated from both atoms. 2: as 0, and every build also writes the per-atom
   * rows (for inspection with rmd_debug_neighbours). Both structures give the same forces
   * bit for bit. No reference counterpart. */
  int32_t pair_list;
} rmd_options;

#define RMD_NO_PRESSURE (-1.0e300)

/* energy() — webgpu/simulation.js:1073-1230 */
typedef struct {
  int64_t step;
  double time;                  /* ps */
  double bonded, harmonic_bond, harmonic_angle, periodic_torsion;
  double lennard_jones, dispersion;
  double coulomb_direct, coulomb_reciprocal, coulomb_self, coulomb;
  double position_restraint;
  int32_t restrained_atoms;
  double potential, kinetic, total;
  double temperature, kinetic_for_temperature;
  int32_t kinetic_sampled_before_closing_kick; /* kineticSampledAt */
  double volume;
  double box_vectors[9];
  /* dU/dlnV for molecules scaled rigidly about their centres of mass, from the virial of this
   * evaluation (the learned barostat's first-order term; no reference counterpart) */
  double volume_derivative;
} rmd_energy_report;

/* attemptVolumeChange() — webgpu/simulation.js:995-1070 */
typedef struct {
  int32_t attempted;            /* 0: no barostat on this handle (the reference returns null) */
  int32_t accepted;
  int32_t refused;              /* cutoff would not fit the proposed box */
  int32_t screened;             /* learned barostat: rejected at stage 1 without an exact evaluation */
  double weight, delta_volume, length_scale;
  double old_potential, new_potential;
  double volume, volume_scale, acceptance_rate;
} rmd_volume_move;

/* minimise() — webgpu/simulation.js:880-979 */
typedef struct {
  int32_t iterations, rejected, stalled, converged;
  double potential, max_force, max_step;
} rmd_minimise_result;

/* diagnostics() — webgpu/simulation.js:1264-1334 */
typedef struct {
  int32_t max_shake_iterations;
  int32_t shake_hit_iteration_cap, rattle_hit_iteration_cap;
  double worst_stalled_residual;
  int32_t neighbour_required, neighbour_capacity, worst_neighbour_required, neighbour_growths;
  double skin, worst_displacement, worst_skin_ratio;
  int32_t skin_violations;
  int64_t steps_with_stale_list;
  int32_t rebuild_interval, requested_rebuild_interval, rebuild_shrinks, rebuild_growths;
  double worst_skin_usage;
  int32_t adaptive_rebuild;
  double volume;
  int32_t barostat_attempts, barostat_accepted, barostat_refused, barostat_screened,
      barostat_exact_evaluations;
  double volume_scale;
  double constraint_tolerance, requested_tolerance, tolerance_floor;
  int32_t cell_counts[3];
  int32_t pme_grid[3];
  double pme_alpha;
  int32_t pme_order;
  int32_t cluster_count, settle_count;
  int64_t device_bytes;
  int64_t list_builds;       /* neighbour-list builds so far (every system of a handle builds together) */
  int32_t rebuild_on_demand; /* the option in effect */
  int32_t pair_list;         /* the neighbour structure in effect (rmd_options.pair_list) */
} rmd_diagnostics_report;

/* Fills `options` with the reference's defaults. */
void rmd_default_options(rmd_options *options);

/* The cell plan, skin and PME parameters of one system, computed on the host with no device
 * work (callable without a GPU), exactly as rmd_create plans each system: skinFor
 * (shared/topology/cells.js:67-91) unless options->skin is given, planCellList
 * (cells.js:101-171) and pmeParameters (shared/pme/parameters.js:227-252). These are the
 * numbers GpuSimulation exposes as plan.counts, pme.grid and pme.alpha
 * (web/app.js:1140-1142). */
typedef struct {
  double skin, cutoff, list_cutoff;   /* nm */
  int32_t counts[3];                  /* cells per axis */
  int32_t cell_count;
  int32_t stencil_cells;              /* cells of the deduplicated stencil (axisOffsets) */
  double estimated_neighbours;        /* density x (4/3) pi list_cutoff^3 */
  int32_t max_neighbours;             /* planCellList's maxNeighbours */
  int32_t capacity;                   /* entries a neighbour row holds: maxNeighbours rounded up to a
                                         multiple of 4, so rows start on 16-byte boundaries */
  double mean_occupancy;              /* atoms per cell */
  double alpha;                       /* Ewald splitting, 1/nm */
  int32_t grid[3];
  int32_t order;
} rmd_plan;
rmd_status rmd_plan_system(const rmd_system *system, const rmd_options *options, rmd_plan *out);

/* grownPlan(plan, required) — cells.js:282-288: the row capacity after a build that needed
 * `required` entries a row: max(capacity + 32, ceil(1.25 required)), rounded up to a
 * multiple of 4. The engine grows its lists by this rule. */
int32_t rmd_grown_capacity(int32_t capacity, int32_t required);

/* new GpuSimulation(device, system, options) — simulation.js:83-190 */
rmd_status rmd_create(const rmd_system *system, const rmd_options *options, rmd_sim **out);

/* A batch of independent systems of uneven size advanced together: every kernel launch
 * covers all of them, and a block of steps is one CUDA graph. No reference counterpart
 * (the reference runs one GpuSimulation per system); every other call takes a
 * `system_index` into it through the *_at variants below. */
rmd_status rmd_create_batch(int32_t count, const rmd_system *systems, const rmd_options *options,
                            rmd_sim **out);
int32_t rmd_system_count(const rmd_sim *sim);

/* setState(positions, velocities, {step, suppliedNoise}) — simulation.js:357-369.
 * velocities may be NULL (zero). Applies to system 0. */
rmd_status rmd_set_state(rmd_sim *sim, const double *positions, const double *velocities,
                         int64_t step, int32_t supplied_noise);
rmd_status rmd_set_state_at(rmd_sim *sim, int32_t system_index, const double *positions,
                            const double *velocities, int64_t step, int32_t supplied_noise);

/* setNoise(noise) — simulation.js:371; f32 [3N] standard normals for the thermostat. */
rmd_status rmd_set_noise(rmd_sim *sim, const float *noise);
rmd_status rmd_set_noise_at(rmd_sim *sim, int32_t system_index, const float *noise);

/* initialise() — simulation.js:412-443: one force evaluation with a fresh neighbour list,
 * growing the list capacity if the measured requirement exceeds it. All systems. */
rmd_status rmd_initialise(rmd_sim *sim);

/* run(count, {blockSize, stopSignal}) — simulation.js:456-527. All systems advance
 * `count` steps in blocks of `block_size` (<= 0: the rebuild interval). `stop_flag`, if
 * not NULL, is polled between blocks (a nonzero value stops with RMD_ERR_STOPPED).
 * `step_out` (may be NULL) receives system 0's step afterwards. */
rmd_status rmd_run(rmd_sim *sim, int64_t count, int32_t block_size, const volatile int32_t *stop_flag,
                   int64_t *step_out);

/* minimise({maxIterations, forceTolerance, maxStep, maxDisplacement}) — simulation.js:880-979 */
rmd_status rmd_minimise(rmd_sim *sim, int32_t max_iterations, double force_tolerance,
                        double max_step, double max_displacement, rmd_minimise_result *out);

/* attemptVolumeChange() — simulation.js:995-1070. One Monte Carlo volume move on every
 * system of the handle; `out` describes system 0. */
rmd_status rmd_attempt_volume_change(rmd_sim *sim, rmd_volume_move *out);
rmd_status rmd_last_volume_move_at(rmd_sim *sim, int32_t system_index, rmd_volume_move *out);

/* scaleVolume(s) — simulation.js:801-811: scale molecular centroids and the box of
 * system 0 by a length factor and return the potential energy there. */
rmd_status rmd_scale_volume(rmd_sim *sim, double length_scale, double *potential_out);

/* energy() — simulation.js:1073-1230 */
rmd_status rmd_energy(rmd_sim *sim, rmd_energy_report *out);
rmd_status rmd_energy_at(rmd_sim *sim, int32_t system_index, rmd_energy_report *out);

/* readPositions() — simulation.js:1239 (f32 [3N]) */
rmd_status rmd_read_positions(rmd_sim *sim, float *positions);

/* readState() — simulation.js:1244-1261. Any output pointer may be NULL. */
rmd_status rmd_read_state(rmd_sim *sim, float *positions, float *velocities, float *forces,
                          double box_vectors[9], double *volume);
rmd_status rmd_read_state_at(rmd_sim *sim, int32_t system_index, float *positions,
                             float *velocities, float *forces, double box_vectors[9],
                             double *volume);

/* diagnostics() — simulation.js:1264-1334 */
rmd_status rmd_diagnostics(rmd_sim *sim, rmd_diagnostics_report *out);
rmd_status rmd_diagnostics_at(rmd_sim *sim, int32_t system_index, rmd_diagnostics_report *out);

/* release() — simulation.js:1336-1340 */
void rmd_destroy(rmd_sim *sim);

/* The message of the last failed call on `sim` (or of the last failed create when NULL). */
const char *rmd_last_error(const rmd_sim *sim);

/* --- Inspection entry points used by the parity tests (no reference counterpart; they
 * expose the device's index structures and the grid so they can be compared with the
 * reference's own intermediate buffers: cellStart/cellAtoms, neighbours, the spread grid). */

/* The cell list of system `system_index` after the last rebuild: counts[3], cell_start
 * [cells+1] and cell_atoms [N] (local atom indices). Pass NULL to query sizes only. */
rmd_status rmd_debug_cells(rmd_sim *sim, int32_t system_index, int32_t counts[3],
                           int32_t *cell_start, int32_t *cell_atoms);
/* The neighbour list: capacity, then per-atom count [N] and rows [N*capacity]. */
rmd_status rmd_debug_neighbours(rmd_sim *sim, int32_t system_index, int32_t *capacity,
                                int32_t *counts, int32_t *rows, int32_t *required);
/* Evaluate forces and energies at the current positions, with a fresh list, and return
 * the per-term breakdown (same fields as rmd_energy) and forces (f64 from fixed point). */
rmd_status rmd_debug_evaluate(rmd_sim *sim, int32_t system_index, rmd_energy_report *energy,
                              double *forces);
/* Forces of one term alone at the current positions and list: 0 direct space with the
 * exceptions, 1 bonded and restraints, 2 PME reciprocal space. */
rmd_status rmd_debug_force_term(rmd_sim *sim, int32_t system_index, int32_t term, double *forces);
/* The group-pair rows (pair_list 0 or 2) of one system, mapped to the system's own atom
 * indices: the number of group slots and the row capacity (call with the arrays NULL for
 * these), then per group slot its GROUP_ATOMS (4) atoms (-1 past the end of a short group or
 * for an unused slot), its row length, and per entry [groups x capacity] the partner atom, the
 * lattice image code (ka+1)*9+(kb+1)*3+(kc+1) of the partner's image (d = x_i - x_j - S) and
 * the 4-bit mask of group atoms that skip the entry. For parity tests. */
rmd_status rmd_debug_group_rows(rmd_sim *sim, int32_t system_index, int32_t *groups, int32_t *capacity,
                                int32_t *atoms, int32_t *counts, int32_t *partners, int32_t *codes,
                                int32_t *masks);

/* Copy a work buffer: 0 the real grid of the last evaluation after the inverse transform
 * (K^3 doubles), 1 its half spectrum (2*Kx*Ky*(Kz/2+1) doubles), 2 the positions the current
 * neighbour list was built from (3N doubles, the f32 values exactly; the displacement
 * check's origin, simulation.js:380-386). */
rmd_status rmd_debug_read(rmd_sim *sim, int32_t system_index, int32_t which, double *out);
/* The real spread charge grid (K^3, z fastest) of the last evaluation. */
rmd_status rmd_debug_charge_grid(rmd_sim *sim, int32_t system_index, double *grid);
/* A forward+inverse 3D transform check: runs the engine's R2C/C2R FFT on `data`
 * (real K^3) and returns the unnormalised round trip and the forward half spectrum
 * ([Kx*Ky*(Kz/2+1)] complex, interleaved) of system `system_index`'s grid size. */
rmd_status rmd_debug_fft(rmd_sim *sim, int32_t system_index, const double *data,
                         double *half_spectrum, double *round_trip);

/* How the reciprocal-space FFT transforms the y and x axes of an nx x ny grid plane: 1 = the
 * fused y-x-convolve-x-y pass with one thread block a kz plane, 4 = the same pass with a
 * 4-block thread-block cluster a plane, 0 = separate y and x passes. A host-side rule that
 * depends on the grid alone (no device call); no reference counterpart. */
int32_t rmd_debug_plane_pass(int32_t nx, int32_t ny);

/* The thermostat's counter-based draws on the device for atoms [atom0, atom0 + count) at
 * `step`, through the device functions the integrator calls: uniformAt(seed, atom, step, c)
 * for c = 0..3 (shared/random.js:59) into uniforms[4 count], and gaussianTriple
 * (random.js:66-87) into normals[3 count]. Host buffers; for parity tests. */
rmd_status rmd_debug_draws(uint32_t seed, uint32_t atom0, int32_t count, uint32_t step, float *uniforms,
                           float *normals);
/* Average device time of one launch of a kernel group on the engine's own stream, by CUDA
 * events over `reps` back-to-back launches: 0 nonbonded (no energy), 1 the PME kernels
 * (five to seven, by grid), 2 the fused integrator, 3 bonded, 4 the list-rebuild kernels,
 * 5 nonbonded with energies. Positions and velocities are put back afterwards and the forces
 * re-evaluated, so the simulation continues from where it was. For roofline measurement;
 * no reference counterpart. */
rmd_status rmd_debug_time_kernel(rmd_sim *sim, int32_t which, int32_t reps, double *ms_per_launch);
/* run() with every block's CUDA graph bracketed by CUDA events on the engine's stream;
 * `device_ms` receives the summed device time of the blocks (host bookkeeping between
 * blocks excluded). With `flush_l2`, a 256 MB buffer is written before each block, outside
 * the timed interval, so no block starts with the previous one's data in L2. */
rmd_status rmd_bench_run(rmd_sim *sim, int64_t count, int32_t block_size, int32_t flush_l2,
                         double *device_ms);
/* Kernels this handle has launched so far (graph replays included). */
int64_t rmd_debug_kernel_launches(const rmd_sim *sim);
/* The learned barostat's surrogate for system `system_index` (no reference counterpart). */
typedef struct {
  int64_t samples;             /* exact (inputs, energy change) pairs seen */
  int64_t train_steps;         /* Adam steps taken */
  double loss;                 /* running mean training loss (targets in kT / sqrt(N_mol)) */
  double prediction_error_kT;  /* running mean |surrogate weight - exact weight| / kT */
  int32_t screening;           /* 1 once the warm-up is over and stage 1 screens moves */
  int64_t attempts, exact_evaluations, screened, accepted;
  int64_t exact_passes, skipped_passes; /* batch-wide: moves that ran / skipped the exact evaluation */
} rmd_surrogate_report;
rmd_status rmd_surrogate_report_at(rmd_sim *sim, int32_t system_index, rmd_surrogate_report *out);
/* The surrogate's FP32 master parameters (4801 floats: W1[64][8], b1[64], W2[64][64], b2[64],
 * W3[64], b3), e.g. to check its predictions on the CPU. */
rmd_status rmd_surrogate_weights(rmd_sim *sim, int32_t system_index, float *params);
/* The surrogate's device forward pass and its mean-squared-error gradient on given data, for
 * any parameters (host arrays; count <= 64 samples of 8 inputs). The weights go through BF16
 * exactly as in training. `outputs` or `grads` may be NULL. */
rmd_status rmd_surrogate_evaluate(const float *params, const float *inputs, const float *targets, int32_t count,
                                  float *outputs, float *grads, double *loss);

/* Kernel launch shapes in use: shapes = {atoms per neighbour-search warp, lanes per atom in
 * the pair loop, atoms per PME spreading block}. When the options left a shape at 0,
 * initialise() chose it by timing every candidate (the engine's autotuner); tune_ms (may be
 * NULL) receives those times in ms per launch, in the order group 4/8/16, lanes 8/16/32
 * (32/64/128 on group-pair rows), spreading 4/8/16, with -1 for shapes that were not tuned. No reference counterpart: the
 * reference's WGSL kernels have fixed workgroup sizes. */
rmd_status rmd_kernel_shapes(const rmd_sim *sim, int32_t shapes[3], double tune_ms[9]);
/* Set launch shapes by hand (0 keeps the current one). Results do not depend on them, except
 * the pair loop's lanes under per-lane f32 accumulation. */
rmd_status rmd_set_kernel_shapes(rmd_sim *sim, int32_t group_atoms, int32_t nonbonded_lanes,
                                 int32_t spread_atoms);
/* The nonbonded kernel's shape, the autotuner's knobs: lanes per atom (8, 16 or 32) and
 * per-pair fixed-point (1) or per-lane f32 (0) force accumulation. */
rmd_status rmd_debug_set_nonbonded(rmd_sim *sim, int32_t lanes, int32_t pair_fixed);

/* ---- On-device trajectory output (shared/traj/imaging.js, dcd.js, rst7.js). The page feeds
 * readPositions() into these writers on the host; here the device images and packs the frame
 * from its own position buffer and the caller receives finished bytes. */

/* imageMolecules (shared/traj/imaging.js:39-91) of the system's current positions: every
 * molecule translated by whole lattice vectors (c, then b, then a) so that its centroid lies in
 * the cell, as FP64 nm, 3 per atom. */
rmd_status rmd_image_molecules_at(rmd_sim *sim, int32_t system_index, double *positions_out);

/* Bytes of one DCD frame (shared/traj/dcd.js:130-160): the 56-byte cell record when
 * `periodic`, then the x, y and z records of 4 * atom_count + 8 bytes each. */
int64_t rmd_dcd_frame_bytes(int32_t atom_count, int32_t periodic);

/* DcdWriter.appendFrame (shared/traj/dcd.js:96-161) from the device: the frame's bytes,
 * imaged by molecule when `image` (the writer's `molecules` option) and carrying the live
 * box's cell record when `periodic`. A non-finite coordinate refuses the frame with
 * RMD_ERR_NON_FINITE (dcd.js:112-128) and writes nothing. */
rmd_status rmd_dcd_frame_at(rmd_sim *sim, int32_t system_index, int32_t periodic, int32_t image,
                            uint8_t *frame_out);

/* The 276-byte header DcdWriter.finish writes (shared/traj/dcd.js:175-199): `created` is the
 * second title line (the reference writes "Created <ISO time>"); NULL leaves it empty. Needs no
 * simulation and no GPU. */
rmd_status rmd_dcd_header(int32_t atom_count, int32_t frames, int32_t first_step, int32_t interval,
                          double timestep, int32_t periodic, const char *title, const char *created,
                          uint8_t header_out[276]);

/* writeRestart (shared/traj/rst7.js:63-101) of the system's device state: the title line, the
 * atom count and `time` (ps), positions in angstroms, velocities in angstroms per AMBER time
 * unit when `velocities`, and the live box as lengths and angles when `box`, every value as
 * ECMAScript's toFixed(7) in 12 columns, six to a line. `out` NULL: only `*bytes` is set. A
 * non-finite value gives RMD_ERR_NON_FINITE and one wider than 12 columns RMD_ERR_INVALID,
 * whichever comes first in the file, and nothing is written. */
rmd_status rmd_restart_at(rmd_sim *sim, int32_t system_index, const char *title, double time,
                          int32_t velocities, int32_t box, char *out, int64_t capacity, int64_t *bytes);

/* ---- Headless structure rendering (web/viewer.js): the viewer's sphere-impostor pass
 * (viewer.js:230-308) and cartoon-ribbon pass (viewer.js:83-228) drawn by CUDA into an RGBA8
 * image, row 0 at the top, with no window, swapchain or graphics API. */

/* The viewer's camera uniform (viewer.js:683-692): view-projection (column-major), the
 * camera's right, up and forward vectors, and the centre the scene is drawn about. */
typedef struct {
  float view_projection[16];
  float right[4], up[4], forward[4], centre[4];
} rmd_camera;

/* StructureViewer.draw() over the system's own device positions: `styles` holds four floats
 * an atom (colour rgb, radius in nm; 0 hides the atom, viewer.js:440-462), `guides` twelve a
 * guide and `segments` four guide indices a segment as buildRibbon returns them
 * (shared/analysis/ribbon.js:110-231). `rgba` receives width * height * 4 bytes. */
rmd_status rmd_render_at(rmd_sim *sim, int32_t system_index, const rmd_camera *camera, const float *styles,
                         const float *guides, int32_t guide_count, const uint32_t *segments,
                         int32_t segment_count, int32_t draw_spheres, int32_t draw_ribbon, int32_t width,
                         int32_t height, uint8_t *rgba);
/* The same from host coordinates (3 floats an atom, nm): StructureViewer.upload() + draw(). */
rmd_status rmd_render_positions(const float *positions, int32_t atom_count, const rmd_camera *camera,
                                const float *styles, const float *guides, int32_t guide_count,
                                const uint32_t *segments, int32_t segment_count, int32_t draw_spheres,
                                int32_t draw_ribbon, int32_t width, int32_t height, uint8_t *rgba);

/* Allocation-free PME charge spreading, for callers that cannot call cudaMalloc: code
 * recording into its own CUDA graph during stream capture, hosts whose device memory all
 * comes from their own arena, and latency-bound callers that cannot take cudaMalloc's
 * implicit synchronisation. This entry point has no counterpart in the reference.
 * `posq` is a device array of float4 (x, y, z in nm, charge in e) for `atom_count` atoms;
 * `grid_out` a device array of grid[0]*grid[1]*grid[2] doubles (z fastest) that receives
 * the spread charge, exactly as the engine's spreading computes it (B-spline `order` 4 or 5,
 * 64-bit fixed-point accumulation). The fixed-point grid lives in a static device array of
 * at most 64^3 points (2 MiB); larger grids return RMD_ERR_INVALID. Work is queued on
 * `stream` (NULL: the legacy default stream) and is complete when the stream is. The
 * array is shared by all calls: calls that overlap on the GPU race. The first call on a
 * device resolves the array's device address (cudaGetSymbolAddress) and loads the kernels
 * it launches; it must come before any stream capture. The resolved address is not valid
 * after cudaDeviceReset on that device. Sizes are checked before anything is launched; an
 * error already pending from earlier work returns RMD_ERR_CUDA before anything is launched. */
rmd_status rmd_spread_charges_noalloc(const void *posq, int32_t atom_count, const double box_vectors[9],
                                      const int32_t grid[3], int32_t order, double *grid_out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* RMD_H */
