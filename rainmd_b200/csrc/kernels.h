// Launch interface between the host engine (engine.cu) and the kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace rmd {

// One FFT axis of one system: length, Stockham radices and its twiddle table offset.
// Division by a divisor fixed per plan, without a hardware divide: for 1 <= d < 2^31 and
// 0 <= x < 2^31, x / d = (umulhi(x, magic) + x) >> shift with shift = ceil(log2 d) and
// magic = floor(2^32 (2^shift - d) / d) + 1 (T. Granlund and P. L. Montgomery, "Division by
// invariant integers using multiplication", PLDI 1994; the sum cannot overflow since
// umulhi(x, magic) < x < 2^31).
struct FastDiv {
  uint32_t magic, shift;
};
struct FftAxis {
  int n;
  int nstages;
  int radix[12];
  int tw_base;
  FastDiv per_line[12];  // stage s: n / radix[s] butterflies a line
  FastDiv span[12];      // stage s: the product of the earlier radices
  FastDiv n_div, half_div;  // n and n / 2 + 1
};
struct FftPlan {
  FftAxis axis[3];
};
// A block's share of an FFT pass: lines [first, first+count) of system `sys`; `fixed` is
// the other fixed index (x for the y pass, y for the x pass).
struct FftTask {
  int sys, fixed, first, count;
};

// Integrator parameters per system (integrate.js:39-63 `Integrator`).
struct DevInteg {
  float half_step, decay, noise_scale, kT;
  float tolerance;
  uint32_t seed;
  int max_iterations;
  int supplied_noise;
};

// SETTLE geometry of one water (masses and the canonical triangle).
struct DevSettle {
  float m_o, m_h, ra, rb, rc, d_oh, d_hh, pad;
};

enum IntegrateMode {
  INT_OPEN = 1,          // B R A S O R A S
  INT_CLOSE = 2,         // B R (the closing half kick of the previous step)
  INT_OPEN_KINETIC = 4,  // per-atom kinetic energy after the opening part
  INT_CLOSE_KINETIC = 8, // per-atom kinetic energy after the closing part
  INT_CONSTRAIN = 16     // positions only: SHAKE/SETTLE towards saved_posq (minimiser)
};

struct IntegrateArgs {
  int n_units, n_free, n_clusters, n_settle, n_atoms, n_systems;
  const int *free_atoms;
  const int *cl_atom_start, *cl_atoms, *cl_con_start;
  const int2 *cl_con_pair;
  const float *cl_con_dist;
  const int3 *settle_atoms;
  const DevSettle *settle_param;
  const int *sys_of_atom;
  const int *sys_atom_start;
  const DevInteg *integ;
  const long long *step_base;
  int step_offset;
  float4 *posq;
  float4 *vel;
  const unsigned long long *force;
  const float *noise;
  const float4 *origin;
  unsigned *disp;  // [n_systems] since the last rebuild, then [n_systems] since block start
  int *diag;
  double *ke_post, *ke_early;
  const float4 *saved_posq;
  float4 *spos;
  const int *rank;
  const float4 *wrap;
};

struct LaunchCtx {
  int n_atoms, n_systems;
  float4 *posq;
  const int *atom_type;
  const int *sys_of_atom;
  DevSys *sys;
  DevSysD *sysd;
  // lists
  int *cell_of_atom, *cell_count, *cell_start, *cell_atoms, *cell_sys;
  int n_cells_total;
  // neighbour-search groups: per cell the first group (scan of ceil(count / 32), indexed like
  // cell_start), the cell's slots in sub-cell order, and the system of each group slot
  int *cell_gstart, *group_order;
  const int *group_sys;
  int n_groups_total;
  int group_atoms;  // atoms per neighbour-search group: 4, 8, 16 or 32
  const int *rebuild_only;  // per-system flags: rebuild only the flagged systems (null: every system)
  const int *excl_start, *excl_partners;
  int *nbr, *nbr_count, *required;
  float4 *origin;
  // 0: the pair loop walks group-pair rows; 1: per-atom rows; 2: group-pair rows, and every
  // build also writes the per-atom rows (rmd_options.pair_list)
  int pair_list;
  int *gnbr, *gnbr_count;  // group-pair rows and their lengths, per group slot
  int *gfirst, *gsize;     // per group slot: its first position in group_order, its atoms (0: unused)
  int2 *slot_info;         // per slot: LJ type, original index
  int *order_pos;          // per slot: its position in group_order
  float4 *group_box;       // per group slot: bounding box lo, hi of its atoms' wrapped positions
  unsigned long long *e_acc;  // per-atom integer energy sums of the group-pair kernel (3 N)
  bool force_cleared;  // the force array was zeroed since the last evaluation (launch_nonbonded skips its clear)
  // cell-ordered copies written at each rebuild and kept current by the integrator:
  // spos[slot] = position minus the atom's wrap shift (w = charge), the original index,
  // the LJ type; rank[atom] = slot and wrap[atom] = that shift
  float4 *spos;
  int *sorted_orig, *sorted_type, *rank;
  float4 *wrap;
  // nonbonded
  const float2 *lj;
  int lj_entries;  // float2 entries of `lj` (all systems' type tables)
  const int *exc_start, *exc_partner;
  const float4 *exc_param;
  unsigned long long *force;
  double *e_lj, *e_coul, *e_vir;
  // molecules, for the molecular virial correction (energy evaluations only)
  const int *mol_start, *mol_atoms;
  const float *masses;
  double *mol_vir;
  int n_molecules;
  int pair_fixed;  // 1: per-pair fixed-point accumulation (precision form), 0: per-lane f32
  // bonded
  const int2 *bond_atoms;
  const float2 *bond_param;
  int n_bonds;
  const int4 *angle_atoms;
  const float2 *angle_param;
  int n_angles;
  const int4 *tor_atoms;
  const float4 *tor_param;
  int n_tors;
  const int *rest_atom;
  const float4 *rest_param;
  int n_rest;
  double *e_term, *e_term_vir;
  // pme
  int pme_on, pme_order;
  // The reciprocal chain's kernels (on their own branch of the step graph) are launched chained
  // (programmatic dependent launch) when the lists are rebuilt on demand. With the reference's
  // host schedule they are plain launches: measured on one B200 at 23,558 atoms, chaining them
  // took a step from 0.1429 to 0.1380 ms on demand (a build every 6.3 steps) but from 0.161 to
  // 0.182 ms with a build every 4 steps (the early-scheduled plane clusters slow the concurrent
  // list rebuild).
  int chain_pme;
  int spread_atoms;  // atoms per spreading block: 4, 8 or 16
  unsigned long long *fixed_grid;
  float2 *half;
  float *real_grid;
  const float *moduli;
  const float2 *twiddles;
  const FftPlan *fft_plans;
  // z tasks cover every system; y and x tasks the systems on the separate passes; plane tasks
  // (one per kz plane) the systems whose planes a block transforms alone, cluster tasks (one
  // per kz plane) those whose planes a cluster of PLANE_CLUSTER blocks shares; *_all cover
  // every system (the debug transforms)
  const FftTask *tasks_z, *tasks_y, *tasks_x, *tasks_plane, *tasks_cluster, *tasks_y_all, *tasks_x_all;
  int n_tasks_z, n_tasks_y, n_tasks_x, n_tasks_plane, n_tasks_cluster, n_tasks_y_all, n_tasks_x_all;
  int plane_stride;  // complex values per plane buffer (the largest plane among the one-block systems)
  int cluster_rows, cluster_cols;  // complex values per row / column buffer of a cluster block
  // energy partials: one per x task, then one per plane task, then PLANE_CLUSTER per cluster task
  double *e_pme, *e_pme_vir;
};

void launch_rebuild(const LaunchCtx &c, cudaStream_t stream);
int rebuild_launches(const LaunchCtx &c);  // kernels launch_rebuild issues (without the reset)
// Rebuild on demand (lists.cu): flag the systems that have moved past half their skin since
// their last build and set `handle` (an IF node's condition) when any has; and the reset every
// rebuild starts with (of the flagged systems, or of all when `only` is null).
// `clear_force` (if not null): the 3 N-word force array, zeroed by the same launch.
void launch_rebuild_decide(cudaGraphConditionalHandle handle, const unsigned *disp, const float *allow,
                           const DevSys *sys, int S, int *stale, unsigned long long *rebuilds,
                           unsigned long long *clear_force, int n_atoms, cudaStream_t stream);
void launch_rebuild_reset(int *required, int *required_max, unsigned *disp, float *allow, int *rebuilt, int S,
                          unsigned long long *builds, const int *only, cudaStream_t stream);
// group slots a system needs for a given group size (its search groups never exceed this)
int neighbour_group_slots(int atoms, int cells, int group_atoms);
void launch_nonbonded(const LaunchCtx &c, bool energy, int lanes, cudaStream_t stream);
int nonbonded_launches(const LaunchCtx &c, bool energy);  // kernels launch_nonbonded issues
void launch_bonded(const LaunchCtx &c, bool energy, cudaStream_t stream);
void launch_molecular_virial(const LaunchCtx &c, cudaStream_t stream);
void launch_pme(const LaunchCtx &c, bool energy, cudaStream_t stream);
// launch_pme split in two: the grid chain (spread .. inverse transform) and the force gather
void launch_pme_grid(const LaunchCtx &c, bool energy, cudaStream_t stream);
void launch_pme_gather(const LaunchCtx &c, cudaStream_t stream);
int pme_launches(const LaunchCtx &c);  // kernels launch_pme issues
// The fused y-x-convolve-x-y pass over kz planes (pme.cu). fft_plane_split gives how a system's
// nx x ny planes are transformed: 1 = one block a plane, PLANE_CLUSTER = a thread-block cluster
// of that many blocks a plane (rows and columns split between them, exchanged through
// distributed shared memory), 0 = the separate y and x passes.
constexpr long long FFT_PLANE_SMEM_MAX = 200 * 1024;
constexpr int PLANE_CLUSTER = 4;
int fft_plane_split(int nx, int ny);
// complex values per shared buffer for a split: the whole padded plane for 1; for a cluster,
// a block's rows (rows_per x (ny + 1)) and its columns (cols_per x (nx + 1))
void fft_plane_buffers(int nx, int ny, int split, int *rows, int *cols);
cudaError_t fft_plane_prepare();
void launch_fft_forward(const LaunchCtx &c, cudaStream_t stream);
void launch_spread_only(const LaunchCtx &c, cudaStream_t stream);
void launch_fft_inverse(const LaunchCtx &c, cudaStream_t stream);
void launch_integrate(const IntegrateArgs &a, int mode, cudaStream_t stream);
void launch_draws(uint32_t seed, uint32_t atom0, int count, uint32_t step, float *uniforms, float *normals,
                  cudaStream_t stream);

// Energy segments reduced per system (reduce.cu). Each segment is [start, end) of one
// per-item FP64 array; the result lands in energies[sys * N_ENERGY + term].
enum EnergyTerm {
  E_BOND = 0, E_ANGLE, E_TORSION, E_LJ, E_COUL_DIRECT, E_RECIP, E_RESTRAINT, E_KINETIC,
  E_KINETIC_EARLY, E_SELF, E_NET, E_DISPERSION, E_POTENTIAL,
  // not energies: the atomic virial sum F.r of the pair, exception and bonded terms; the
  // reciprocal-space sum sum_k E_k (1 + pi^2 m^2 / alpha^2); sum_i F_i.(r_i - R_mol(i)) over
  // atoms with R the molecule's centre of mass; and from them dU/dlnV when molecules are
  // scaled rigidly about their centres (the barostat's move)
  E_VIR_SR, E_VIR_REC, E_VIR_MOL, E_DUDLNV, N_ENERGY
};
struct Segment {
  int sys, term;
  const double *data;
  long long start, end;
  const double *data2;  // optional second array summed over the same range (LJ: nonbonded)
};
void launch_energy_reduce(const Segment *segments, int n_segments, double *seg_out,
                          double *energies, const DevSysD *sysd, int n_systems, cudaStream_t stream);

// Barostat and utility kernels (reduce.cu).
struct BaroArgs {
  int n_systems, n_atoms, n_molecules;
  float4 *posq;
  float4 *saved_posq;
  unsigned long long *force, *saved_force;
  const int *mol_start, *mol_atoms, *mol_of_atom;
  const int *sys_of_atom;
  float4 *centroid;  // per molecule
  DevSys *sys;
  DevSysD *sysd;
  double *baro;      // per system BARO_* slots
  double *energies;  // per system N_ENERGY
  double *saved_energies;
  const float *masses;
  unsigned *disp;    // per system: largest squared displacement since the lists were built (f32 bits)
  // A move evaluated on the current lists (keep_lists: the step graphs with lists rebuilt on
  // demand): the atoms' wrap shifts and displacement origins are scaled with them (saved first),
  // and `allow` grows by the most the move can change a pair distance by, per atom (saved
  // first); `rebuilt` tells whether the trial evaluation rebuilt the lists anyway.
  int keep_lists;
  float4 *wrap, *saved_wrap, *origin, *saved_origin, *spos;
  const int *rank;
  float *allow, *saved_allow;
  int *rebuilt;
  unsigned *spread_bits;  // per system: largest distance of an atom from its molecule's centroid (f32 bits)
};
enum BaroSlot {
  B_ACTIVE = 0, B_PRESSURE, B_KT, B_NMOL, B_SEED, B_ATTEMPTS, B_ACCEPTED, B_WINDOW_ATT, B_WINDOW_ACC,
  B_SCALE, B_DV, B_LSCALE, B_OLD_E, B_NEW_E, B_WEIGHT, B_ACCEPT, B_REFUSED, B_REFUSALS,
  B_OLD_VOL, B_SCREENED, B_SCREENED_TOTAL, B_EXACT_EVALS,
  // learned barostat (surrogate.cu): on/off, moves before screening starts, the reference
  // volume of the inputs, degrees of freedom, the last four exact energy changes, the
  // surrogate's weights for the forward and reverse move, dU/dlnV of the move's start,
  // replay fill, training steps, running loss and prediction error, and the move's inputs
  B_LEARNED, B_WARMUP, B_VOL_REF, B_DOF, B_HIST0, B_HIST1, B_HIST2, B_HIST3, B_PRED, B_PRED_REV,
  B_DUDLNV, B_REPLAY_N, B_TRAIN_STEPS, B_LOSS, B_PRED_ERR, B_SCREENING, B_FEATURE0,
  N_BARO = B_FEATURE0 + 8 + 4
};
void launch_baro_propose(const BaroArgs &a, cudaStream_t stream);
// Learned barostat (surrogate.cu). The MLP: 8 inputs, two tanh layers of 64, one output;
// FP32 master weights with Adam moments, BF16 copies for every forward pass.
constexpr int MLP_IN = 8, MLP_H = 64;
constexpr int MLP_W1 = 0, MLP_B1 = MLP_W1 + MLP_H * MLP_IN, MLP_W2 = MLP_B1 + MLP_H,
              MLP_B2 = MLP_W2 + MLP_H * MLP_H, MLP_W3 = MLP_B2 + MLP_H, MLP_B3 = MLP_W3 + MLP_H,
              MLP_PARAMS = MLP_B3 + 1, MLP_STRIDE = 4864;
constexpr int MLP_REPLAY = 4096;  // (inputs, target) samples kept per system
constexpr int MLP_BATCH = 64;     // training minibatch
struct SurrogateArgs {
  int n_systems;
  float *master, *adam_m, *adam_v;  // [system][MLP_STRIDE]
  unsigned short *wbf;              // BF16 bits of the master weights, [system][MLP_STRIDE]
  float *replay;                    // [system][MLP_REPLAY][MLP_IN + 1]
  double *baro;
  double *energies;
  DevSysD *sysd;
  float lr;
  int steps;                        // gradient steps per training launch
};
void launch_surrogate_stage1(const BaroArgs &a, const SurrogateArgs &m, cudaStream_t stream);
void launch_surrogate_train(const SurrogateArgs &m, cudaStream_t stream);
// the stage-1 weight of the reverse move around the trial state (after its exact evaluation)
void launch_surrogate_reverse(const BaroArgs &a, const SurrogateArgs &m, cudaStream_t stream);
// standalone forward and gradient of one network on given data (for the gradient check)
void surrogate_predict(const float *params, const float *x, int count, float *out, cudaStream_t stream);
void surrogate_gradients(const float *params, const float *x, const float *target, int count,
                         float *grads, float *loss, cudaStream_t stream);
void launch_baro_scale(const BaroArgs &a, cudaStream_t stream);
void launch_baro_allow(const BaroArgs &a, cudaStream_t stream);  // keep_lists moves: grow `allow`
void launch_baro_decide(const BaroArgs &a, cudaStream_t stream);
void launch_baro_restore(const BaroArgs &a, cudaStream_t stream);
void launch_scale_fixed(const BaroArgs &a, const double *scales, cudaStream_t stream);
void launch_update_box(DevSys *sys, DevSysD *sysd, int n_systems, cudaStream_t stream);
void launch_advance_steps(long long *step_base, int n_systems, int count, cudaStream_t stream);

// Minimiser helpers (minimise.cu): largest force magnitude per system (as float bits), and
// x += scale_s * F capped at max_disp per atom (integrate.js:589-666).
void launch_max_force(const unsigned long long *force, const int *sys_of_atom, int n_atoms,
                      unsigned *out_bits, cudaStream_t stream);
void launch_displace(float4 *posq, const unsigned long long *force, const int *sys_of_atom, int n_atoms,
                     const float *scale, float max_disp, cudaStream_t stream);

// On-device trajectory output (traj.cu): one system's atoms and molecules, the per-molecule
// translations, the output staging buffer and two error slots (first non-finite and first
// too-wide value; INT_MAX when none).
struct TrajArgs {
  const float4 *posq, *vel;
  const int *mol_start, *mol_atoms, *mol_of_atom;
  const DevSysD *sysd;
  int sys, atom_start, atom_count, mol_first, mol_count, image;
  double3 *shift;
  unsigned char *out;
  int *status;
};
struct Rst7Box {
  double values[6];      // lengths in angstroms, angles in degrees
  double velocity_unit;  // nm/ps per angstrom per AMBER time unit
};
void launch_traj_shifts(const TrajArgs &t, cudaStream_t stream);
void launch_traj_image(const TrajArgs &t, double *out, cudaStream_t stream);
void launch_dcd_pack(const TrajArgs &t, int periodic, cudaStream_t stream);
void launch_rst7_format(const TrajArgs &t, long long header, int velocities, int box, const Rst7Box &b,
                        cudaStream_t stream);
// host forms of the same arithmetic (the header line, the box line)
int fixed7_text(double x, char field[12]);
long long rst7_block_size(long long values);
void dcd_cell_host(const double *box, double cell[6]);
double script_hypot(double x, double y, double z);

// Headless structure rendering (raster.cu): the viewer's 36-float camera uniform, and one
// frame's inputs, scratch and output.
struct RenderCamera {
  float vp[16];  // view-projection, column-major
  float right[4], up[4], forward[4], centre[4];
};
struct RenderArgs {
  RenderCamera camera;
  const float4 *positions;  // xyz in nm (w unused)
  const float4 *styles;     // colour rgb, radius (0 hides the atom)
  int atom_count;
  const float *guides;      // 12 floats a guide: position, half width, side, half thickness, colour, pad
  const uint4 *segments;    // four control guides a segment
  int segment_count;
  int draw_spheres, draw_ribbon, width, height;
  float4 *sphere_corners;   // 4 per atom
  float *ribbon_vertices;   // 12 floats per vertex, 24 * 8 vertices per segment
  unsigned long long *keys; // per pixel: depth bits << 32 | primitive order
  uchar4 *image;            // RGBA8, row 0 at the top
};
void launch_render(const RenderArgs &a, cudaStream_t stream);

// Line-search state of one system, owned by the device while the minimiser runs: every
// accept/reject decision is taken by min_decide, so a trial needs no host round trip.
struct MinState {
  double potential;  // energy of the accepted structure
  double step;       // line-search step (nm^2 mol/kJ scale of the largest force)
  float worst;       // largest force of the accepted structure (kJ/mol/nm)
  int iterations, rejected, attempt;
  int open;       // an iteration is under way (its start structure is in saved_posq/saved_force)
  int done, stalled;
  int trial;      // this trial displaced the system
  int save;       // this trial opened an iteration: copy the structure aside first
  int reject_now; // this trial was rejected: put the accepted structure back
  int overflow;   // a trial's neighbour list overflowed; paused until the host grows the list
  int need;       // largest neighbour requirement seen in an overflowing trial
};
constexpr int MIN_ATTEMPTS = 14;  // trials per iteration (simulation.js:880-979)

void launch_min_begin(MinState *st, const unsigned *worst_bits, float *scale, int n_systems, int max_iterations,
                      float force_tolerance, cudaStream_t stream);
void launch_min_save(const MinState *st, const float4 *posq, const unsigned long long *force, float4 *saved_posq,
                     unsigned long long *saved_force, const int *sys_of_atom, int n_atoms, cudaStream_t stream);
void launch_min_decide(MinState *st, const double *energies, const int *required, const DevSys *sys,
                       int n_systems, cudaStream_t stream);
void launch_min_restore(const MinState *st, float4 *posq, unsigned long long *force, const float4 *saved_posq,
                        const unsigned long long *saved_force, const int *sys_of_atom, int n_atoms,
                        cudaStream_t stream);

}  // namespace rmd
