// Host engine and C ABI (include/rmd.h) of the B200 RainMD step engine.
//
// Mirrors RainMD's `class GpuSimulation` (webgpu/simulation.js:82-1341): host set-up of the
// device arrays, step blocks, the adaptive rebuild and skin check, capacity growth, the
// barostat, energy and state readback. The host-side derivations are restated from the
// reference's shared/ modules and cited where they appear. The step itself is a CUDA graph
// per block of steps: one replay launches every kernel of every step of every system.
#include <algorithm>
#include <cstddef>
#include <array>
#include <climits>
#include <cmath>
#include <functional>
#include <map>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <map>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/rmd.h"
#include "common.cuh"
#include "kernels.h"

namespace rmd {

struct Error : std::runtime_error {
  rmd_status code;
  Error(rmd_status c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define CUDA_OK(expr)                                                                       \
  do {                                                                                      \
    cudaError_t e_ = (expr);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      throw ::rmd::Error(RMD_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));        \
  } while (0)

template <class T>
struct DevArray {
  T *p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    release();
    n = count;
    if (count) CUDA_OK(cudaMalloc(&p, sizeof(T) * count));
  }
  void upload(const std::vector<T> &v) {
    alloc(v.size());
    if (!v.empty()) CUDA_OK(cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  }
  void zero() {
    if (n) CUDA_OK(cudaMemset(p, 0, sizeof(T) * n));
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return sizeof(T) * n; }
};

// -------------------------------------------------------------- host-side derivations
static unsigned short bf16_round_bits(float v) {  // round to nearest even (finite inputs)
  uint32_t u;
  memcpy(&u, &v, 4);
  u += 0x7fffu + ((u >> 16) & 1u);
  return (unsigned short)(u >> 16);
}
static double alpha_from_tolerance(double cutoff, double tol) {  // parameters.js:43-49
  return std::sqrt(-std::log(2.0 * tol)) / cutoff;
}
static bool transformable(int v) {  // parameters.js:68-74
  int r = v;
  for (int p : {2, 3, 5})
    while (r % p == 0) r /= p;
  return r == 1;
}
static void bspline_host(double u, int order, double *w) {  // parameters.js:121-149 (weights)
  std::vector<double> dw(order);
  for (int k = 0; k < order; ++k) w[k] = 0;
  w[0] = 1 - u;
  w[1] = u;
  for (int k = 3; k < order; ++k) {
    double div = 1.0 / (k - 1);
    w[k - 1] = div * u * w[k - 2];
    for (int j = 1; j < k - 1; ++j) w[k - j - 1] = div * ((u + j) * w[k - j - 2] + (k - j - u) * w[k - j - 1]);
    w[0] = div * (1 - u) * w[0];
  }
  double div = 1.0 / (order - 1);
  w[order - 1] = div * u * w[order - 2];
  for (int j = 1; j < order - 1; ++j)
    w[order - j - 1] = div * ((u + j) * w[order - j - 2] + (order - j - u) * w[order - j - 1]);
  w[0] = div * (1 - u) * w[0];
}
static std::vector<double> bspline_moduli(int K, int order) {  // parameters.js:164-215
  std::vector<double> w(order), raw(K), out(K);
  bspline_host(0.0, order, w.data());
  for (int m = 0; m < K; ++m) {
    double re = 0, im = 0;
    for (int k = 0; k < order; ++k) {
      double a = 2.0 * M_PI * m * k / K;
      re += w[k] * std::cos(a);
      im += w[k] * std::sin(a);
    }
    raw[m] = re * re + im * im;
  }
  for (int m = 0; m < K; ++m) {
    out[m] = raw[m] < 1e-7 ? 0.5 * (raw[(m - 1 + K) % K] + raw[(m + 1) % K]) : raw[m];
    if (!(out[m] > 0))
      throw Error(RMD_ERR_INVALID, "B-spline modulus " + std::to_string(m) + " of " + std::to_string(K) +
                                       " is still zero after the neighbour substitution: the grid is "
                                       "too small for this interpolation order");
  }
  return out;
}

struct Cluster {
  std::vector<int> atoms;             // global, ascending
  std::vector<std::pair<int, int>> c;  // local index pairs
  std::vector<float> d;
};

// Per-system host state.
struct HostSystem {
  int n = 0, atom_start = 0;
  rmd_options opt{};
  std::vector<double> charges, masses;
  std::vector<int> types;
  int type_count = 0;
  std::vector<double> lj_a, lj_b;
  std::vector<double> box;  // 9
  double cutoff = 1.0, skin = 0.1, list_cutoff = 1.1, alpha = 0;
  int grid[3] = {0, 0, 0}, order = 5;
  int counts[3] = {1, 1, 1};
  int capacity = 32;
  double estimated_neighbours = 0;
  int dof = 0, n_molecules = 0;
  double q2 = 0, qsum = 0, disp_a = 0, disp_b = 0;
  double tolerance = 1e-5, tol_floor = 0, requested_tol = 1e-5;
  double min_constraint = 0;
  std::vector<double> restraint_reference;  // 3 per restrained atom
  std::vector<int> restraint_atoms;
  int64_t step = 0;
  // adaptive rebuild (simulation.js:105-118, 544-623)
  int rebuild_interval = 20, requested_rebuild = 20;
  bool adaptive = true;
  bool on_demand = true;  // the device decides each step (rmd_options.rebuild_on_demand)
  int calm_blocks = 0, rebuild_growths = 0, rebuild_shrinks = 0, skin_violations = 0;
  int64_t steps_with_stale = 0;
  int64_t steps_since_rebuild = 1LL << 40;
  double worst_displacement = 0, worst_skin_ratio = 0, worst_skin_usage = 0;
  int worst_required = 0, neighbour_growths = 0, last_required = 0;
  bool kinetic_sampled_in_step = false;
  int64_t kinetic_sampled_at = -1;
  int n_clusters = 0, n_settle = 0;
  int barostat_interval = 25;
  int64_t steps_since_barostat = 0;
  bool has_pressure = false;
  rmd_volume_move last_move{};
};

static const double LIGHT_ANCHOR_SKIN = 0.40;  // cells.js:67-91

// Neighbour rows hold a multiple of 4 entries so that every row starts on a 16-byte boundary
// (a departure from planCellList's maxNeighbours, which it rounds up, never down).
static int row_capacity(int max_neighbours) { return (max_neighbours + 3) & ~3; }

// grownPlan (cells.js:282-288): past the measured requirement by a quarter, and at least 32
// more than before, as a row capacity.
static int grown_capacity(int capacity, int required) {
  return row_capacity(std::max(capacity + 32, (int)std::ceil(required * 1.25)));
}

// How a force evaluation treats the neighbour lists.
enum RebuildMode { REBUILD_NONE = 0, REBUILD_FORCED = 1, REBUILD_IF_STALE = 2 };

struct Engine {
  std::vector<HostSystem> hs;
  int S = 0, N = 0;
  cudaStream_t stream = nullptr;
  // the reciprocal-space branch of a force evaluation runs on `side`, forked from and joined
  // back to `stream` with events (inside a captured graph these become parallel branches)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_clear = nullptr;
  // the stream a conditional rebuild body is captured on (record_forces)
  cudaStream_t cond = nullptr;
  bool on_demand = true;  // lists rebuilt when the device finds them stale (all systems agree)
  std::string last_error;
  int nb_lanes = 32;
  int group_atoms = 8;   // atoms per neighbour-search warp
  int spread_atoms = 8;  // atoms per PME spreading block
  int pair_fixed = 1;
  int pme_order = 5;
  bool pme_on = true;

  // device arrays
  DevArray<float4> posq, vel, origin, saved_posq;
  DevArray<int> atom_type, sys_of_atom, sys_atom_start;
  DevArray<float> masses, noise;
  DevArray<unsigned long long> force, saved_force;
  DevArray<double> e_lj, e_coul, e_vir, ke_post, ke_early, e_term, e_pme, e_pme_vir;
  DevArray<float2> lj;
  DevArray<int> excl_start, excl_partners, exc_start, exc_partner;
  DevArray<float4> exc_param;
  DevArray<int> cell_of_atom, cell_count, cell_start, cell_atoms, cell_sys;
  int n_cells_total = 0;
  DevArray<int> cell_gstart, group_order, group_sys;
  int n_groups_total = 0;
  DevArray<int> nbr, nbr_count, required, required_max, stale;
  // group-pair rows (pair_list 0 and 2): rows, lengths, first order position and atoms per group
  // slot; per slot its partner record and order position; per-atom integer energy sums
  int pair_list = 1;
  DevArray<int> gnbr, gnbr_count, gfirst, gsize, order_pos;
  DevArray<float4> group_box;
  // volume moves evaluated on the current lists (reduce.cu k_baro_centroid_scale, k_baro_allow)
  DevArray<float4> saved_wrap, saved_origin;
  DevArray<float> list_allow, saved_allow;
  DevArray<int> list_rebuilt;
  DevArray<unsigned> spread_bits;
  DevArray<int2> slot_info;
  DevArray<unsigned long long> e_acc;
  // list builds counted on the device: [0] those an IF node took, [1] all of them
  DevArray<unsigned long long> list_builds;
  unsigned long long conditional_builds_seen = 0;
  DevArray<float4> spos, wrap;
  DevArray<int> sorted_orig, sorted_type, rank;
  DevArray<int2> bond_atoms;
  DevArray<float2> bond_param, angle_param;
  DevArray<int4> angle_atoms, tor_atoms;
  DevArray<float4> tor_param, rest_param;
  DevArray<int> rest_atom;
  int n_bonds = 0, n_angles = 0, n_tors = 0, n_rest = 0;
  std::vector<int> term_start;  // per system: bonds, angles, torsions, restraints offsets (4*S+4)
  DevArray<unsigned long long> fixed_grid;
  DevArray<float2> half, twiddles;
  DevArray<float> real_grid, moduli;
  DevArray<FftPlan> fft_plans;
  DevArray<FftTask> tasks_z, tasks_y, tasks_x, tasks_plane, tasks_cluster, tasks_y_all, tasks_x_all;
  std::vector<long long> recip_lo, recip_hi;  // per system range [lo, hi) of reciprocal energy partials
  int plane_stride = 0, cluster_rows = 0, cluster_cols = 0;
  DevArray<DevSys> sys;
  DevArray<DevSysD> sysd;
  std::vector<DevSys> h_sys;
  std::vector<DevSysD> h_sysd;
  DevArray<DevInteg> integ;
  DevArray<long long> step_base;
  DevArray<unsigned> disp;
  DevArray<int> diag;
  DevArray<double> energies, saved_energies, baro, seg_out, fixed_scales;
  DevArray<Segment> segments;
  int n_segments = 0;
  DevArray<int> free_atoms, cl_atom_start, cl_atoms, cl_con_start;
  DevArray<int2> cl_con_pair;
  DevArray<float> cl_con_dist;
  DevArray<int3> settle_atoms;
  DevArray<DevSettle> settle_param;
  int n_free = 0, n_clusters = 0, n_settle = 0;
  DevArray<int> mol_start, mol_atoms, mol_of_atom;
  // trajectory output (traj.cu): per-molecule translations, a staging buffer, error slots
  DevArray<double3> traj_shift;
  DevArray<unsigned char> traj_out;
  DevArray<int> traj_status;
  TrajArgs traj_args(int s, bool image);  // sizes the scratch; computes the translations when imaging
  DevArray<double> mol_vir, e_term_vir;
  std::vector<int> mol_base;  // first molecule of each system (S + 1)
  int n_molecules_total = 0;
  bool any_pressure = false;
  bool supplied_noise_any = false;
  // true while `energies` holds the potential at the current positions and box because the
  // last step graph ended with an energy-enabled evaluation; a volume move then needs no
  // evaluation of its own first. Every other evaluation or change of state clears it.
  bool energy_fresh = false;

  std::map<std::string, cudaGraphExec_t> graphs;
  std::map<std::string, long long> graph_launches;  // kernels recorded in each graph
  long long recorded = 0;                            // kernels recorded by record_* calls
  long long kernel_launches = 0;                     // kernels launched so far (graphs and direct)

  ~Engine() {
    if (pinned) cudaFreeHost(pinned);
    for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (ev_clear) cudaEventDestroy(ev_clear);
    if (side) cudaStreamDestroy(side);
    if (cond) cudaStreamDestroy(cond);
    if (stream) cudaStreamDestroy(stream);
  }

  // ---------------------------------------------------------------- construction
  void build(int count, const rmd_system *systems, const rmd_options *options);
  static void plan_system(HostSystem &h, const rmd_system &s);
  void upload_all(const std::vector<const rmd_system *> &src);
  void allocate_neighbours();
  LaunchCtx ctx() const;
  IntegrateArgs iargs(int step_offset) const;
  BaroArgs bargs() const;
  // learned barostat (surrogate.cu)
  bool learned = false;
  DevArray<float> mlp_master, mlp_m, mlp_v, mlp_replay;
  DevArray<unsigned short> mlp_wbf;
  int learned_steps = 4;
  float learned_lr = 1e-3f;
  long long exact_passes = 0, skipped_passes = 0;
  SurrogateArgs sargs();
  bool surrogate_stage1();  // true when some system's move needs the exact evaluation
  void surrogate_train();

  // ---------------------------------------------------------------- operations
  // rebuild: REBUILD_NONE, REBUILD_FORCED, or REBUILD_IF_STALE (captured graphs only)
  void record_forces(int rebuild, bool energy);
  void record_conditional_rebuild(const LaunchCtx &c);
  void record_barostat(bool keep_lists);
  void evaluate(bool rebuild, bool energy);
  void set_state(int s, const double *pos, const double *vel, int64_t step, int supplied);
  void initialise();
  // kernel-shape autotuner: which shapes were left to it, and what it measured
  bool tune_group = false, tune_lanes = false, tune_spread = false;
  double tune_ms[9] = {-1, -1, -1, -1, -1, -1, -1, -1, -1};
  bool autotune();  // true when it launched timing work (the force array then holds its sums)
  void drop_graphs();
  int check_capacity();  // returns max required; grows if needed
  bool capacity_grew = false;  // the last check_capacity grew the lists (and rebuilt them, forces only)
  void run(int64_t count, int block, const volatile int32_t *stop);
  void run_block(int n, bool barostat, bool energy_last);
  std::map<std::string, cudaGraphExec_t>::iterator block_graph(int n, bool barostat, bool energy_last);
  // timing hooks for run(): events around each block's graph, optional L2 flush between
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;
  bool timing = false, flush = false;
  double timed_ms = 0.0;
  DevArray<unsigned char> flush_buffer;
  void check_block(int steps);
  void energy(int s, rmd_energy_report *out);
  void sync() { CUDA_OK(cudaStreamSynchronize(stream)); }
  // Page-locked staging for the state copies of setState and readState: every copy of a call
  // is one asynchronous transfer on the engine stream, and the call waits once.
  void *pinned = nullptr;
  size_t pinned_bytes = 0;
  char *staging(size_t bytes) {
    if (bytes > pinned_bytes) {
      if (pinned) CUDA_OK(cudaFreeHost(pinned));
      pinned = nullptr;
      pinned_bytes = 0;
      CUDA_OK(cudaMallocHost(&pinned, bytes));
      pinned_bytes = bytes;
    }
    return static_cast<char *>(pinned);
  }
  void update_box_from_host(int s);
  void attempt_volume_change();
  double scale_volume(int s, double ls);
  std::vector<float> max_forces();
  void minimise(int max_iterations, double force_tolerance, double max_step, double cap,
                rmd_minimise_result *out);
  std::vector<double> read_energies();
};

// ------------------------------------------------------------------------ set-up
void Engine::plan_system(HostSystem &h, const rmd_system &s) {
  const rmd_options &o = h.opt;
  h.n = s.atom_count;
  if (h.n <= 0) throw Error(RMD_ERR_INVALID, "atom_count must be positive");
  if (s.box_vectors == nullptr)
    throw Error(RMD_ERR_INVALID,
                "the device path needs a periodic box: a cell list cannot be built without one "
                "(cells.js:109-115); a non-periodic system uses the all-pairs host path");
  h.box.assign(s.box_vectors, s.box_vectors + 9);
  for (int k : {1, 2, 5})
    if (h.box[k] != 0.0) throw Error(RMD_ERR_INVALID, "box vectors must be reduced upper-triangular (a along x, b in xy)");
  h.cutoff = s.cutoff;
  const double widths[3] = {std::fabs(h.box[0]), std::fabs(h.box[4]), std::fabs(h.box[8])};
  const double smallest = std::min(widths[0], std::min(widths[1], widths[2]));
  if (!(h.cutoff > 0) || h.cutoff > 0.5 * smallest) {  // system.js:70-89
    char msg[256];
    snprintf(msg, sizeof msg, "a %g nm cutoff does not fit in a box whose smallest width is %.4f nm: "
             "the cutoff must be at most half of it", h.cutoff, smallest);
    throw Error(RMD_ERR_INVALID, msg);
  }
  h.charges.assign(s.charges, s.charges + h.n);
  h.masses.assign(s.masses, s.masses + h.n);
  h.types.assign(s.atom_types, s.atom_types + h.n);
  h.type_count = s.type_count;
  h.lj_a.assign(s.lj_a, s.lj_a + (size_t)h.type_count * h.type_count);
  h.lj_b.assign(s.lj_b, s.lj_b + (size_t)h.type_count * h.type_count);
  h.dof = s.degrees_of_freedom;
  h.n_molecules = s.molecule_count;

  // skinFor (cells.js:67-91), unless given.
  if (o.skin > 0) {
    h.skin = o.skin;
  } else {
    double lightest = INFINITY;
    for (double m : h.masses)
      if (m > 0 && m < lightest) lightest = m;
    if (!std::isfinite(lightest)) lightest = 1.008;
    const double speed = std::sqrt((o.temperature / 298.0) * (1.008 / lightest));
    const double scaled = LIGHT_ANCHOR_SKIN * (o.timestep / 0.002) * speed;
    const double room = 0.5 * smallest - h.cutoff;
    h.skin = std::max(0.1, std::min(scaled, room > 0 ? room * 0.9 : 0.1));
  }
  h.list_cutoff = h.cutoff + h.skin;
  // planCellList (cells.js:101-171)
  for (int d = 0; d < 3; ++d) h.counts[d] = std::max(1, (int)std::floor(widths[d] / h.list_cutoff));
  const double volume = widths[0] * widths[1] * widths[2];
  const double density = h.n / volume;
  h.estimated_neighbours = density * (4.0 / 3.0) * M_PI * std::pow(h.list_cutoff, 3);
  const double slack = o.neighbour_slack > 0 ? o.neighbour_slack : 2.0;
  h.capacity = o.max_neighbours > 0 ? o.max_neighbours
                                    : std::max(32, (int)std::ceil(h.estimated_neighbours * slack));
  h.capacity = row_capacity(h.capacity);
  // pmeParameters (parameters.js:227-252)
  const double tol = o.ewald_tolerance > 0 ? o.ewald_tolerance : 5e-4;
  h.alpha = o.alpha > 0 ? o.alpha : alpha_from_tolerance(h.cutoff, tol);
  h.order = o.pme_order == 4 ? 4 : 5;
  for (int d = 0; d < 3; ++d) {
    if (o.grid[d] > 0) {
      h.grid[d] = o.grid[d];
    } else {
      const double len = std::sqrt(h.box[3 * d] * h.box[3 * d] + h.box[3 * d + 1] * h.box[3 * d + 1] +
                                   h.box[3 * d + 2] * h.box[3 * d + 2]);
      int c = std::max(2, (int)std::ceil(2.0 * h.alpha * len / (3.0 * std::pow(tol, 0.2))));
      while (!transformable(c)) ++c;
      h.grid[d] = c;
    }
    if (!transformable(h.grid[d]))
      throw Error(RMD_ERR_INVALID, "PME grid size " + std::to_string(h.grid[d]) +
                                       " is not a product of 2, 3 and 5, which is what the FFT can transform");
    if (h.grid[d] < h.order)
      throw Error(RMD_ERR_INVALID, "PME grid size smaller than the interpolation order; the box is too "
                                   "small for this cutoff");
    if (h.grid[d] > 2048) throw Error(RMD_ERR_INVALID, "PME grid sizes above 2048 are not supported");
  }
  h.q2 = 0;
  h.qsum = 0;
  for (double q : h.charges) {
    h.q2 += q * q;
    h.qsum += q;
  }
  // dispersionCoefficients (dispersion.js:37-64)
  {
    const int T = h.type_count;
    std::vector<double> cnt(T, 0.0);
    for (int t : h.types) cnt[t] += 1.0;
    double oa = 0, ob = 0, da = 0, db = 0;
    for (int i = 0; i < T; ++i) {
      for (int j = 0; j < T; ++j) {
        oa += cnt[i] * cnt[j] * h.lj_a[T * i + j];
        ob += cnt[i] * cnt[j] * h.lj_b[T * i + j];
      }
      da += cnt[i] * h.lj_a[T * i + i];
      db += cnt[i] * h.lj_b[T * i + i];
    }
    const double sc = (double)h.n / (h.n + 1);
    h.disp_a = (oa + da) * sc;
    h.disp_b = (ob + db) * sc;
  }
  h.requested_rebuild = o.rebuild_interval > 0 ? o.rebuild_interval : 20;
  h.adaptive = o.adaptive_rebuild != 0;
  h.on_demand = o.rebuild_on_demand != 0;
  h.rebuild_interval = h.adaptive ? std::min(h.requested_rebuild, 4) : h.requested_rebuild;
  h.has_pressure = o.pressure > -1e299;
  h.barostat_interval = o.barostat_interval > 0 ? o.barostat_interval : 25;
  h.requested_tol = o.tolerance > 0 ? o.tolerance : 1e-5;
  h.tolerance = h.requested_tol;
  h.min_constraint = INFINITY;
  for (int k = 0; k < s.constraint_count; ++k) h.min_constraint = std::min(h.min_constraint, s.constraint_distance[k]);
  if (o.restraint_force > 0 && o.restraint_count > 0) {
    h.restraint_atoms.assign(o.restraint_atoms, o.restraint_atoms + o.restraint_count);
    for (int a : h.restraint_atoms) {
      if (a < 0 || a >= h.n) throw Error(RMD_ERR_INVALID, "restraint atom out of range");
      for (int c = 0; c < 3; ++c) h.restraint_reference.push_back(o.restraint_reference[3 * a + c]);
    }
  }
}

static FastDiv make_fast_div(uint32_t d) {
  if (d == 0 || d >= (1u << 31)) throw Error(RMD_ERR_INVALID, "divisor out of range");
  uint32_t shift = 0;
  while ((1ull << shift) < d) ++shift;
  const unsigned long long magic = (((1ull << 32) * ((1ull << shift) - d)) / d) + 1;
  return FastDiv{(uint32_t)magic, shift};
}

static void fft_axis_plan(int n, FftAxis &ax, int tw_base) {
  ax.n = n;
  ax.nstages = 0;
  ax.tw_base = tw_base;
  int r = n;
  while (r % 4 == 0) { ax.radix[ax.nstages++] = 4; r /= 4; }
  while (r % 2 == 0) { ax.radix[ax.nstages++] = 2; r /= 2; }
  while (r % 3 == 0) { ax.radix[ax.nstages++] = 3; r /= 3; }
  while (r % 5 == 0) { ax.radix[ax.nstages++] = 5; r /= 5; }
  int span = 1;
  for (int st = 0; st < ax.nstages; ++st) {
    ax.per_line[st] = make_fast_div((uint32_t)(n / ax.radix[st]));
    ax.span[st] = make_fast_div((uint32_t)span);
    span *= ax.radix[st];
  }
  ax.n_div = make_fast_div((uint32_t)n);
  ax.half_div = make_fast_div((uint32_t)(n / 2 + 1));
}

constexpr int FFT_SMEM_HOST = 2048;

void Engine::build(int count, const rmd_system *systems, const rmd_options *options) {
  S = count;
  hs.resize(S);
  std::vector<const rmd_system *> src(S);
  N = 0;
  for (int s = 0; s < S; ++s) {
    hs[s].opt = options[s];
    src[s] = &systems[s];
    plan_system(hs[s], systems[s]);
    hs[s].atom_start = N;
    N += hs[s].n;
  }
  pme_order = hs[0].order;
  pair_fixed = options[0].force_accumulation == 1 ? 0 : 1;
  // the group-pair rows need the precision form (every pair force quantised) and slot indices
  // that fit their 23 bits; otherwise the per-atom rows
  pair_list = options[0].pair_list;
  if (pair_list != 1 && pair_list != 2) pair_list = 0;
  if (!pair_fixed || N > GROUP_SLOT_MASK) pair_list = 1;
  {
    const rmd_options &o = options[0];
    auto pick = [](int v, int a, int b, int c, int dflt) { return v == a || v == b || v == c ? v : dflt; };
    group_atoms = o.neighbour_group_atoms == 32 ? 32 : pick(o.neighbour_group_atoms, 4, 8, 16, 8);
    nb_lanes = pick(o.nonbonded_lanes, 8, 16, 32, 32);
    spread_atoms = pick(o.spread_atoms_per_block, 4, 8, 16, 8);
    tune_group = o.neighbour_group_atoms == 0;
    tune_lanes = o.nonbonded_lanes == 0;
    tune_spread = o.spread_atoms_per_block == 0;
    if (pair_list != 1) {  // group-pair rows: 4-atom search groups; lanes per group row 32 x the
      group_atoms = GROUP_ATOMS;  // warps that share it (32, 64 or 128)
      nb_lanes = pick(o.nonbonded_lanes, 32, 64, 128, 64);
      tune_group = false;
    }
  }
  for (auto &h : hs)
    if (h.order != pme_order) throw Error(RMD_ERR_INVALID, "every system of a batch must use the same PME order");
  // A blocking stream: work on it is ordered after the legacy default stream's, which is
  // where the host-side uploads (cudaMemcpy from pageable memory, which may return before
  // its DMA lands; cudaMemset, which is asynchronous) go. A non-blocking stream would let a
  // kernel read a buffer before such an upload had finished.
  CUDA_OK(cudaStreamCreateWithFlags(&stream, cudaStreamDefault));
  // The reciprocal branch's stream. Step graphs are instantiated without per-node priorities,
  // so its kernels run at the graph's launch priority; measured on one B200 (23,558 atoms),
  // giving them the highest priority (cudaGraphInstantiateFlagUseNodePriority) slowed the NVT
  // step from 0.101 to 0.104 ms, and the pair branch the higher one changed nothing.
  CUDA_OK(cudaStreamCreateWithFlags(&side, cudaStreamDefault));
  CUDA_OK(cudaStreamCreateWithFlags(&cond, cudaStreamNonBlocking));
  on_demand = true;
  for (auto &h : hs) on_demand = on_demand && h.on_demand;
  CUDA_OK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
  CUDA_OK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
  CUDA_OK(cudaEventCreateWithFlags(&ev_clear, cudaEventDisableTiming));
  upload_all(src);
}

void Engine::upload_all(const std::vector<const rmd_system *> &src) {
  // ---- atoms
  std::vector<float4> h_posq(N), h_vel(N);
  std::vector<int> h_type(N), h_sys_of(N), h_sys_start(S);
  std::vector<float> h_mass(N);
  std::vector<float2> h_lj;
  std::vector<int> lj_base(S);
  for (int s = 0; s < S; ++s) {
    const HostSystem &h = hs[s];
    h_sys_start[s] = h.atom_start;
    lj_base[s] = (int)h_lj.size();
    for (int k = 0; k < h.type_count * h.type_count; ++k) h_lj.push_back(make_float2((float)h.lj_a[k], (float)h.lj_b[k]));
    for (int i = 0; i < h.n; ++i) {
      const int g = h.atom_start + i;
      h_posq[g] = make_float4(0, 0, 0, (float)h.charges[i]);
      h_vel[g] = make_float4(0, 0, 0, h.masses[i] > 0 ? (float)(1.0 / h.masses[i]) : 0.f);
      h_type[g] = h.types[i];
      h_sys_of[g] = s;
      h_mass[g] = (float)h.masses[i];
    }
  }
  posq.upload(h_posq);
  vel.upload(h_vel);
  origin.upload(h_posq);
  saved_posq.upload(h_posq);
  atom_type.upload(h_type);
  sys_of_atom.upload(h_sys_of);
  sys_atom_start.upload(h_sys_start);
  masses.upload(h_mass);
  lj.upload(h_lj);
  noise.alloc(3 * (size_t)N);
  noise.zero();
  force.alloc(3 * (size_t)N + 1);  // rounded up to even: k_rebuild_decide clears it two words at a time
  force.zero();
  saved_force.alloc(3 * (size_t)N);
  saved_force.zero();
  for (auto *a : {&e_lj, &e_coul, &e_vir, &ke_post, &ke_early}) {
    a->alloc(N);
    a->zero();
  }

  // ---- exclusions (buildExclusionGather, cells.js:191-227) and exceptions
  //      (buildExceptionGather, cells.js:237-271), global atom indices
  std::vector<int> ex_start(N + 1, 0), ex_part, xs(N + 1, 0), xp;
  std::vector<float4> xparam;
  {
    std::vector<std::vector<int>> ex(N);
    std::vector<std::vector<std::pair<int, float4>>> xc(N);
    for (int s = 0; s < S; ++s) {
      const rmd_system &r = *src[s];
      const int base = hs[s].atom_start;
      for (int a = 0; a < r.atom_count; ++a)
        for (int c = r.exclusion_start[a]; c < r.exclusion_start[a + 1]; ++c) {
          const int b = r.exclusion_partners[c];
          if (b < 0 || b >= r.atom_count) throw Error(RMD_ERR_INVALID, "exclusion partner out of range");
          ex[base + a].push_back(base + b);
          ex[base + b].push_back(base + a);
        }
      for (int k = 0; k < r.exception_count; ++k) {
        const int a = r.exception_atoms[2 * k], b = r.exception_atoms[2 * k + 1];
        if (a < 0 || b < 0 || a >= r.atom_count || b >= r.atom_count)
          throw Error(RMD_ERR_INVALID, "exception atom out of range");
        const float qa = (float)r.charges[a], qb = (float)r.charges[b];
        (void)qa; (void)qb;
        const float full_ab = (float)(r.charges[a] * r.charges[b]);
        float4 p = make_float4((float)r.exception_charge_product[k], (float)r.exception_lj_a[k],
                               (float)r.exception_lj_b[k], full_ab);
        xc[base + a].push_back({base + b, p});
        xc[base + b].push_back({base + a, p});
      }
    }
    for (int i = 0; i < N; ++i) {
      std::sort(ex[i].begin(), ex[i].end());
      ex_start[i + 1] = ex_start[i] + (int)ex[i].size();
      ex_part.insert(ex_part.end(), ex[i].begin(), ex[i].end());
      xs[i + 1] = xs[i] + (int)xc[i].size();
      for (auto &pr : xc[i]) {
        xp.push_back(pr.first);
        xparam.push_back(pr.second);
      }
    }
  }
  if (ex_part.empty()) ex_part.push_back(0);
  if (xp.empty()) {
    xp.push_back(0);
    xparam.push_back(make_float4(0, 0, 0, 0));
  }
  excl_start.upload(ex_start);
  excl_partners.upload(ex_part);
  exc_start.upload(xs);
  exc_partner.upload(xp);
  exc_param.upload(xparam);

  // ---- bonded terms and restraints, per system in order
  std::vector<int2> hb;
  std::vector<float2> hbp, hap;
  std::vector<int4> ha, ht;
  std::vector<float4> htp, hrp;
  std::vector<int> hra;
  std::vector<int> bstart(S + 1), astart(S + 1), tstart(S + 1), rstart(S + 1);
  for (int s = 0; s < S; ++s) {
    const rmd_system &r = *src[s];
    const int base = hs[s].atom_start;
    bstart[s] = (int)hb.size();
    for (int k = 0; k < r.bond_count; ++k) {
      hb.push_back(make_int2(base + r.bond_atoms[2 * k], base + r.bond_atoms[2 * k + 1]));
      hbp.push_back(make_float2((float)r.bond_k[k], (float)r.bond_r0[k]));
    }
    astart[s] = (int)ha.size();
    for (int k = 0; k < r.angle_count; ++k) {
      ha.push_back(make_int4(base + r.angle_atoms[3 * k], base + r.angle_atoms[3 * k + 1],
                             base + r.angle_atoms[3 * k + 2], 0));
      hap.push_back(make_float2((float)r.angle_k[k], (float)r.angle_theta0[k]));
    }
    tstart[s] = (int)ht.size();
    for (int k = 0; k < r.torsion_count; ++k) {
      ht.push_back(make_int4(base + r.torsion_atoms[4 * k], base + r.torsion_atoms[4 * k + 1],
                             base + r.torsion_atoms[4 * k + 2], base + r.torsion_atoms[4 * k + 3]));
      htp.push_back(make_float4((float)r.torsion_k[k], (float)r.torsion_periodicity[k],
                                (float)r.torsion_phase[k], 0.f));
    }
    rstart[s] = (int)hra.size();
    const HostSystem &h = hs[s];
    for (size_t k = 0; k < h.restraint_atoms.size(); ++k) {
      hra.push_back(base + h.restraint_atoms[k]);
      hrp.push_back(make_float4((float)h.restraint_reference[3 * k], (float)h.restraint_reference[3 * k + 1],
                                (float)h.restraint_reference[3 * k + 2], (float)h.opt.restraint_force));
    }
  }
  bstart[S] = (int)hb.size();
  astart[S] = (int)ha.size();
  tstart[S] = (int)ht.size();
  rstart[S] = (int)hra.size();
  n_bonds = (int)hb.size();
  n_angles = (int)ha.size();
  n_tors = (int)ht.size();
  n_rest = (int)hra.size();
  bond_atoms.upload(hb);
  bond_param.upload(hbp);
  angle_atoms.upload(ha);
  angle_param.upload(hap);
  tor_atoms.upload(ht);
  tor_param.upload(htp);
  rest_atom.upload(hra);
  rest_param.upload(hrp);
  e_term.alloc(std::max(1, n_bonds + n_angles + n_tors + n_rest));
  e_term.zero();
  e_term_vir.alloc(std::max(1, n_bonds + n_angles + n_tors + n_rest));
  e_term_vir.zero();

  // ---- constraint clusters (buildConstraintClusters, clusters.js:20-57) and SETTLE waters
  std::vector<int> h_free, h_cl_as, h_cl_atoms, h_cl_cs;
  std::vector<int2> h_pairs;
  std::vector<float> h_dist;
  std::vector<int3> h_settle;
  std::vector<DevSettle> h_settle_p;
  h_cl_as.push_back(0);
  h_cl_cs.push_back(0);
  for (int s = 0; s < S; ++s) {
    const rmd_system &r = *src[s];
    HostSystem &h = hs[s];
    const int base = h.atom_start;
    std::vector<int> parent(h.n);
    std::iota(parent.begin(), parent.end(), 0);
    auto find = [&](int x) {
      int root = x;
      while (parent[root] != root) root = parent[root];
      while (parent[x] != root) {
        int nx = parent[x];
        parent[x] = root;
        x = nx;
      }
      return root;
    };
    for (int k = 0; k < r.constraint_count; ++k) {
      const int a = r.constraint_atoms[2 * k], b = r.constraint_atoms[2 * k + 1];
      if (a < 0 || b < 0 || a >= h.n || b >= h.n) throw Error(RMD_ERR_INVALID, "constraint atom out of range");
      const int ra = find(a), rb = find(b);
      if (ra != rb) parent[rb] = ra;
    }
    std::map<int, std::vector<int>> by_root;  // root -> constraint indices, in order
    std::vector<int> root_order;
    for (int k = 0; k < r.constraint_count; ++k) {
      const int root = find(r.constraint_atoms[2 * k]);
      if (!by_root.count(root)) root_order.push_back(root);
      by_root[root].push_back(k);
    }
    std::vector<char> in_cluster(h.n, 0);
    h.n_clusters = 0;
    h.n_settle = 0;
    for (int root : root_order) {
      const auto &members = by_root[root];
      std::vector<int> atoms;
      for (int k : members) {
        atoms.push_back(r.constraint_atoms[2 * k]);
        atoms.push_back(r.constraint_atoms[2 * k + 1]);
      }
      std::sort(atoms.begin(), atoms.end());
      atoms.erase(std::unique(atoms.begin(), atoms.end()), atoms.end());
      for (int a : atoms) in_cluster[a] = 1;
      // SETTLE candidate: a 3-atom triangle, apex the heaviest, equal light masses and
      // equal apex distances (findWaterClusters, constraints.js:36-85).
      if (h.opt.water_solver == 1 && members.size() == 3 && atoms.size() == 3) {
        int apex = atoms[0];
        for (int a : atoms)
          if (h.masses[a] > h.masses[apex]) apex = a;
        std::vector<int> light;
        for (int a : atoms)
          if (a != apex) light.push_back(a);
        auto length = [&](int p, int q) {
          for (int k : members) {
            const int a = r.constraint_atoms[2 * k], b = r.constraint_atoms[2 * k + 1];
            if ((a == p && b == q) || (a == q && b == p)) return r.constraint_distance[k];
          }
          return -1.0;
        };
        const double d1 = length(apex, light[0]), d2 = length(apex, light[1]), d3 = length(light[0], light[1]);
        const double mo = h.masses[apex], mh = h.masses[light[0]];
        if (d1 > 0 && d2 > 0 && d3 > 0 && std::fabs(d1 - d2) < 1e-9 * d1 &&
            std::fabs(h.masses[light[1]] - mh) < 1e-9 * mh && mo > 0 && mh > 0) {
          DevSettle w;
          w.m_o = (float)mo;
          w.m_h = (float)mh;
          const double rc = 0.5 * d3, height = std::sqrt(d1 * d1 - rc * rc);
          const double wt = mo + 2 * mh;
          w.ra = (float)(2.0 * mh * height / wt);
          w.rb = (float)(height - 2.0 * mh * height / wt);
          w.rc = (float)rc;
          w.d_oh = (float)d1;
          w.d_hh = (float)d3;
          w.pad = 0.f;
          h_settle.push_back(make_int3(base + apex, base + light[0], base + light[1]));
          h_settle_p.push_back(w);
          h.n_settle++;
          continue;
        }
      }
      if ((int)atoms.size() > MAX_CLUSTER_ATOMS || (int)members.size() > MAX_CLUSTER_CONSTRAINTS)
        throw Error(RMD_ERR_INVALID, "a constraint cluster of " + std::to_string(atoms.size()) + " atoms and " +
                                         std::to_string(members.size()) +
                                         " constraints exceeds the per-thread solver limit (8 atoms, 12 "
                                         "constraints); use HBonds constraints");
      for (int a : atoms) h_cl_atoms.push_back(base + a);
      h_cl_as.push_back((int)h_cl_atoms.size());
      for (int k : members) {
        const int a = r.constraint_atoms[2 * k], b = r.constraint_atoms[2 * k + 1];
        const int la = (int)(std::lower_bound(atoms.begin(), atoms.end(), a) - atoms.begin());
        const int lb = (int)(std::lower_bound(atoms.begin(), atoms.end(), b) - atoms.begin());
        h_pairs.push_back(make_int2(la, lb));
        h_dist.push_back((float)r.constraint_distance[k]);
      }
      h_cl_cs.push_back((int)h_pairs.size());
      h.n_clusters++;
    }
    for (int a = 0; a < h.n; ++a)
      if (!in_cluster[a]) h_free.push_back(base + a);
  }
  // units in order: free atoms, SHAKE clusters, SETTLE waters
  n_free = (int)h_free.size();
  n_clusters = (int)h_cl_as.size() - 1;
  n_settle = (int)h_settle.size();
  if (h_free.empty()) h_free.push_back(0);
  if (h_cl_atoms.empty()) h_cl_atoms.push_back(0);
  if (h_pairs.empty()) {
    h_pairs.push_back(make_int2(0, 0));
    h_dist.push_back(0.f);
  }
  if (h_settle.empty()) {
    h_settle.push_back(make_int3(0, 0, 0));
    h_settle_p.push_back(DevSettle{});
  }
  free_atoms.upload(h_free);
  cl_atom_start.upload(h_cl_as);
  cl_atoms.upload(h_cl_atoms);
  cl_con_start.upload(h_cl_cs);
  cl_con_pair.upload(h_pairs);
  cl_con_dist.upload(h_dist);
  settle_atoms.upload(h_settle);
  settle_param.upload(h_settle_p);

  // ---- molecules (global CSR over all systems)
  {
    std::vector<int> ms(1, 0), ma, moa(N, 0);
    mol_base.assign(1, 0);
    for (int s = 0; s < S; ++s) {
      const rmd_system &r = *src[s];
      mol_base.push_back(mol_base.back() + r.molecule_count);
      const int base = hs[s].atom_start;
      std::vector<std::vector<int>> mol(r.molecule_count);
      for (int a = 0; a < r.atom_count; ++a) {
        const int m = r.molecule_of_atom[a];
        if (m < 0 || m >= r.molecule_count) throw Error(RMD_ERR_INVALID, "molecule index out of range");
        mol[m].push_back(base + a);
        moa[base + a] = mol_base[s] + m;
      }
      for (auto &m : mol) {
        ma.insert(ma.end(), m.begin(), m.end());
        ms.push_back((int)ma.size());
      }
    }
    n_molecules_total = (int)ms.size() - 1;
    mol_vir.alloc(std::max(1, n_molecules_total));
    mol_vir.zero();
    if (ma.empty()) ma.push_back(0);
    mol_start.upload(ms);
    mol_atoms.upload(ma);
    mol_of_atom.upload(moa);
  }

  // ---- cells
  std::vector<int> h_cell_sys, h_group_sys;
  h_sys.resize(S);
  h_sysd.resize(S);
  int cell_base = 0, cell_start_base = 0;
  for (int s = 0; s < S; ++s) {
    HostSystem &h = hs[s];
    DevSys &d = h_sys[s];
    DevSysD &dd = h_sysd[s];
    memset(&d, 0, sizeof d);
    memset(&dd, 0, sizeof dd);
    d.cutoff = (float)h.cutoff;
    d.cutoff2 = d.cutoff * d.cutoff;
    d.list_cutoff = (float)h.list_cutoff;
    d.list_cutoff2 = d.list_cutoff * d.list_cutoff;
    d.alpha = (float)h.alpha;
    d.atom_start = h.atom_start;
    d.atom_count = h.n;
    d.type_count = h.type_count;
    d.lj_base = lj_base[s];
    const int cells = h.counts[0] * h.counts[1] * h.counts[2];
    for (int k = 0; k < 3; ++k) {
      d.cell_counts[k] = h.counts[k];
      dd.max_counts[k] = h.counts[k];
    }
    d.cell_base = cell_base;
    d.cell_start_base = cell_start_base;
    d.cell_capacity = cells;
    for (int c = 0; c < cells; ++c) h_cell_sys.push_back(s);
    // search groups: at most ceil(n / 32) full ones plus one partial group per cell
    d.group_base = (int)h_group_sys.size();
    const int groups = neighbour_group_slots(h.n, cells, 4);  // enough for every group size
    for (int q = 0; q < groups; ++q) h_group_sys.push_back(s);
    cell_base += cells;
    cell_start_base += cells + 1;
    d.order = h.order;
    d.molecule_count = h.n_molecules;
    dd.q2_sum = h.q2;
    dd.q_sum = h.qsum;
    dd.disp_a = h.disp_a;
    dd.disp_b = h.disp_b;
    dd.cutoff = h.cutoff;
    dd.alpha = h.alpha;
    dd.list_cutoff = h.list_cutoff;
    dd.dispersion_on = h.opt.dispersion_correction != 0;
    for (int k = 0; k < 9; ++k) dd.box[k] = h.box[k];
  }
  n_cells_total = cell_base;
  cell_sys.upload(h_cell_sys);
  cell_count.alloc(n_cells_total);
  cell_count.zero();
  cell_start.alloc(cell_start_base);
  cell_start.zero();
  cell_gstart.alloc(cell_start_base);
  cell_gstart.zero();
  n_groups_total = (int)h_group_sys.size();
  group_sys.upload(h_group_sys);
  group_order.alloc(N);
  cell_atoms.alloc(N);
  cell_of_atom.alloc(N);
  spos.alloc(N);
  spos.zero();
  wrap.alloc(N);
  wrap.zero();
  sorted_orig.alloc(N);
  sorted_orig.zero();
  sorted_type.alloc(N);
  sorted_type.zero();
  slot_info.alloc(N);
  slot_info.zero();
  order_pos.alloc(N);
  order_pos.zero();
  e_acc.alloc(3 * (size_t)N);
  e_acc.zero();
  rank.alloc(N);
  rank.zero();
  required.alloc(2 * (size_t)S);  // longest per-atom row, then longest group-pair row, per system
  required.zero();
  required_max.alloc(S);
  required_max.zero();
  stale.alloc(S);
  stale.zero();
  saved_wrap.alloc(N);
  saved_origin.alloc(N);
  for (auto *a : {&list_allow, &saved_allow}) {
    a->alloc(S);
    a->zero();
  }
  list_rebuilt.alloc(S);
  list_rebuilt.zero();
  spread_bits.alloc(S);
  spread_bits.zero();
  list_builds.alloc(2);
  list_builds.zero();

  // ---- PME grids, moduli, twiddles, FFT plans and task tables
  {
    long long gbase = 0, hbase = 0;
    std::vector<float> h_mod;
    std::vector<float2> h_tw;
    std::vector<FftPlan> h_plans(S);
    std::vector<FftTask> tz, ty, tx, tp, tq, ty_all, tx_all;
    std::vector<int> split(S);
    plane_stride = cluster_rows = cluster_cols = 0;
    // Lines per block. The z and y passes (no sums across lines) are sized from the whole
    // batch's line count: as many lines as fit the shared buffers and about 2 elements per
    // thread, but few enough that a pass has at least ~4 blocks per SM (592 on 148 SMs), so 64
    // small grids fill blocks as one large grid does. The x pass also sums the reciprocal
    // energy per block, so its size depends on the line length alone: a system's energy
    // partials are grouped the same way in a batch as alone, and come out bit for bit equal.
    long long all_pairs = 0, all_ylines = 0;
    for (int s = 0; s < S; ++s) {
      all_pairs += ((long long)hs[s].grid[0] * hs[s].grid[1] + 1) / 2;
      all_ylines += (long long)hs[s].grid[0] * (hs[s].grid[2] / 2 + 1);
    }
    auto lines_per_block = [](long long total_lines, int n, int cap) {
      int m = std::max(1, std::min(cap, FFT_SMEM_HOST / n));
      m = (int)std::min<long long>(m, std::max(1LL, (long long)std::ceil(total_lines / 592.0)));
      m = std::min(m, std::max(1, 512 / n));
      return m;
    };
    for (int s = 0; s < S; ++s) {
      HostSystem &h = hs[s];
      DevSys &d = h_sys[s];
      const int nx = h.grid[0], ny = h.grid[1], nz = h.grid[2], nzh = nz / 2 + 1;
      for (int k = 0; k < 3; ++k) d.grid[k] = h.grid[k];
      d.grid_base = gbase;
      d.half_base = hbase;
      d.moduli_base = (int)h_mod.size();
      gbase += (long long)nx * ny * nz;
      hbase += (long long)nx * ny * nzh;
      for (int ax = 0; ax < 3; ++ax) {
        for (double m : bspline_moduli(h.grid[ax], h.order)) h_mod.push_back((float)m);
        fft_axis_plan(h.grid[ax], h_plans[s].axis[ax], (int)h_tw.size());
        for (int k = 0; k < h.grid[ax]; ++k) {
          const double a = -2.0 * M_PI * k / h.grid[ax];
          h_tw.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
        }
      }
      // z pass: pairs of real lines
      const int lines = nx * ny, pairs = (lines + 1) / 2;
      const int mz = lines_per_block(all_pairs, nz, 64);
      for (int p = 0; p < pairs; p += mz) tz.push_back(FftTask{s, 0, p, std::min(mz, pairs - p)});
      // A system whose kz plane fits shared memory runs the fused y-x-convolve-x-y pass, one
      // block or one cluster of blocks a plane; the others run the separate y and x passes. The
      // debug transforms run the separate passes over every system.
      split[s] = fft_plane_split(nx, ny);
      const bool fused = split[s] > 0;
      const int my = lines_per_block(all_ylines, ny + 1, nzh);  // y and x lines are padded to n + 1
      const int mx = std::max(1, std::min(nzh, std::min(FFT_SMEM_HOST / (nx + 1), 512 / (nx + 1))));
      for (int x = 0; x < nx; ++x)
        for (int k = 0; k < nzh; k += my) {
          ty_all.push_back(FftTask{s, x, k, std::min(my, nzh - k)});
          if (!fused) ty.push_back(ty_all.back());
        }
      for (int y = 0; y < ny; ++y)
        for (int k = 0; k < nzh; k += mx) {
          tx_all.push_back(FftTask{s, y, k, std::min(mx, nzh - k)});
          if (!fused) tx.push_back(tx_all.back());
        }
      int rows = 0, cols = 0;
      if (fused) fft_plane_buffers(nx, ny, split[s], &rows, &cols);
      std::vector<FftTask> &planes = split[s] == 1 ? tp : tq;
      for (int kz = 0; fused && kz < nzh; ++kz) planes.push_back(FftTask{s, kz, 0, 0});
      if (split[s] == 1) plane_stride = std::max(plane_stride, rows);
      if (split[s] > 1) {
        cluster_rows = std::max(cluster_rows, rows);
        cluster_cols = std::max(cluster_cols, cols);
      }
    }
    // energy partials: the x tasks' (one each), the planes' (one each), the clusters'
    // (PLANE_CLUSTER each); a system's are contiguous within its pass's range
    {
      const long long base_p = (long long)tx.size(), base_q = base_p + (long long)tp.size();
      recip_lo.assign(S, 0);
      recip_hi.assign(S, 0);
      for (int s = 0; s < S; ++s) recip_lo[s] = LLONG_MAX;
      auto cover = [&](int s, long long k) {
        recip_lo[s] = std::min(recip_lo[s], k);
        recip_hi[s] = std::max(recip_hi[s], k + 1);
      };
      for (size_t k = 0; k < tx.size(); ++k) cover(tx[k].sys, (long long)k);
      for (size_t k = 0; k < tp.size(); ++k) cover(tp[k].sys, base_p + (long long)k);
      for (size_t k = 0; k < tq.size(); ++k)
        for (int r = 0; r < PLANE_CLUSTER; ++r) cover(tq[k].sys, base_q + (long long)k * PLANE_CLUSTER + r);
      for (int s = 0; s < S; ++s)
        if (recip_lo[s] == LLONG_MAX) recip_lo[s] = recip_hi[s] = 0;  // no reciprocal tasks
    }
    if (!tp.empty() || !tq.empty()) CUDA_OK(fft_plane_prepare());
    fixed_grid.alloc(gbase);
    fixed_grid.zero();
    half.alloc(hbase);
    real_grid.alloc(gbase);
    real_grid.zero();
    moduli.upload(h_mod);
    twiddles.upload(h_tw);
    fft_plans.upload(h_plans);
    tasks_z.upload(tz);
    tasks_y.upload(ty);
    tasks_x.upload(tx);
    tasks_plane.upload(tp);
    tasks_cluster.upload(tq);
    tasks_y_all.upload(ty_all);
    tasks_x_all.upload(tx_all);
    const size_t partials = std::max<size_t>(1, tx.size() + tp.size() + tq.size() * PLANE_CLUSTER);
    e_pme.alloc(partials);
    e_pme.zero();
    e_pme_vir.alloc(partials);
    e_pme_vir.zero();
  }

  // ---- per-system device state
  sysd.upload(h_sysd);
  sys.upload(h_sys);
  launch_update_box(sys.p, sysd.p, S, stream);
  CUDA_OK(cudaStreamSynchronize(stream));
  CUDA_OK(cudaMemcpy(h_sys.data(), sys.p, sizeof(DevSys) * S, cudaMemcpyDeviceToHost));
  allocate_neighbours();

  std::vector<DevInteg> h_integ(S);
  for (int s = 0; s < S; ++s) {
    const rmd_options &o = hs[s].opt;
    const double decay = std::exp(-o.friction * o.timestep);
    h_integ[s] = DevInteg{(float)(0.5 * o.timestep), (float)decay,
                          (float)std::sqrt(std::max(0.0, 1.0 - decay * decay)),
                          (float)(BOLTZMANN * o.temperature), (float)hs[s].tolerance, o.seed,
                          o.max_constraint_iterations > 0 ? o.max_constraint_iterations : 150, 0};
  }
  integ.upload(h_integ);
  step_base.alloc(S);
  step_base.zero();
  disp.alloc(2 * S);
  disp.zero();
  diag.alloc(4 * S);
  diag.zero();
  energies.alloc((size_t)S * N_ENERGY);
  energies.zero();
  saved_energies.alloc((size_t)S * N_ENERGY);
  saved_energies.zero();
  fixed_scales.alloc(S);
  {
    std::vector<double> hb(S * (size_t)N_BARO, 0.0);
    for (int s = 0; s < S; ++s) {
      const HostSystem &h = hs[s];
      double *b = hb.data() + (size_t)s * N_BARO;
      any_pressure = any_pressure || h.has_pressure;
      b[B_ACTIVE] = h.has_pressure ? 1.0 : 0.0;
      b[B_PRESSURE] = h.has_pressure ? h.opt.pressure * BAR_TO_KJ_PER_MOL_NM3 : 0.0;
      b[B_KT] = BOLTZMANN * h.opt.temperature;
      b[B_NMOL] = h.n_molecules;
      b[B_SEED] = (double)h.opt.seed;
      const bool lb = h.has_pressure && h.opt.learned_barostat != 0;
      learned = learned || lb;
      b[B_LEARNED] = lb ? 1.0 : 0.0;
      b[B_WARMUP] = h.opt.learned_warmup_moves > 0 ? h.opt.learned_warmup_moves : 2000;
      b[B_VOL_REF] = std::fabs(h.box[0] * h.box[4] * h.box[8]);
      b[B_DOF] = h.dof;
    }
    if (learned) {
      // Xavier-uniform weights (the output layer scaled down), zero biases, from the seed
      std::vector<float> w((size_t)S * MLP_STRIDE, 0.f);
      for (int s = 0; s < S; ++s) {
        uint64_t state = 0x9e3779b97f4a7c15ULL ^ (uint64_t)hs[s].opt.seed * 0xbf58476d1ce4e5b9ULL;
        auto uniform = [&state]() {
          state ^= state << 13;
          state ^= state >> 7;
          state ^= state << 17;
          return (double)(state >> 11) * (1.0 / 9007199254740992.0);
        };
        float *p = w.data() + (size_t)s * MLP_STRIDE;
        const double l1 = std::sqrt(6.0 / (MLP_IN + MLP_H)), l2 = std::sqrt(6.0 / (2 * MLP_H)),
                     l3 = 0.1 * std::sqrt(6.0 / (MLP_H + 1));
        for (int k = 0; k < MLP_H * MLP_IN; ++k) p[MLP_W1 + k] = (float)((2 * uniform() - 1) * l1);
        for (int k = 0; k < MLP_H * MLP_H; ++k) p[MLP_W2 + k] = (float)((2 * uniform() - 1) * l2);
        for (int k = 0; k < MLP_H; ++k) p[MLP_W3 + k] = (float)((2 * uniform() - 1) * l3);
      }
      std::vector<unsigned short> wb(w.size());
      for (size_t k = 0; k < w.size(); ++k) wb[k] = bf16_round_bits(w[k]);
      mlp_master.upload(w);
      mlp_wbf.upload(wb);
      mlp_m.alloc(w.size());
      mlp_m.zero();
      mlp_v.alloc(w.size());
      mlp_v.zero();
      mlp_replay.alloc((size_t)S * MLP_REPLAY * (MLP_IN + 1));
      mlp_replay.zero();
      const rmd_options &o0 = hs[0].opt;
      if (o0.learned_steps_per_move > 0) learned_steps = o0.learned_steps_per_move;
      if (o0.learned_rate > 0) learned_lr = (float)o0.learned_rate;
    }
    std::vector<double> tmp = hb;
    baro.upload(tmp);
  }
  // ---- energy segments
  {
    std::vector<Segment> seg;
    auto recip_begin = [&](int s) { return recip_lo[s]; };
    auto recip_end = [&](int s) { return recip_hi[s]; };
    for (int s = 0; s < S; ++s) {
      const HostSystem &h = hs[s];
      const long long a0 = h.atom_start, a1 = h.atom_start + h.n;
      seg.push_back(Segment{s, E_BOND, e_term.p, bstart[s], bstart[s + 1], nullptr});
      seg.push_back(Segment{s, E_ANGLE, e_term.p, n_bonds + astart[s], n_bonds + astart[s + 1], nullptr});
      seg.push_back(Segment{s, E_TORSION, e_term.p, n_bonds + n_angles + tstart[s],
                            n_bonds + n_angles + tstart[s + 1], nullptr});
      seg.push_back(Segment{s, E_RESTRAINT, e_term.p, n_bonds + n_angles + n_tors + rstart[s],
                            n_bonds + n_angles + n_tors + rstart[s + 1], nullptr});
      seg.push_back(Segment{s, E_LJ, e_lj.p, a0, a1, nullptr});
      seg.push_back(Segment{s, E_COUL_DIRECT, e_coul.p, a0, a1, nullptr});
      seg.push_back(Segment{s, E_RECIP, e_pme.p, recip_begin(s), recip_end(s), nullptr});
      seg.push_back(Segment{s, E_VIR_SR, e_vir.p, a0, a1, nullptr});
      seg.push_back(Segment{s, E_VIR_SR, e_term_vir.p, bstart[s], bstart[s + 1], nullptr});
      seg.push_back(Segment{s, E_VIR_SR, e_term_vir.p, n_bonds + astart[s], n_bonds + astart[s + 1], nullptr});
      seg.push_back(Segment{s, E_VIR_SR, e_term_vir.p, n_bonds + n_angles + tstart[s],
                            n_bonds + n_angles + tstart[s + 1], nullptr});
      seg.push_back(Segment{s, E_VIR_SR, e_term_vir.p, n_bonds + n_angles + n_tors + rstart[s],
                            n_bonds + n_angles + n_tors + rstart[s + 1], nullptr});
      seg.push_back(Segment{s, E_VIR_MOL, mol_vir.p, mol_base[s], mol_base[s + 1], nullptr});
      seg.push_back(Segment{s, E_VIR_REC, e_pme_vir.p, recip_begin(s), recip_end(s), nullptr});
      seg.push_back(Segment{s, E_KINETIC, ke_post.p, a0, a1, nullptr});
      seg.push_back(Segment{s, E_KINETIC_EARLY, ke_early.p, a0, a1, nullptr});
    }
    n_segments = (int)seg.size();
    segments.upload(seg);
    seg_out.alloc(n_segments);
  }
}

void Engine::allocate_neighbours() {
  long long total = 0, group_total = 0;
  for (int s = 0; s < S; ++s) {
    h_sys[s].nbr_base = total;
    h_sys[s].nbr_capacity = hs[s].capacity;
    total += (long long)hs[s].n * hs[s].capacity;
    const int groups = (s + 1 < S ? h_sys[s + 1].group_base : n_groups_total) - h_sys[s].group_base;
    h_sys[s].gnbr_base = group_total;
    if (pair_list != 1) group_total += (long long)groups * hs[s].capacity;
  }
  // per-atom rows only where the pair loop or an inspection reads them
  nbr.alloc(pair_list == 0 ? 1 : total);
  nbr.zero();
  nbr_count.alloc(N);
  nbr_count.zero();
  gnbr.alloc(std::max<long long>(1, group_total));
  gnbr.zero();
  for (auto *a : {&gnbr_count, &gfirst, &gsize}) {
    a->alloc(std::max(1, n_groups_total));
    a->zero();
  }
  if (group_box.n < 2 * (size_t)std::max(1, n_groups_total)) {
    group_box.alloc(2 * (size_t)std::max(1, n_groups_total));
    group_box.zero();
  }
  // push only the neighbour fields (the box may have been changed on the device)
  std::vector<DevSys> cur(S);
  CUDA_OK(cudaMemcpy(cur.data(), sys.p, sizeof(DevSys) * S, cudaMemcpyDeviceToHost));
  for (int s = 0; s < S; ++s) {
    cur[s].nbr_base = h_sys[s].nbr_base;
    cur[s].nbr_capacity = h_sys[s].nbr_capacity;
    cur[s].gnbr_base = h_sys[s].gnbr_base;
  }
  CUDA_OK(cudaMemcpy(sys.p, cur.data(), sizeof(DevSys) * S, cudaMemcpyHostToDevice));
  h_sys = cur;
  for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
  graphs.clear();
}

LaunchCtx Engine::ctx() const {
  LaunchCtx c{};
  c.chain_pme = on_demand ? 1 : 0;
  c.n_atoms = N;
  c.n_systems = S;
  c.posq = posq.p;
  c.atom_type = atom_type.p;
  c.sys_of_atom = sys_of_atom.p;
  c.sys = sys.p;
  c.sysd = sysd.p;
  c.cell_of_atom = cell_of_atom.p;
  c.cell_count = cell_count.p;
  c.cell_start = cell_start.p;
  c.cell_atoms = cell_atoms.p;
  c.cell_sys = cell_sys.p;
  c.n_cells_total = n_cells_total;
  c.cell_gstart = cell_gstart.p;
  c.group_order = group_order.p;
  c.group_sys = group_sys.p;
  c.n_groups_total = n_groups_total;
  c.group_atoms = group_atoms;
  c.spread_atoms = spread_atoms;
  c.excl_start = excl_start.p;
  c.excl_partners = excl_partners.p;
  c.nbr = nbr.p;
  c.nbr_count = nbr_count.p;
  c.required = required.p;
  c.pair_list = pair_list;
  c.gnbr = gnbr.p;
  c.gnbr_count = gnbr_count.p;
  c.gfirst = gfirst.p;
  c.gsize = gsize.p;
  c.slot_info = slot_info.p;
  c.order_pos = order_pos.p;
  c.group_box = group_box.p;
  c.e_acc = e_acc.p;
  c.origin = origin.p;
  c.spos = spos.p;
  c.wrap = wrap.p;
  c.sorted_orig = sorted_orig.p;
  c.sorted_type = sorted_type.p;
  c.rank = rank.p;
  c.lj = lj.p;
  c.lj_entries = (int)lj.n;
  c.exc_start = exc_start.p;
  c.exc_partner = exc_partner.p;
  c.exc_param = exc_param.p;
  c.force = force.p;
  c.force_cleared = false;
  c.e_lj = e_lj.p;
  c.e_coul = e_coul.p;
  c.e_vir = e_vir.p;
  c.pair_fixed = pair_fixed;
  c.bond_atoms = bond_atoms.p;
  c.bond_param = bond_param.p;
  c.n_bonds = n_bonds;
  c.angle_atoms = angle_atoms.p;
  c.angle_param = angle_param.p;
  c.n_angles = n_angles;
  c.tor_atoms = tor_atoms.p;
  c.tor_param = tor_param.p;
  c.n_tors = n_tors;
  c.rest_atom = rest_atom.p;
  c.rest_param = rest_param.p;
  c.n_rest = n_rest;
  c.e_term = e_term.p;
  c.e_term_vir = e_term_vir.p;
  c.mol_start = mol_start.p;
  c.mol_atoms = mol_atoms.p;
  c.masses = masses.p;
  c.mol_vir = mol_vir.p;
  c.n_molecules = n_molecules_total;
  c.pme_on = pme_on ? 1 : 0;
  c.pme_order = pme_order;
  c.fixed_grid = fixed_grid.p;
  c.half = half.p;
  c.real_grid = real_grid.p;
  c.moduli = moduli.p;
  c.twiddles = twiddles.p;
  c.fft_plans = fft_plans.p;
  c.tasks_z = tasks_z.p;
  c.tasks_y = tasks_y.p;
  c.tasks_x = tasks_x.p;
  c.tasks_plane = tasks_plane.p;
  c.tasks_y_all = tasks_y_all.p;
  c.tasks_x_all = tasks_x_all.p;
  c.n_tasks_plane = (int)tasks_plane.n;
  c.tasks_cluster = tasks_cluster.p;
  c.n_tasks_cluster = (int)tasks_cluster.n;
  c.cluster_rows = cluster_rows;
  c.cluster_cols = cluster_cols;
  c.n_tasks_y_all = (int)tasks_y_all.n;
  c.n_tasks_x_all = (int)tasks_x_all.n;
  c.plane_stride = plane_stride;
  c.n_tasks_z = (int)tasks_z.n;
  c.n_tasks_y = (int)tasks_y.n;
  c.n_tasks_x = (int)tasks_x.n;
  c.e_pme = e_pme.p;
  c.e_pme_vir = e_pme_vir.p;
  return c;
}

IntegrateArgs Engine::iargs(int step_offset) const {
  IntegrateArgs a{};
  a.n_free = n_free;
  a.n_clusters = n_clusters;
  a.n_settle = n_settle;
  a.n_units = n_free + n_clusters + n_settle;
  a.n_atoms = N;
  a.n_systems = S;
  a.free_atoms = free_atoms.p;
  a.cl_atom_start = cl_atom_start.p;
  a.cl_atoms = cl_atoms.p;
  a.cl_con_start = cl_con_start.p;
  a.cl_con_pair = cl_con_pair.p;
  a.cl_con_dist = cl_con_dist.p;
  a.settle_atoms = settle_atoms.p;
  a.settle_param = settle_param.p;
  a.sys_of_atom = sys_of_atom.p;
  a.sys_atom_start = sys_atom_start.p;
  a.integ = integ.p;
  a.step_base = step_base.p;
  a.step_offset = step_offset;
  a.posq = posq.p;
  a.vel = vel.p;
  a.force = force.p;
  a.noise = noise.p;
  a.origin = origin.p;
  a.disp = disp.p;
  a.diag = diag.p;
  a.ke_post = ke_post.p;
  a.ke_early = ke_early.p;
  a.saved_posq = saved_posq.p;
  a.spos = spos.p;
  a.rank = rank.p;
  a.wrap = wrap.p;
  return a;
}

SurrogateArgs Engine::sargs() {
  SurrogateArgs m{};
  m.n_systems = S;
  m.master = mlp_master.p;
  m.adam_m = mlp_m.p;
  m.adam_v = mlp_v.p;
  m.wbf = mlp_wbf.p;
  m.replay = mlp_replay.p;
  m.baro = baro.p;
  m.energies = energies.p;
  m.sysd = sysd.p;
  m.lr = learned_lr;
  m.steps = learned_steps;
  return m;
}

// Stage 1 of the learned barostat on every system (after the energy evaluation of the
// current state); whether any system's move still needs the exact evaluation.
bool Engine::surrogate_stage1() {
  launch_surrogate_stage1(bargs(), sargs(), stream);
  kernel_launches += 1;
  std::vector<double> b((size_t)S * N_BARO);
  CUDA_OK(cudaMemcpyAsync(b.data(), baro.p, sizeof(double) * b.size(), cudaMemcpyDeviceToHost, stream));
  sync();
  bool exact = false;
  for (int s = 0; s < S; ++s) {
    const double *x = b.data() + (size_t)s * N_BARO;
    if (x[B_ACTIVE] == 0.0) continue;
    if (x[B_LEARNED] == 0.0 || (x[B_REFUSED] == 0.0 && x[B_SCREENED] == 0.0)) exact = true;
  }
  if (exact) exact_passes++;
  else skipped_passes++;
  return exact;
}

void Engine::surrogate_train() {
  launch_surrogate_train(sargs(), stream);
  kernel_launches += 1;
}

BaroArgs Engine::bargs() const {
  BaroArgs a{};
  a.n_systems = S;
  a.n_atoms = N;
  a.n_molecules = n_molecules_total;
  a.posq = posq.p;
  a.saved_posq = saved_posq.p;
  a.force = force.p;
  a.saved_force = saved_force.p;
  a.mol_start = mol_start.p;
  a.mol_atoms = mol_atoms.p;
  a.sys_of_atom = sys_of_atom.p;
  a.sys = sys.p;
  a.sysd = sysd.p;
  a.baro = baro.p;
  a.energies = energies.p;
  a.saved_energies = saved_energies.p;
  a.masses = masses.p;
  a.disp = disp.p;
  a.keep_lists = 0;
  a.wrap = wrap.p;
  a.saved_wrap = saved_wrap.p;
  a.origin = origin.p;
  a.saved_origin = saved_origin.p;
  a.spos = spos.p;
  a.rank = rank.p;
  a.allow = list_allow.p;
  a.saved_allow = saved_allow.p;
  a.rebuilt = list_rebuilt.p;
  a.spread_bits = spread_bits.p;
  return a;
}

// ------------------------------------------------------------------------ operations
void Engine::record_forces(int rebuild, bool energy) {
  const LaunchCtx c = ctx();
  // The reciprocal-space chain up to the convolved grid only reads positions, so it runs
  // concurrently with the list rebuild and the pair and bonded kernels. The gather adds into
  // the force array (and reads the cell order the rebuild writes). With group-pair rows every
  // force is an integer atomic add, so the gather joins that branch as soon as the array is
  // cleared and the rebuild is done, beside the pair kernel; the per-atom-row pair kernel
  // stores its atoms' forces, so there the gather waits for both branches.
  const bool gather_beside = pme_on && c.pair_list != 1;
  if (pme_on) {
    CUDA_OK(cudaEventRecord(ev_fork, stream));
    CUDA_OK(cudaStreamWaitEvent(side, ev_fork, 0));
    launch_pme_grid(c, energy, side);
    if (!gather_beside) CUDA_OK(cudaEventRecord(ev_join, side));
  }
  if (rebuild == REBUILD_FORCED) {
    launch_rebuild_reset(required.p, required_max.p, disp.p, list_allow.p, list_rebuilt.p, S, list_builds.p + 1,
                         nullptr, stream);  // disp slot 0: since rebuild
    launch_rebuild(c, stream);
    recorded += 1 + rebuild_launches(c);
  } else if (rebuild == REBUILD_IF_STALE) {
    record_conditional_rebuild(c);  // its decision kernel also clears the force array
  }
  LaunchCtx nb = c;
  nb.force_cleared = rebuild == REBUILD_IF_STALE;
  if (gather_beside) {
    if (!nb.force_cleared) {
      CUDA_OK(cudaMemsetAsync(force.p, 0, sizeof(unsigned long long) * 3 * (size_t)N, stream));
      nb.force_cleared = true;
    }
    CUDA_OK(cudaEventRecord(ev_clear, stream));
    CUDA_OK(cudaStreamWaitEvent(side, ev_clear, 0));
    launch_pme_gather(c, side);
    CUDA_OK(cudaEventRecord(ev_join, side));
  }
  launch_nonbonded(nb, energy, nb_lanes, stream);
  launch_bonded(c, energy, stream);
  if (pme_on) {
    CUDA_OK(cudaStreamWaitEvent(stream, ev_join, 0));
    if (!gather_beside) launch_pme_gather(c, stream);
  }
  recorded += nonbonded_launches(c, energy) + (n_bonds + n_angles + n_tors + n_rest > 0 ? 1 : 0) + pme_launches(c);
  if (energy) {
    launch_molecular_virial(c, stream);
    launch_energy_reduce(segments.p, n_segments, seg_out.p, energies.p, sysd.p, S, stream);
    recorded += 3;
  }
}

// The rebuild as the body of an IF node of the graph being captured on `stream`: a one-block
// kernel sets the condition from the displacement the integrator just reduced, and the body
// (reset + cell and neighbour kernels) is captured into the node's child graph on `cond`.
// The body's kernels are counted when they run (list_builds), not here.
void Engine::record_conditional_rebuild(const LaunchCtx &c) {
  cudaStreamCaptureStatus status;
  cudaGraph_t graph;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  CUDA_OK(cudaStreamGetCaptureInfo(stream, &status, nullptr, &graph, &deps, &ndeps));
  if (status != cudaStreamCaptureStatusActive)
    throw Error(RMD_ERR_CUDA, "a conditional rebuild can only be recorded into a captured graph");
  cudaGraphConditionalHandle handle;
  CUDA_OK(cudaGraphConditionalHandleCreate(&handle, graph, 0, 0));
  launch_rebuild_decide(handle, disp.p, list_allow.p, sys.p, S, stale.p, list_builds.p,
                        c.pair_list != 1 ? force.p : nullptr, N, stream);
  recorded += 1;
  CUDA_OK(cudaStreamGetCaptureInfo(stream, &status, nullptr, &graph, &deps, &ndeps));
  cudaGraphNodeParams params = {};
  params.type = cudaGraphNodeTypeConditional;
  params.conditional.handle = handle;
  params.conditional.type = cudaGraphCondTypeIf;
  params.conditional.size = 1;
  cudaGraphNode_t node;
  CUDA_OK(cudaGraphAddNode(&node, graph, deps, ndeps, &params));
  CUDA_OK(cudaStreamUpdateCaptureDependencies(stream, &node, 1, cudaStreamSetCaptureDependencies));
  cudaGraph_t body = params.conditional.phGraph_out[0];
  CUDA_OK(cudaStreamBeginCaptureToGraph(cond, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  LaunchCtx only = c;  // the systems of the batch that have gone stale
  only.rebuild_only = stale.p;
  launch_rebuild_reset(required.p, required_max.p, disp.p, list_allow.p, list_rebuilt.p, S, list_builds.p + 1,
                       stale.p, cond);
  launch_rebuild(only, cond);
  cudaGraph_t captured;
  CUDA_OK(cudaStreamEndCapture(cond, &captured));
}

void Engine::evaluate(bool rebuild, bool energy) {
  energy_fresh = false;
  const long long before = recorded;
  record_forces(rebuild, energy);
  kernel_launches += recorded - before;
  CUDA_OK(cudaGetLastError());
}

// A volume move. keep_lists (step graphs with lists rebuilt on demand): the trial state is
// evaluated on the current lists when the displacement check, with the move's allowance,
// finds them still valid (the atoms' wraps and origins are scaled with them, and restored on
// a rejection); otherwise, and outside a graph, the trial rebuilds them.
void Engine::record_barostat(bool keep_lists) {
  BaroArgs b = bargs();
  b.keep_lists = keep_lists ? 1 : 0;
  launch_baro_propose(b, stream);
  launch_baro_scale(b, stream);
  if (keep_lists) {
    launch_baro_allow(b, stream);
    recorded += 1;
  }
  record_forces(keep_lists ? REBUILD_IF_STALE : REBUILD_FORCED, true);
  if (learned) {
    launch_surrogate_reverse(b, sargs(), stream);
    recorded += 1;
  }
  launch_baro_decide(b, stream);
  launch_baro_restore(b, stream);
  recorded += 4;
}

void Engine::set_state(int s, const double *pos, const double *vel_in, int64_t step, int supplied) {
  energy_fresh = false;
  HostSystem &h = hs[s];
  // constraintToleranceFloor (clusters.js:136-148)
  double span = 0;
  for (int k = 0; k < 3 * h.n; ++k) span = std::max(span, std::fabs(pos[k]));
  h.tol_floor = std::isfinite(h.min_constraint) ? 4.0 * span * std::ldexp(1.0, -24) / h.min_constraint : 0.0;
  h.tolerance = std::max(h.requested_tol, h.tol_floor);
  sync();  // the staging buffer may still feed an earlier call's copies
  char *stage = staging(sizeof(float4) * 2 * (size_t)h.n + 16);
  float4 *p = reinterpret_cast<float4 *>(stage), *v = p + h.n;
  for (int i = 0; i < h.n; ++i) {
    p[i] = make_float4((float)pos[3 * i], (float)pos[3 * i + 1], (float)pos[3 * i + 2], (float)h.charges[i]);
    v[i] = make_float4(vel_in ? (float)vel_in[3 * i] : 0.f, vel_in ? (float)vel_in[3 * i + 1] : 0.f,
                       vel_in ? (float)vel_in[3 * i + 2] : 0.f, h.masses[i] > 0 ? (float)(1.0 / h.masses[i]) : 0.f);
  }
  long long *sb = reinterpret_cast<long long *>(v + h.n);
  float *tol = reinterpret_cast<float *>(sb + 1);
  int *sup = reinterpret_cast<int *>(tol + 1);
  *sb = step;
  *tol = (float)h.tolerance;
  *sup = supplied;
  CUDA_OK(cudaMemcpyAsync(posq.p + h.atom_start, p, sizeof(float4) * h.n, cudaMemcpyHostToDevice, stream));
  CUDA_OK(cudaMemcpyAsync(vel.p + h.atom_start, v, sizeof(float4) * h.n, cudaMemcpyHostToDevice, stream));
  CUDA_OK(cudaMemcpyAsync(step_base.p + s, sb, sizeof(long long), cudaMemcpyHostToDevice, stream));
  // the integrator's tolerance and noise source of this system (two fields of its DevInteg)
  char *di = reinterpret_cast<char *>(integ.p + s);
  CUDA_OK(cudaMemcpyAsync(di + offsetof(DevInteg, tolerance), tol, sizeof(float), cudaMemcpyHostToDevice, stream));
  CUDA_OK(cudaMemcpyAsync(di + offsetof(DevInteg, supplied_noise), sup, sizeof(int), cudaMemcpyHostToDevice, stream));
  CUDA_OK(cudaMemsetAsync(diag.p + 4 * s, 0, sizeof(int) * 4, stream));
  sync();
  h.step = step;
  h.steps_since_rebuild = 1LL << 40;
  h.kinetic_sampled_in_step = false;
}

int Engine::check_capacity() {
  // the last build's requirement, and the largest of the builds before it since the last check;
  // the rows the pair loop walks are what diagnostics report
  std::vector<int> req(S), earlier(S);
  auto read_required = [&]() {
    std::vector<int> both(2 * (size_t)S);
    CUDA_OK(cudaMemcpy(both.data(), required.p, sizeof(int) * both.size(), cudaMemcpyDeviceToHost));
    for (int s = 0; s < S; ++s) req[s] = std::max(both[s], both[S + s]);
  };
  read_required();
  capacity_grew = false;
  CUDA_OK(cudaMemcpy(earlier.data(), required_max.p, sizeof(int) * S, cudaMemcpyDeviceToHost));
  CUDA_OK(cudaMemset(required_max.p, 0, sizeof(int) * S));
  bool grow = false;
  int worst = 0;
  for (int s = 0; s < S; ++s) {
    const int most = std::max(req[s], earlier[s]);
    hs[s].last_required = req[s];
    hs[s].worst_required = std::max(hs[s].worst_required, most);
    worst = std::max(worst, most);
    if (most > hs[s].capacity) {
      hs[s].capacity = grown_capacity(hs[s].capacity, most);
      hs[s].neighbour_growths++;
      grow = true;
    }
  }
  if (grow) {
    allocate_neighbours();
    evaluate(true, false);
    sync();
    CUDA_OK(cudaMemset(required_max.p, 0, sizeof(int) * S));
    read_required();
    capacity_grew = true;
    for (int s = 0; s < S; ++s) {
      if (req[s] > hs[s].capacity)
        throw Error(RMD_ERR_NEIGHBOUR_OVERFLOW,
                    "the neighbour list needed " + std::to_string(req[s]) + " slots per atom and the capacity is " +
                        std::to_string(hs[s].capacity) + ". Pairs were dropped, so the forces from this build are "
                        "not usable. Rebuild with a larger neighbourSlack, or a smaller skin.");
      hs[s].last_required = req[s];
    }
  }
  return worst;
}

void Engine::drop_graphs() {
  for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
  graphs.clear();
  graph_launches.clear();
}

namespace {
// Shapes chosen per workload, kept for the life of the process so that engines of the same
// shape (a benchmark's repeated runs, a batch rebuilt after a restart) tune once.
std::mutex g_tune_mutex;
std::map<std::string, std::array<int, 3>> g_tuned;
}  // namespace

// The kernel-shape autotuner. Three launch shapes change speed but not results (neighbour
// rows are the same for every group size; fixed-point pair forces and the fixed-point charge
// grid are independent of summation order): atoms per neighbour-search warp (4, 8, 16),
// lanes per atom in the pair loop (8, 16, 32) and atoms per spreading block (4, 8, 16).
// Each candidate is timed with CUDA events on the engine's stream over a few launches on the
// engine's own current state, the fastest is kept, and the choice is cached by workload
// shape (atoms, systems, cells, PME grids and order, accumulation mode).
bool Engine::autotune() {
  if (!(tune_group || tune_lanes || tune_spread)) return false;
  // captured step graphs hold the shapes they were recorded with: they stay valid (and are
  // replayed without re-capture by the next run) unless the tuned shapes change
  const std::array<int, 3> before = {group_atoms, nb_lanes, spread_atoms};
  auto keep_or_drop_graphs = [&]() {
    if (std::array<int, 3>{group_atoms, nb_lanes, spread_atoms} != before) drop_graphs();
  };
  std::string key = std::to_string(S) + ":" + std::to_string(N) + ":" + std::to_string(n_cells_total) + ":" +
                    std::to_string(pme_order) + ":" + std::to_string(pair_fixed) + ":" + std::to_string(pair_list);
  for (auto &h : hs) key += ":" + std::to_string(h.grid[0] * 100000LL + h.grid[1] * 1000LL + h.grid[2]);
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      if (tune_group) group_atoms = it->second[0];
      if (tune_lanes) nb_lanes = it->second[1];
      if (tune_spread) spread_atoms = it->second[2];
      keep_or_drop_graphs();
      return false;
    }
  }
  cudaEvent_t a, b;
  CUDA_OK(cudaEventCreate(&a));
  CUDA_OK(cudaEventCreate(&b));
  auto time = [&](const std::function<void()> &one) {
    constexpr int reps = 5;
    one();  // warm
    CUDA_OK(cudaEventRecord(a, stream));
    for (int k = 0; k < reps; ++k) one();
    CUDA_OK(cudaEventRecord(b, stream));
    CUDA_OK(cudaEventSynchronize(b));
    float ms = 0;
    CUDA_OK(cudaEventElapsedTime(&ms, a, b));
    return (double)ms / reps;
  };
  const int groups[3] = {4, 8, 16}, spreads[3] = {4, 8, 16};
  int lanes[3] = {8, 16, 32};
  if (pair_list != 1) lanes[0] = 32, lanes[1] = 64, lanes[2] = 128;  // 1, 2 or 4 warps a group row
  if (tune_group) {
    double best = 1e30;
    int pick = group_atoms;
    for (int k = 0; k < 3; ++k) {
      group_atoms = groups[k];
      const LaunchCtx c = ctx();
      tune_ms[k] = time([&]() { launch_rebuild(c, stream); });
      if (tune_ms[k] < best) best = tune_ms[k], pick = groups[k];
    }
    group_atoms = pick;
    // leave the lists as the chosen shape builds them (they are the same for every shape)
    const LaunchCtx c = ctx();
    launch_rebuild(c, stream);
  }
  if (tune_lanes) {
    double best = 1e30;
    int pick = nb_lanes;
    const LaunchCtx c = ctx();
    for (int k = 0; k < 3; ++k) {
      tune_ms[3 + k] = time([&]() { launch_nonbonded(c, false, lanes[k], stream); });
      if (tune_ms[3 + k] < best) best = tune_ms[3 + k], pick = lanes[k];
    }
    nb_lanes = pick;
  }
  if (tune_spread && pme_on) {
    double best = 1e30;
    int pick = spread_atoms;
    for (int k = 0; k < 3; ++k) {
      spread_atoms = spreads[k];
      const LaunchCtx c = ctx();
      tune_ms[6 + k] = time([&]() { launch_spread_only(c, stream); });
      if (tune_ms[6 + k] < best) best = tune_ms[6 + k], pick = spreads[k];
    }
    spread_atoms = pick;
    CUDA_OK(cudaMemsetAsync(fixed_grid.p, 0, fixed_grid.bytes(), stream));  // the z pass expects it clear
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  CUDA_OK(cudaGetLastError());
  sync();
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tuned[key] = {group_atoms, nb_lanes, spread_atoms};
  }
  keep_or_drop_graphs();
  return true;
}

void Engine::initialise() {
  evaluate(true, false);
  sync();
  for (auto &h : hs) h.steps_since_rebuild = 0;
  check_capacity();
  // the forces from a clean evaluation when the autotuner's timed pair-loop launches added into
  // them (every launch shape gives the same forces, so a cached choice keeps the first ones)
  if (autotune()) {
    evaluate(false, false);
    sync();
  }
  // kinetic energies of the current velocities, for energy() before any step
  launch_integrate(iargs(0), INT_CLOSE_KINETIC, stream);
  kernel_launches += 1;
  sync();
}

// The captured graph of a block of n steps (with a volume move first, and an energy-enabled
// last evaluation), captured and instantiated on first use and kept by its rebuild pattern.
std::map<std::string, cudaGraphExec_t>::iterator Engine::block_graph(int n, bool barostat, bool energy_last) {
  // rebuild pattern, identical for every system of the batch (the smallest interval wins)
  int interval = 1 << 30;
  int64_t since = 1LL << 40;
  for (auto &h : hs) {
    interval = std::min(interval, h.rebuild_interval);
    since = std::min<int64_t>(since, h.steps_since_rebuild);
  }
  // A volume move's trial evaluation rebuilds the lists at the scaled positions and restarts
  // the displacement check from them: an accepted move keeps them, and after a rejected one the
  // check sees the restored positions' distance from the trial ones, so on demand the step after
  // a move asks the device like any other. The host schedule rebuilds after every move.
  if (barostat && !on_demand) since = 1LL << 40;
  std::string key = "n" + std::to_string(n) + (barostat ? "B" : "") + (energy_last ? "E" : "") + ":";
  std::vector<char> rebuild(n, REBUILD_NONE);
  if (on_demand) {
    // a list from before a box change, a new state or a capacity change is not measured by
    // the displacement check: build it; every other step asks the device
    for (int k = 0; k < n; ++k) rebuild[k] = REBUILD_IF_STALE;
    if (since >= (1LL << 39) && !barostat) rebuild[0] = REBUILD_FORCED;
    key += rebuild[0] == REBUILD_FORCED ? "F" : "C";
  } else {
    for (int k = 0; k < n; ++k) {
      if (since >= interval) {
        rebuild[k] = REBUILD_FORCED;
        since = 0;
      }
      since++;
      key.push_back(rebuild[k] ? 'r' : '.');
    }
  }
  auto it = graphs.find(key);
  if (it == graphs.end()) {
    cudaGraph_t graph;
    const long long before = recorded;
    CUDA_OK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    CUDA_OK(cudaMemsetAsync(disp.p + S, 0, sizeof(unsigned) * S, stream));  // slot 1: since block start
    if (barostat) record_barostat(on_demand);
    for (int k = 0; k < n; ++k) {
      int mode = (k == 0 ? INT_OPEN : (INT_CLOSE | INT_OPEN));
      if (k == n - 1) mode |= INT_OPEN_KINETIC;
      launch_integrate(iargs(k), mode, stream);
      record_forces(rebuild[k], energy_last && k == n - 1);
    }
    launch_integrate(iargs(n - 1), INT_CLOSE | INT_CLOSE_KINETIC, stream);
    launch_advance_steps(step_base.p, S, n, stream);
    recorded += n + 2;
    CUDA_OK(cudaStreamEndCapture(stream, &graph));
    graph_launches[key] = recorded - before;
    cudaGraphExec_t exec;
    CUDA_OK(cudaGraphInstantiate(&exec, graph, 0));
    CUDA_OK(cudaGraphDestroy(graph));
    it = graphs.emplace(key, exec).first;
  }
  return it;
}

void Engine::run_block(int n, bool barostat, bool energy_last) {
  auto it = block_graph(n, barostat, energy_last);
  const std::string key = it->first;
  CUDA_OK(cudaGraphLaunch(it->second, stream));
  kernel_launches += graph_launches[key];
  energy_fresh = energy_last;
  // host bookkeeping mirrors the device
  int interval = 1 << 30;
  for (auto &h : hs) interval = std::min(interval, h.rebuild_interval);
  for (auto &h : hs) {
    int64_t s2 = barostat ? (1LL << 40) : h.steps_since_rebuild;
    if (on_demand) {
      s2 = 1;  // the device keeps the lists fresh from here on
    } else {
      for (int k = 0; k < n; ++k) {
        if (s2 >= interval) s2 = 0;
        s2++;
      }
    }
    h.steps_since_rebuild = s2;
    h.step += n;
    h.kinetic_sampled_in_step = true;
    h.kinetic_sampled_at = h.step;
  }
}

// #checkSkin (simulation.js:544-623) and #checkNeighbourCapacity (simulation.js:424-443)
void Engine::check_block(int steps) {
  std::vector<unsigned> d(2 * S);
  CUDA_OK(cudaMemcpy(d.data(), disp.p, sizeof(unsigned) * 2 * S, cudaMemcpyDeviceToHost));
  if (on_demand) {  // the rebuild bodies that ran inside the block's graph
    unsigned long long taken = 0;
    CUDA_OK(cudaMemcpy(&taken, list_builds.p, sizeof taken, cudaMemcpyDeviceToHost));
    kernel_launches += (1LL + rebuild_launches(ctx())) * (long long)(taken - conditional_builds_seen);
    conditional_builds_seen = taken;
  }
  for (int s = 0; s < S; ++s) {
    HostSystem &h = hs[s];
    float f0, f1;
    memcpy(&f0, &d[s], 4);
    memcpy(&f1, &d[S + s], 4);
    const float sq = std::max(f0, f1);
    if (!std::isfinite(f0) || !std::isfinite(f1))
      throw Error(RMD_ERR_NON_FINITE,
                  "the simulation is no longer a number: the maximum atomic displacement over the last block "
                  "went non-finite at step " + std::to_string(h.step) +
                  ". The usual causes, commonest first: a timestep too large for this system; two atoms at the "
                  "same coordinate in the input; a structure that was never minimised; or a restart whose "
                  "velocities do not belong to its positions.");
    const double worst = std::sqrt(std::max(0.0, (double)sq));
    h.worst_displacement = std::max(h.worst_displacement, worst);
    const double usage = 2.0 * worst / h.skin;
    if (on_demand) {
      // the block's largest displacement was measured before the step's rebuild decision:
      // every force evaluation used a list that the check had found valid
      h.worst_skin_usage = std::max(h.worst_skin_usage, std::min(usage, 1.0));
      continue;
    }
    h.worst_skin_usage = std::max(h.worst_skin_usage, usage);
    if (usage <= 1.0) {
      h.calm_blocks++;
      if (h.adaptive && usage < 0.4 && h.calm_blocks >= 3 && h.rebuild_interval < h.requested_rebuild) {
        h.rebuild_interval = std::min(h.requested_rebuild,
                                      std::max(h.rebuild_interval + 1, (int)std::floor(h.rebuild_interval * 1.25)));
        h.rebuild_growths++;
        h.calm_blocks = 0;
      }
      continue;
    }
    h.skin_violations++;
    h.calm_blocks = 0;
    h.steps_with_stale += steps;
    h.worst_skin_ratio = std::max(h.worst_skin_ratio, usage);
    const int shrunk = std::max(1, h.rebuild_interval / 2);
    if (h.adaptive && shrunk != h.rebuild_interval) {
      h.rebuild_interval = shrunk;
      h.rebuild_shrinks++;
    }
    h.steps_since_rebuild = 1LL << 40;
  }
  check_capacity();
}

void Engine::run(int64_t count, int block, const volatile int32_t *stop) {
  int64_t remaining = count;
  while (remaining > 0) {
    if (stop && *stop) throw Error(RMD_ERR_STOPPED, "the simulation was stopped");
    bool due = false;
    for (auto &h : hs)
      if (h.has_pressure && h.steps_since_barostat >= h.barostat_interval) due = true;
    int interval = 1 << 30;
    for (auto &h : hs) interval = std::min(interval, h.rebuild_interval);
    int n = block > 0 ? block : interval;
    n = (int)std::min<int64_t>(n, remaining);
    // the last force evaluation of a block is energy-enabled when a volume move follows
    bool next_due = false;
    for (auto &h : hs)
      if (h.has_pressure && (due ? 0 : h.steps_since_barostat) + n >= h.barostat_interval) next_due = true;
    bool exact_move = due;
    // timed runs (rmd_bench_run): L2 is flushed before each block, outside the events, and
    // the events bracket all of the block's device work: the energy evaluation and the
    // surrogate screening before a volume move, the block's graph and the training after it
    if (timing) {
      // the block's graph is captured (on first use) before the events, so host-side capture
      // and instantiation are never timed as device work
      block_graph(n, exact_move, next_due);
      if (flush) CUDA_OK(cudaMemsetAsync(flush_buffer.p, (int)(kernel_launches & 0xff), flush_buffer.n, stream));
      CUDA_OK(cudaEventRecord(ev_a, stream));
    }
    if (due) {
      // the move needs the energy at the current positions: the previous block's last
      // evaluation computed it when this move was due at its end
      if (!energy_fresh) evaluate(false, true);
      // with the learned barostat, stage 1 may screen every system's move out: the block
      // then runs without the exact trial evaluation
      if (learned) exact_move = surrogate_stage1();
    }
    run_block(n, exact_move, next_due);
    if (due && learned && exact_move) surrogate_train();
    if (timing) {
      CUDA_OK(cudaEventRecord(ev_b, stream));
      CUDA_OK(cudaEventSynchronize(ev_b));
      float ms = 0.f;
      CUDA_OK(cudaEventElapsedTime(&ms, ev_a, ev_b));
      timed_ms += ms;
    }
    sync();
    if (due) {
      for (auto &h : hs) h.steps_since_barostat = 0;
      std::vector<double> b((size_t)S * N_BARO);
      CUDA_OK(cudaMemcpy(b.data(), baro.p, sizeof(double) * b.size(), cudaMemcpyDeviceToHost));
      for (int s = 0; s < S; ++s) {
        HostSystem &h = hs[s];
        const double *bb = b.data() + (size_t)s * N_BARO;
        if (!h.has_pressure) continue;
        rmd_volume_move &m = h.last_move;
        m.attempted = 1;
        m.screened = bb[B_SCREENED] != 0.0;
        m.refused = bb[B_REFUSED] != 0.0;
        m.accepted = exact_move && bb[B_ACCEPT] != 0.0 && !m.refused && !m.screened;
        m.weight = bb[B_WEIGHT];
        m.delta_volume = bb[B_DV];
        m.length_scale = bb[B_LSCALE];
        m.old_potential = bb[B_OLD_E];
        m.new_potential = bb[B_NEW_E];
        m.volume_scale = bb[B_SCALE];
        m.acceptance_rate = bb[B_ATTEMPTS] > 0 ? bb[B_ACCEPTED] / bb[B_ATTEMPTS] : 0;
      }
    }
    for (auto &h : hs)
      if (h.has_pressure) h.steps_since_barostat += n;
    check_block(n);
    remaining -= n;
  }
}

std::vector<double> Engine::read_energies() {
  std::vector<double> e((size_t)S * N_ENERGY);
  CUDA_OK(cudaMemcpy(e.data(), energies.p, sizeof(double) * e.size(), cudaMemcpyDeviceToHost));
  return e;
}

void Engine::energy(int s, rmd_energy_report *out) {
  // forces and energies at the current positions, with the current list (no rebuild: the
  // skin keeps it valid), then the kinetic sums (simulation.js:1073-1230)
  evaluate(false, true);
  sync();
  const std::vector<double> all = read_energies();
  const double *e = all.data() + (size_t)s * N_ENERGY;
  HostSystem &h = hs[s];
  DevSysD d;
  CUDA_OK(cudaMemcpy(&d, sysd.p + s, sizeof d, cudaMemcpyDeviceToHost));
  memset(out, 0, sizeof *out);
  out->step = h.step;
  out->time = h.step * h.opt.timestep;
  out->harmonic_bond = e[E_BOND];
  out->harmonic_angle = e[E_ANGLE];
  out->periodic_torsion = e[E_TORSION];
  out->bonded = e[E_BOND] + e[E_ANGLE] + e[E_TORSION];
  out->lennard_jones = e[E_LJ];
  out->dispersion = e[E_DISPERSION];
  out->coulomb_direct = e[E_COUL_DIRECT];
  out->coulomb_reciprocal = e[E_RECIP];
  out->coulomb_self = e[E_SELF] + e[E_NET];
  out->coulomb = e[E_COUL_DIRECT] + e[E_RECIP] + e[E_SELF] + e[E_NET];
  out->position_restraint = e[E_RESTRAINT];
  out->restrained_atoms = (int)h.restraint_atoms.size();
  out->potential = e[E_POTENTIAL];
  out->kinetic = e[E_KINETIC];
  out->total = out->potential + out->kinetic;
  double kt = e[E_KINETIC];
  out->kinetic_sampled_before_closing_kick = 0;
  if (h.kinetic_sampled_in_step && h.kinetic_sampled_at == h.step && (e[E_KINETIC_EARLY] > 0 || kt <= 0)) {
    kt = e[E_KINETIC_EARLY];
    out->kinetic_sampled_before_closing_kick = 1;
  }
  out->kinetic_for_temperature = kt;
  out->temperature = 2.0 * kt / (h.dof * BOLTZMANN);
  out->volume = d.volume;
  for (int k = 0; k < 9; ++k) out->box_vectors[k] = d.box[k];
  out->volume_derivative = e[E_DUDLNV];
  if (!std::isfinite(out->potential) || !std::isfinite(out->kinetic))
    throw Error(RMD_ERR_NON_FINITE, std::string("the simulation is no longer a number: the ") +
                                        (!std::isfinite(out->potential) ? "potential" : "kinetic") +
                                        " energy went non-finite at step " + std::to_string(h.step));
}

void Engine::attempt_volume_change() {
  // energy at the current positions, then one device-side move on every system
  evaluate(false, true);
  const BaroArgs b = bargs();
  const bool exact_move = learned ? surrogate_stage1() : true;
  if (exact_move) {
    record_barostat(false);
    if (learned) surrogate_train();
  }
  CUDA_OK(cudaGetLastError());
  sync();
  for (auto &h : hs) h.steps_since_rebuild = 1LL << 40;
  std::vector<double> bb((size_t)S * N_BARO);
  CUDA_OK(cudaMemcpy(bb.data(), baro.p, sizeof(double) * bb.size(), cudaMemcpyDeviceToHost));
  // a rejected move leaves lists built in the trial box: rebuild them at the restored state
  // before anything evaluates (the reference evaluates the restored state, simulation.js:1049-1056)
  bool rejected = false;
  for (int s = 0; s < S; ++s) {
    const double *x = bb.data() + (size_t)s * N_BARO;
    if (exact_move && hs[s].has_pressure && x[B_REFUSED] == 0.0 && x[B_SCREENED] == 0.0 && x[B_ACCEPT] == 0.0)
      rejected = true;
  }
  if (rejected) {
    evaluate(true, false);
    sync();
  }
  std::vector<DevSysD> dd(S);
  CUDA_OK(cudaMemcpy(dd.data(), sysd.p, sizeof(DevSysD) * S, cudaMemcpyDeviceToHost));
  (void)b;
  for (int s = 0; s < S; ++s) {
    HostSystem &h = hs[s];
    const double *x = bb.data() + (size_t)s * N_BARO;
    rmd_volume_move &m = h.last_move;
    memset(&m, 0, sizeof m);
    if (!h.has_pressure) continue;
    m.attempted = 1;
    m.refused = x[B_REFUSED] != 0.0;
    m.screened = x[B_SCREENED] != 0.0;
    m.accepted = exact_move && !m.refused && !m.screened && x[B_ACCEPT] != 0.0;
    m.weight = x[B_WEIGHT];
    m.delta_volume = x[B_DV];
    m.length_scale = x[B_LSCALE];
    m.old_potential = x[B_OLD_E];
    m.new_potential = x[B_NEW_E];
    m.volume = dd[s].volume;
    m.volume_scale = x[B_SCALE];
    m.acceptance_rate = x[B_ATTEMPTS] > 0 ? x[B_ACCEPTED] / x[B_ATTEMPTS] : 0.0;
  }
}

double Engine::scale_volume(int s, double ls) {
  energy_fresh = false;
  // scaleVolume (simulation.js:801-811): centroid scaling and the box, then the potential
  std::vector<double> scales(S, 1.0);
  scales[s] = ls;
  CUDA_OK(cudaMemcpy(fixed_scales.p, scales.data(), sizeof(double) * S, cudaMemcpyHostToDevice));
  launch_scale_fixed(bargs(), fixed_scales.p, stream);
  DevSysD d;
  CUDA_OK(cudaMemcpy(&d, sysd.p + s, sizeof d, cudaMemcpyDeviceToHost));
  for (int k = 0; k < 9; ++k) d.box[k] *= ls;
  CUDA_OK(cudaMemcpy(sysd.p + s, &d, sizeof d, cudaMemcpyHostToDevice));
  launch_update_box(sys.p, sysd.p, S, stream);
  evaluate(true, true);
  sync();
  for (auto &h : hs) h.steps_since_rebuild = 0;
  check_capacity();
  if (capacity_grew) {  // the first evaluation dropped pairs: its energy is not the potential
    evaluate(false, true);
    sync();
  }
  return read_energies()[(size_t)s * N_ENERGY + E_POTENTIAL];
}

std::vector<float> Engine::max_forces() {
  DevArray<unsigned> bits;
  bits.alloc(S);
  bits.zero();
  launch_max_force(force.p, sys_of_atom.p, N, bits.p, stream);
  sync();
  std::vector<unsigned> b(S);
  CUDA_OK(cudaMemcpy(b.data(), bits.p, sizeof(unsigned) * S, cudaMemcpyDeviceToHost));
  bits.release();
  std::vector<float> out(S);
  for (int s = 0; s < S; ++s) memcpy(&out[s], &b[s], 4);
  return out;
}

// minimise (simulation.js:880-979): steepest descent with a backtracking line search. Every
// system of a batch keeps its own step and acceptance, and every decision is taken on the
// device (minimise.cu): one trial is one captured graph, launched in batches of 16 with the
// states read back between batches. A trial whose neighbour list overflowed is undone on the
// device; the host grows the list, re-captures and the trial runs again.
// Departure: the positions AND forces of the last accepted structure are restored after a
// rejected trial, so the next trial moves along the accepted gradient.
void Engine::minimise(int max_iterations, double force_tolerance, double max_step, double cap,
                      rmd_minimise_result *out) {
  energy_fresh = false;
  if (max_iterations <= 0) max_iterations = 200;
  if (!(force_tolerance > 0)) force_tolerance = 500;
  if (!(max_step > 0)) max_step = 0.002;
  if (!(cap > 0)) cap = 0.05;
  auto potentials = [&]() {
    evaluate(true, true);
    sync();
    for (auto &h : hs) h.steps_since_rebuild = 0;
    check_capacity();
    std::vector<double> e = read_energies(), p(S);
    for (int s = 0; s < S; ++s) p[s] = e[(size_t)s * N_ENERGY + E_POTENTIAL];
    return p;
  };
  const std::vector<double> start = potentials();
  std::vector<MinState> state(S);
  for (int s = 0; s < S; ++s) {
    state[s] = MinState{};
    state[s].potential = start[s];
    state[s].step = max_step;
  }
  DevArray<MinState> dstate;
  DevArray<float> scale;
  DevArray<unsigned> worst_bits;
  dstate.alloc(S);
  scale.alloc(S);
  worst_bits.alloc(S);
  CUDA_OK(cudaMemcpy(dstate.p, state.data(), sizeof(MinState) * S, cudaMemcpyHostToDevice));
  cudaGraphExec_t trial = nullptr;
  long long trial_kernels = 0;
  auto capture = [&]() {
    cudaGraph_t graph;
    const long long before = recorded;
    CUDA_OK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    CUDA_OK(cudaMemsetAsync(worst_bits.p, 0, sizeof(unsigned) * S, stream));
    launch_max_force(force.p, sys_of_atom.p, N, worst_bits.p, stream);
    launch_min_begin(dstate.p, worst_bits.p, scale.p, S, max_iterations, (float)force_tolerance, stream);
    launch_min_save(dstate.p, posq.p, force.p, saved_posq.p, saved_force.p, sys_of_atom.p, N, stream);
    launch_displace(posq.p, force.p, sys_of_atom.p, N, scale.p, (float)cap, stream);
    launch_integrate(iargs(0), INT_CONSTRAIN, stream);
    record_forces(true, true);
    launch_min_decide(dstate.p, energies.p, required.p, sys.p, S, stream);
    launch_min_restore(dstate.p, posq.p, force.p, saved_posq.p, saved_force.p, sys_of_atom.p, N, stream);
    recorded += 7;
    CUDA_OK(cudaStreamEndCapture(stream, &graph));
    trial_kernels = recorded - before;
    CUDA_OK(cudaGraphInstantiate(&trial, graph, 0));
    CUDA_OK(cudaGraphDestroy(graph));
  };
  capture();
  // every iteration takes at most 14 trials and one more that finds it converged; each
  // neighbour-list growth repeats one trial
  const long long limit = (long long)(max_iterations + 1) * (MIN_ATTEMPTS + 1) + 64;
  long long trials = 0;
  while (trials < limit) {
    const int batch = (int)std::min<long long>(16, limit - trials);
    for (int k = 0; k < batch; ++k) CUDA_OK(cudaGraphLaunch(trial, stream));
    trials += batch;
    kernel_launches += trial_kernels * batch;
    CUDA_OK(cudaMemcpyAsync(state.data(), dstate.p, sizeof(MinState) * S, cudaMemcpyDeviceToHost, stream));
    sync();
    bool all_done = true, grow = false;
    for (int s = 0; s < S; ++s) {
      if (!state[s].done) all_done = false;
      if (state[s].overflow) {
        HostSystem &h = hs[s];
        h.worst_required = std::max(h.worst_required, state[s].need);
        if (state[s].need > h.capacity) {  // grownPlan (cells.js:282-288)
          h.capacity = (std::max(h.capacity + 32, (int)std::ceil(state[s].need * 1.25)) + 3) & ~3;
          h.neighbour_growths++;
        }
        state[s].overflow = 0;
        state[s].need = 0;
        grow = true;
      }
    }
    if (grow) {
      // the pointers recorded in the trial graph change with the list's storage
      CUDA_OK(cudaGraphExecDestroy(trial));
      trial = nullptr;
      allocate_neighbours();
      CUDA_OK(cudaMemcpy(dstate.p, state.data(), sizeof(MinState) * S, cudaMemcpyHostToDevice));
      capture();
      continue;
    }
    if (all_done) break;
  }
  if (trial) CUDA_OK(cudaGraphExecDestroy(trial));
  dstate.release();
  worst_bits.release();
  scale.release();
  // forces at the final structure, and velocities zeroed (simulation.js:971-973)
  const std::vector<double> potential = potentials();
  std::vector<float> worst = max_forces();
  std::vector<float4> v(N);
  CUDA_OK(cudaMemcpy(v.data(), vel.p, sizeof(float4) * N, cudaMemcpyDeviceToHost));
  for (auto &x : v) x.x = x.y = x.z = 0.f;
  CUDA_OK(cudaMemcpy(vel.p, v.data(), sizeof(float4) * N, cudaMemcpyHostToDevice));
  launch_integrate(iargs(0), INT_CLOSE_KINETIC, stream);
  sync();
  if (out) {
    out->iterations = state[0].iterations;
    out->rejected = state[0].rejected;
    out->stalled = state[0].stalled;
    out->converged = worst[0] <= force_tolerance;
    out->potential = potential[0];
    out->max_force = worst[0];
    out->max_step = state[0].step;
  }
}

TrajArgs Engine::traj_args(int s, bool image) {
  const HostSystem &h = hs[s];
  TrajArgs t{};
  t.posq = posq.p;
  t.vel = vel.p;
  t.mol_start = mol_start.p;
  t.mol_atoms = mol_atoms.p;
  t.mol_of_atom = mol_of_atom.p;
  t.sysd = sysd.p;
  t.sys = s;
  t.atom_start = h.atom_start;
  t.atom_count = h.n;
  t.mol_first = mol_base[s];
  t.mol_count = mol_base[s + 1] - mol_base[s];
  t.image = image && t.mol_count > 0 ? 1 : 0;
  if (traj_shift.n < (size_t)std::max(1, t.mol_count)) traj_shift.alloc(std::max(1, t.mol_count));
  if (traj_status.n < 2) traj_status.alloc(2);
  t.shift = traj_shift.p;
  t.status = traj_status.p;
  const int none[2] = {INT_MAX, INT_MAX};
  CUDA_OK(cudaMemcpyAsync(traj_status.p, none, sizeof none, cudaMemcpyHostToDevice, stream));
  if (t.image) launch_traj_shifts(t, stream);
  return t;
}

}  // namespace rmd

// =========================================================================== C ABI
struct rmd_sim {
  rmd::Engine engine;
};

static std::string g_create_error;

template <class F>
static rmd_status guarded(rmd_sim *sim, F &&f) {
  try {
    f();
    return RMD_OK;
  } catch (const rmd::Error &e) {
    if (sim) sim->engine.last_error = e.what();
    else g_create_error = e.what();
    return e.code;
  } catch (const std::exception &e) {
    if (sim) sim->engine.last_error = e.what();
    else g_create_error = e.what();
    return RMD_ERR_CUDA;
  }
}

static rmd_status check_index(rmd_sim *sim, int32_t s) {
  if (!sim) return RMD_ERR_INVALID;
  if (s < 0 || s >= sim->engine.S) {
    sim->engine.last_error = "system index out of range";
    return RMD_ERR_INVALID;
  }
  return RMD_OK;
}

extern "C" {

void rmd_default_options(rmd_options *o) {
  memset(o, 0, sizeof *o);
  o->timestep = 0.002;
  o->temperature = 298.0;
  o->friction = 1.0;
  o->seed = 0;
  o->tolerance = 1e-5;
  o->max_constraint_iterations = 150;
  o->rebuild_interval = 20;
  o->adaptive_rebuild = 1;
  o->rebuild_on_demand = 1;
  o->pressure = RMD_NO_PRESSURE;
  o->barostat_interval = 25;
  o->dispersion_correction = 1;
  o->neighbour_slack = 2.0;
  o->ewald_tolerance = 5e-4;
  o->pme_order = 5;
  o->pair_list = 0;
}

rmd_status rmd_plan_system(const rmd_system *system, const rmd_options *options, rmd_plan *out) {
  if (!system || !out) return RMD_ERR_INVALID;
  return guarded(nullptr, [&]() {
    rmd::HostSystem h;
    if (options) {
      h.opt = *options;
    } else {
      rmd_default_options(&h.opt);
    }
    rmd::Engine::plan_system(h, *system);
    memset(out, 0, sizeof *out);
    out->skin = h.skin;
    out->cutoff = h.cutoff;
    out->list_cutoff = h.list_cutoff;
    out->cell_count = 1;
    out->stencil_cells = 1;
    for (int d = 0; d < 3; ++d) {
      out->counts[d] = h.counts[d];
      out->cell_count *= h.counts[d];
      out->stencil_cells *= h.counts[d] >= 3 ? 3 : h.counts[d];  // axisOffsets (cells.js:25-29)
      out->grid[d] = h.grid[d];
    }
    out->estimated_neighbours = h.estimated_neighbours;
    const double slack = h.opt.neighbour_slack > 0 ? h.opt.neighbour_slack : 2.0;
    out->max_neighbours = h.opt.max_neighbours > 0
                              ? h.opt.max_neighbours
                              : std::max(32, (int)std::ceil(h.estimated_neighbours * slack));
    out->capacity = h.capacity;
    out->mean_occupancy = (double)h.n / out->cell_count;
    out->alpha = h.alpha;
    out->order = h.order;
  });
}

int32_t rmd_grown_capacity(int32_t capacity, int32_t required) {
  return capacity > 0 && required >= 0 ? rmd::grown_capacity(capacity, required) : 0;
}

rmd_status rmd_create_batch(int32_t count, const rmd_system *systems, const rmd_options *options,
                            rmd_sim **out) {
  *out = nullptr;
  if (count <= 0 || !systems) {
    g_create_error = "rmd_create_batch needs at least one system";
    return RMD_ERR_INVALID;
  }
  rmd_sim *sim = new rmd_sim();
  rmd_options defaults;
  rmd_default_options(&defaults);
  std::vector<rmd_options> per(count, options ? options[0] : defaults);
  if (options)
    for (int s = 0; s < count; ++s) per[s] = options[s];
  rmd_status st = guarded(nullptr, [&]() { sim->engine.build(count, systems, per.data()); });
  if (st != RMD_OK) {
    delete sim;
    return st;
  }
  *out = sim;
  return RMD_OK;
}

rmd_status rmd_create(const rmd_system *system, const rmd_options *options, rmd_sim **out) {
  return rmd_create_batch(1, system, options, out);
}

int32_t rmd_system_count(const rmd_sim *sim) { return sim ? sim->engine.S : 0; }

rmd_status rmd_set_state_at(rmd_sim *sim, int32_t s, const double *positions, const double *velocities,
                            int64_t step, int32_t supplied_noise) {
  if (rmd_status c = check_index(sim, s)) return c;
  if (!positions) return RMD_ERR_INVALID;
  return guarded(sim, [&]() { sim->engine.set_state(s, positions, velocities, step, supplied_noise); });
}

rmd_status rmd_set_state(rmd_sim *sim, const double *positions, const double *velocities, int64_t step,
                         int32_t supplied_noise) {
  return rmd_set_state_at(sim, 0, positions, velocities, step, supplied_noise);
}

rmd_status rmd_set_noise_at(rmd_sim *sim, int32_t s, const float *noise) {
  if (rmd_status c = check_index(sim, s)) return c;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    CUDA_OK(cudaMemcpy(e.noise.p + 3 * (size_t)e.hs[s].atom_start, noise, sizeof(float) * 3 * e.hs[s].n,
                       cudaMemcpyHostToDevice));
  });
}

rmd_status rmd_set_noise(rmd_sim *sim, const float *noise) { return rmd_set_noise_at(sim, 0, noise); }

rmd_status rmd_initialise(rmd_sim *sim) {
  if (!sim) return RMD_ERR_INVALID;
  return guarded(sim, [&]() { sim->engine.initialise(); });
}

rmd_status rmd_run(rmd_sim *sim, int64_t count, int32_t block_size, const volatile int32_t *stop_flag,
                   int64_t *step_out) {
  if (!sim) return RMD_ERR_INVALID;
  rmd_status st = guarded(sim, [&]() { sim->engine.run(count, block_size, stop_flag); });
  if (step_out) *step_out = sim->engine.hs[0].step;
  return st;
}

rmd_status rmd_attempt_volume_change(rmd_sim *sim, rmd_volume_move *out) {
  if (!sim) return RMD_ERR_INVALID;
  rmd_status st = guarded(sim, [&]() { sim->engine.attempt_volume_change(); });
  if (out) *out = sim->engine.hs[0].last_move;
  return st;
}

rmd_status rmd_last_volume_move_at(rmd_sim *sim, int32_t s, rmd_volume_move *out) {
  if (rmd_status c = check_index(sim, s)) return c;
  *out = sim->engine.hs[s].last_move;
  return RMD_OK;
}

rmd_status rmd_scale_volume(rmd_sim *sim, double length_scale, double *potential_out) {
  if (!sim) return RMD_ERR_INVALID;
  return guarded(sim, [&]() {
    const double e = sim->engine.scale_volume(0, length_scale);
    if (potential_out) *potential_out = e;
  });
}

rmd_status rmd_energy_at(rmd_sim *sim, int32_t s, rmd_energy_report *out) {
  if (rmd_status c = check_index(sim, s)) return c;
  return guarded(sim, [&]() { sim->engine.energy(s, out); });
}

rmd_status rmd_energy(rmd_sim *sim, rmd_energy_report *out) { return rmd_energy_at(sim, 0, out); }

rmd_status rmd_read_state_at(rmd_sim *sim, int32_t s, float *positions, float *velocities, float *forces,
                             double box_vectors[9], double *volume) {
  if (rmd_status c = check_index(sim, s)) return c;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    const auto &h = e.hs[s];
    // every requested array in one round of asynchronous copies into page-locked staging
    e.sync();
    const size_t n = (size_t)h.n;
    char *stage = e.staging(sizeof(float4) * 2 * n + sizeof(long long) * 3 * n + sizeof(rmd::DevSysD));
    float4 *p = reinterpret_cast<float4 *>(stage), *v = p + n;
    long long *f = reinterpret_cast<long long *>(v + n);
    rmd::DevSysD *d = reinterpret_cast<rmd::DevSysD *>(f + 3 * n);
    if (positions)
      CUDA_OK(cudaMemcpyAsync(p, e.posq.p + h.atom_start, sizeof(float4) * n, cudaMemcpyDeviceToHost, e.stream));
    if (velocities)
      CUDA_OK(cudaMemcpyAsync(v, e.vel.p + h.atom_start, sizeof(float4) * n, cudaMemcpyDeviceToHost, e.stream));
    if (forces)
      for (int c = 0; c < 3; ++c)
        CUDA_OK(cudaMemcpyAsync(f + c * n, e.force.p + (size_t)c * e.N + h.atom_start, sizeof(long long) * n,
                                cudaMemcpyDeviceToHost, e.stream));
    if (box_vectors || volume)
      CUDA_OK(cudaMemcpyAsync(d, e.sysd.p + s, sizeof(rmd::DevSysD), cudaMemcpyDeviceToHost, e.stream));
    e.sync();
    for (size_t i = 0; i < n; ++i) {
      if (positions) {
        positions[3 * i] = p[i].x;
        positions[3 * i + 1] = p[i].y;
        positions[3 * i + 2] = p[i].z;
      }
      if (velocities) {
        velocities[3 * i] = v[i].x;
        velocities[3 * i + 1] = v[i].y;
        velocities[3 * i + 2] = v[i].z;
      }
      if (forces)
        for (int c = 0; c < 3; ++c) forces[3 * i + c] = (float)((double)f[c * n + i] / rmd::FORCE_SCALE);
    }
    if (box_vectors)
      for (int k = 0; k < 9; ++k) box_vectors[k] = d->box[k];
    if (volume) *volume = d->volume;
  });
}

rmd_status rmd_read_state(rmd_sim *sim, float *positions, float *velocities, float *forces,
                          double box_vectors[9], double *volume) {
  return rmd_read_state_at(sim, 0, positions, velocities, forces, box_vectors, volume);
}

rmd_status rmd_read_positions(rmd_sim *sim, float *positions) {
  return rmd_read_state_at(sim, 0, positions, nullptr, nullptr, nullptr, nullptr);
}

rmd_status rmd_diagnostics_at(rmd_sim *sim, int32_t s, rmd_diagnostics_report *out) {
  if (rmd_status c = check_index(sim, s)) return c;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    const auto &h = e.hs[s];
    e.sync();
    int dg[4];
    CUDA_OK(cudaMemcpy(dg, e.diag.p + 4 * s, sizeof dg, cudaMemcpyDeviceToHost));
    std::vector<double> b(rmd::N_BARO);
    CUDA_OK(cudaMemcpy(b.data(), e.baro.p + (size_t)s * rmd::N_BARO, sizeof(double) * rmd::N_BARO,
                       cudaMemcpyDeviceToHost));
    rmd::DevSys ds;
    rmd::DevSysD dd;
    CUDA_OK(cudaMemcpy(&ds, e.sys.p + s, sizeof ds, cudaMemcpyDeviceToHost));
    CUDA_OK(cudaMemcpy(&dd, e.sysd.p + s, sizeof dd, cudaMemcpyDeviceToHost));
    memset(out, 0, sizeof *out);
    out->max_shake_iterations = dg[0];
    out->shake_hit_iteration_cap = dg[1];
    out->rattle_hit_iteration_cap = dg[2];
    float res;
    memcpy(&res, &dg[3], 4);
    out->worst_stalled_residual = res;
    out->neighbour_required = h.last_required;
    out->neighbour_capacity = h.capacity;
    out->worst_neighbour_required = h.worst_required;
    out->neighbour_growths = h.neighbour_growths;
    out->skin = h.skin;
    out->worst_displacement = h.worst_displacement;
    out->worst_skin_ratio = h.worst_skin_ratio;
    out->skin_violations = h.skin_violations;
    out->steps_with_stale_list = h.steps_with_stale;
    out->rebuild_interval = h.rebuild_interval;
    out->requested_rebuild_interval = h.requested_rebuild;
    out->rebuild_shrinks = h.rebuild_shrinks;
    out->rebuild_growths = h.rebuild_growths;
    out->worst_skin_usage = h.worst_skin_usage;
    out->adaptive_rebuild = h.adaptive;
    out->volume = dd.volume;
    out->barostat_attempts = (int)b[rmd::B_ATTEMPTS];
    out->barostat_accepted = (int)b[rmd::B_ACCEPTED];
    out->barostat_refused = (int)b[rmd::B_REFUSALS];
    out->barostat_screened = (int)b[rmd::B_SCREENED_TOTAL];
    out->barostat_exact_evaluations = (int)b[rmd::B_EXACT_EVALS];
    out->volume_scale = b[rmd::B_SCALE];
    out->constraint_tolerance = h.tolerance;
    out->requested_tolerance = h.requested_tol;
    out->tolerance_floor = h.tol_floor;
    for (int k = 0; k < 3; ++k) {
      out->cell_counts[k] = ds.cell_counts[k];
      out->pme_grid[k] = h.grid[k];
    }
    out->pme_alpha = h.alpha;
    out->pme_order = h.order;
    out->cluster_count = h.n_clusters;
    out->settle_count = h.n_settle;
    size_t bytes = 0;
    bytes += e.posq.bytes() * 4 + e.force.bytes() * 2 + e.nbr.bytes() + e.gnbr.bytes() + e.fixed_grid.bytes() + e.half.bytes() +
             e.real_grid.bytes() + e.cell_atoms.bytes() * 2 + e.e_lj.bytes() * 4;
    out->device_bytes = (int64_t)bytes;
    unsigned long long builds[2] = {0, 0};
    CUDA_OK(cudaMemcpy(builds, e.list_builds.p, sizeof builds, cudaMemcpyDeviceToHost));
    out->list_builds = (int64_t)builds[1];
    out->rebuild_on_demand = e.on_demand ? 1 : 0;
    out->pair_list = e.pair_list;
  });
}

rmd_status rmd_diagnostics(rmd_sim *sim, rmd_diagnostics_report *out) { return rmd_diagnostics_at(sim, 0, out); }

rmd_status rmd_minimise(rmd_sim *sim, int32_t max_iterations, double force_tolerance, double max_step,
                        double max_displacement, rmd_minimise_result *out) {
  if (!sim) return RMD_ERR_INVALID;
  return guarded(sim, [&]() { sim->engine.minimise(max_iterations, force_tolerance, max_step, max_displacement, out); });
}

void rmd_destroy(rmd_sim *sim) { delete sim; }

const char *rmd_last_error(const rmd_sim *sim) {
  return sim ? sim->engine.last_error.c_str() : g_create_error.c_str();
}

rmd_status rmd_debug_cells(rmd_sim *sim, int32_t s, int32_t counts[3], int32_t *cstart, int32_t *catoms) {
  if (rmd_status c = check_index(sim, s)) return c;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    e.sync();
    rmd::DevSys ds;
    CUDA_OK(cudaMemcpy(&ds, e.sys.p + s, sizeof ds, cudaMemcpyDeviceToHost));
    for (int k = 0; k < 3; ++k) counts[k] = ds.cell_counts[k];
    const int cells = ds.cell_counts[0] * ds.cell_counts[1] * ds.cell_counts[2];
    if (cstart) CUDA_OK(cudaMemcpy(cstart, e.cell_start.p + ds.cell_start_base, sizeof(int) * (cells + 1),
                                   cudaMemcpyDeviceToHost));
    if (catoms) {
      CUDA_OK(cudaMemcpy(catoms, e.cell_atoms.p + ds.atom_start, sizeof(int) * ds.atom_count, cudaMemcpyDeviceToHost));
      for (int i = 0; i < ds.atom_count; ++i) catoms[i] -= ds.atom_start;
    }
  });
}

rmd_status rmd_debug_neighbours(rmd_sim *sim, int32_t s, int32_t *capacity, int32_t *counts, int32_t *rows,
                                int32_t *req) {
  if (rmd_status c = check_index(sim, s)) return c;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    e.sync();
    if (e.pair_list == 0)
      throw rmd::Error(RMD_ERR_INVALID, "the per-atom rows are not built with pair_list 0 (group-pair rows); create "
                                        "the simulation with pair_list 2 to build and inspect them");
    const auto &h = e.hs[s];
    const auto &ds = e.h_sys[s];
    if (capacity) *capacity = ds.nbr_capacity;
    // rows are stored per cell-ordered slot with (slot | image code) entries: map both back
    // to the system's own atom indices, as the reference lists them
    const int cap = ds.nbr_capacity;
    std::vector<int> slot_counts(h.n), order(h.n), raw((size_t)h.n * cap);
    CUDA_OK(cudaMemcpy(slot_counts.data(), e.nbr_count.p + h.atom_start, sizeof(int) * h.n, cudaMemcpyDeviceToHost));
    CUDA_OK(cudaMemcpy(order.data(), e.sorted_orig.p + h.atom_start, sizeof(int) * h.n, cudaMemcpyDeviceToHost));
    CUDA_OK(cudaMemcpy(raw.data(), e.nbr.p + ds.nbr_base, sizeof(int) * raw.size(), cudaMemcpyDeviceToHost));
    for (int sl = 0; sl < h.n; ++sl) {
      const int atom = order[sl] - h.atom_start;
      if (counts) counts[atom] = slot_counts[sl];
      if (rows)
        for (int k = 0; k < cap; ++k) {
          const unsigned entry = (unsigned)raw[(size_t)sl * cap + k];
          rows[(size_t)atom * cap + k] =
              k < slot_counts[sl] ? order[(int)(entry & rmd::NBR_SLOT_MASK) - h.atom_start] - h.atom_start : 0;
        }
    }
    if (req) CUDA_OK(cudaMemcpy(req, e.required.p + s, sizeof(int), cudaMemcpyDeviceToHost));
  });
}

rmd_status rmd_debug_group_rows(rmd_sim *sim, int32_t s, int32_t *groups, int32_t *capacity, int32_t *atoms,
                                int32_t *counts, int32_t *partners, int32_t *codes, int32_t *masks) {
  if (rmd_status c = check_index(sim, s)) return c;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    e.sync();
    if (e.pair_list == 1)
      throw rmd::Error(RMD_ERR_INVALID, "this simulation walks per-atom rows (pair_list 1): it has no group-pair rows");
    const auto &h = e.hs[s];
    const auto &ds = e.h_sys[s];
    const int first = ds.group_base;
    const int n = (s + 1 < e.S ? e.h_sys[s + 1].group_base : e.n_groups_total) - first;
    const int cap = ds.nbr_capacity;
    if (groups) *groups = n;
    if (capacity) *capacity = cap;
    if (!atoms && !counts && !partners) return;
    std::vector<int> size(n), start(n), cnt(n), order(h.n), orig(h.n), raw((size_t)n * cap);
    CUDA_OK(cudaMemcpy(size.data(), e.gsize.p + first, sizeof(int) * n, cudaMemcpyDeviceToHost));
    CUDA_OK(cudaMemcpy(start.data(), e.gfirst.p + first, sizeof(int) * n, cudaMemcpyDeviceToHost));
    CUDA_OK(cudaMemcpy(cnt.data(), e.gnbr_count.p + first, sizeof(int) * n, cudaMemcpyDeviceToHost));
    CUDA_OK(cudaMemcpy(order.data(), e.group_order.p + h.atom_start, sizeof(int) * h.n, cudaMemcpyDeviceToHost));
    CUDA_OK(cudaMemcpy(orig.data(), e.sorted_orig.p + h.atom_start, sizeof(int) * h.n, cudaMemcpyDeviceToHost));
    CUDA_OK(cudaMemcpy(raw.data(), e.gnbr.p + ds.gnbr_base, sizeof(int) * raw.size(), cudaMemcpyDeviceToHost));
    // slots and order positions are global: map both back to the system's own atom indices
    auto atom_of_slot = [&](int slot) { return orig[slot - h.atom_start] - h.atom_start; };
    for (int q = 0; q < n; ++q) {
      for (int a = 0; a < rmd::GROUP_ATOMS; ++a)
        if (atoms)
          atoms[q * rmd::GROUP_ATOMS + a] =
              a < size[q] ? atom_of_slot(order[start[q] + a - h.atom_start]) : -1;
      if (counts) counts[q] = size[q] > 0 ? cnt[q] : 0;
      for (int k = 0; k < cap; ++k) {
        const bool used = size[q] > 0 && k < cnt[q];
        const unsigned entry = (unsigned)raw[(size_t)q * cap + k];
        if (partners) partners[(size_t)q * cap + k] = used ? atom_of_slot((int)(entry & rmd::GROUP_SLOT_MASK)) : -1;
        if (codes) codes[(size_t)q * cap + k] = used ? (int)((entry >> rmd::GROUP_CODE_SHIFT) & 31u) : 0;
        if (masks) masks[(size_t)q * cap + k] = used ? (int)(entry >> rmd::GROUP_MASK_SHIFT) : 0;
      }
    }
  });
}

rmd_status rmd_debug_evaluate(rmd_sim *sim, int32_t s, rmd_energy_report *energy, double *forces) {
  if (rmd_status c = check_index(sim, s)) return c;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    e.evaluate(true, true);
    e.sync();
    for (auto &h : e.hs) h.steps_since_rebuild = 0;
    e.check_capacity();
    e.energy(s, energy);
    if (forces) {
      const auto &h = e.hs[s];
      std::vector<long long> f(h.n);
      for (int c = 0; c < 3; ++c) {
        CUDA_OK(cudaMemcpy(f.data(), e.force.p + (size_t)c * e.N + h.atom_start, sizeof(long long) * h.n,
                           cudaMemcpyDeviceToHost));
        for (int i = 0; i < h.n; ++i) forces[3 * i + c] = (double)f[i] / rmd::FORCE_SCALE;
      }
    }
  });
}

rmd_status rmd_debug_force_term(rmd_sim *sim, int32_t s, int32_t term, double *forces) {
  if (rmd_status c = check_index(sim, s)) return c;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    const rmd::LaunchCtx c = e.ctx();
    e.sync();
    CUDA_OK(cudaMemsetAsync(e.force.p, 0, e.force.bytes(), e.stream));
    if (term == 0) rmd::launch_nonbonded(c, false, e.nb_lanes, e.stream);
    else if (term == 1) rmd::launch_bonded(c, false, e.stream);
    else if (term == 2) rmd::launch_pme(c, false, e.stream);
    else throw rmd::Error(RMD_ERR_INVALID, "term is 0 (nonbonded), 1 (bonded) or 2 (reciprocal)");
    e.sync();
    CUDA_OK(cudaGetLastError());
    const auto &h = e.hs[s];
    std::vector<long long> f(h.n);
    for (int k = 0; k < 3; ++k) {
      CUDA_OK(cudaMemcpy(f.data(), e.force.p + (size_t)k * e.N + h.atom_start, sizeof(long long) * h.n,
                         cudaMemcpyDeviceToHost));
      for (int i = 0; i < h.n; ++i) forces[3 * i + k] = (double)f[i] / rmd::FORCE_SCALE;
    }
    // leave the full forces in place for whatever runs next
    e.evaluate(false, false);
    e.sync();
  });
}

rmd_status rmd_debug_read(rmd_sim *sim, int32_t s, int32_t which, double *out) {
  if (rmd_status c = check_index(sim, s)) return c;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    e.sync();
    const auto &h = e.hs[s];
    const auto &ds = e.h_sys[s];
    const size_t pts = (size_t)h.grid[0] * h.grid[1] * h.grid[2];
    const size_t hp = (size_t)h.grid[0] * h.grid[1] * (h.grid[2] / 2 + 1);
    if (which == 0) {  // real grid after the inverse transform
      std::vector<float> g(pts);
      CUDA_OK(cudaMemcpy(g.data(), e.real_grid.p + ds.grid_base, sizeof(float) * pts, cudaMemcpyDeviceToHost));
      for (size_t k = 0; k < pts; ++k) out[k] = g[k];
    } else if (which == 1) {  // half spectrum
      std::vector<float2> g(hp);
      CUDA_OK(cudaMemcpy(g.data(), e.half.p + ds.half_base, sizeof(float2) * hp, cudaMemcpyDeviceToHost));
      for (size_t k = 0; k < hp; ++k) {
        out[2 * k] = g[k].x;
        out[2 * k + 1] = g[k].y;
      }
    } else if (which == 2) {  // the positions the current neighbour list was built from
      std::vector<float4> o(h.n);
      CUDA_OK(cudaMemcpy(o.data(), e.origin.p + h.atom_start, sizeof(float4) * h.n, cudaMemcpyDeviceToHost));
      for (int k = 0; k < h.n; ++k) {
        out[3 * k] = o[k].x;
        out[3 * k + 1] = o[k].y;
        out[3 * k + 2] = o[k].z;
      }
    } else {
      throw rmd::Error(RMD_ERR_INVALID, "buffer is 0 (real grid), 1 (half spectrum) or 2 (list origin)");
    }
  });
}

rmd_status rmd_debug_charge_grid(rmd_sim *sim, int32_t s, double *grid) {
  if (rmd_status c = check_index(sim, s)) return c;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    const auto &h = e.hs[s];
    const rmd::LaunchCtx c = e.ctx();
    // the z pass consumes (and zeroes) the fixed grid inside an evaluation, so spread again
    // into a cleared grid and read it before anything else runs
    e.sync();
    const size_t pts = (size_t)h.grid[0] * h.grid[1] * h.grid[2];
    CUDA_OK(cudaMemsetAsync(e.fixed_grid.p, 0, e.fixed_grid.bytes(), e.stream));
    rmd::launch_spread_only(c, e.stream);
    e.sync();
    std::vector<long long> g(pts);
    CUDA_OK(cudaMemcpy(g.data(), e.fixed_grid.p + e.h_sys[s].grid_base, sizeof(long long) * pts,
                       cudaMemcpyDeviceToHost));
    for (size_t k = 0; k < pts; ++k) grid[k] = (double)g[k] / rmd::FORCE_SCALE;
    CUDA_OK(cudaMemsetAsync(e.fixed_grid.p, 0, e.fixed_grid.bytes(), e.stream));
    e.sync();
  });
}

rmd_status rmd_bench_run(rmd_sim *sim, int64_t count, int32_t block_size, int32_t flush_l2,
                         double *device_ms) {
  if (!sim) return RMD_ERR_INVALID;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    if (!e.ev_a) {
      CUDA_OK(cudaEventCreate(&e.ev_a));
      CUDA_OK(cudaEventCreate(&e.ev_b));
    }
    if (flush_l2 && e.flush_buffer.n == 0) e.flush_buffer.alloc((size_t)256 << 20);  // 2x the 126 MB L2
    e.timing = true;
    e.flush = flush_l2 != 0;
    e.timed_ms = 0.0;
    try {
      e.run(count, block_size, nullptr);
    } catch (...) {
      e.timing = false;
      throw;
    }
    e.timing = false;
    *device_ms = e.timed_ms;
  });
}

rmd_status rmd_debug_time_kernel(rmd_sim *sim, int32_t which, int32_t reps, double *ms_per_launch) {
  if (!sim || reps <= 0) return RMD_ERR_INVALID;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    const rmd::LaunchCtx c = e.ctx();
    auto one = [&]() {
      switch (which) {
        case 0: rmd::launch_nonbonded(c, false, e.nb_lanes, e.stream); break;
        case 1: rmd::launch_pme(c, false, e.stream); break;
        case 2: rmd::launch_integrate(e.iargs(0), rmd::INT_CLOSE | rmd::INT_OPEN, e.stream); break;
        case 3: rmd::launch_bonded(c, false, e.stream); break;
        case 4: rmd::launch_rebuild(c, e.stream); break;
        case 5: rmd::launch_nonbonded(c, true, e.nb_lanes, e.stream); break;
        default: throw rmd::Error(RMD_ERR_INVALID, "unknown kernel group");
      }
    };
    e.sync();
    // the timed launches move atoms (integrator) or add into the force array (PME, bonded):
    // keep the state and put it back afterwards, with forces from a clean evaluation
    rmd::DevArray<float4> keep_pos, keep_vel, keep_spos;
    keep_pos.alloc(e.N);
    keep_vel.alloc(e.N);
    keep_spos.alloc(e.N);
    CUDA_OK(cudaMemcpyAsync(keep_pos.p, e.posq.p, sizeof(float4) * e.N, cudaMemcpyDeviceToDevice, e.stream));
    CUDA_OK(cudaMemcpyAsync(keep_vel.p, e.vel.p, sizeof(float4) * e.N, cudaMemcpyDeviceToDevice, e.stream));
    CUDA_OK(cudaMemcpyAsync(keep_spos.p, e.spos.p, sizeof(float4) * e.N, cudaMemcpyDeviceToDevice, e.stream));
    one();  // warm
    cudaEvent_t a, b;
    CUDA_OK(cudaEventCreate(&a));
    CUDA_OK(cudaEventCreate(&b));
    CUDA_OK(cudaEventRecord(a, e.stream));
    for (int k = 0; k < reps; ++k) one();
    CUDA_OK(cudaEventRecord(b, e.stream));
    CUDA_OK(cudaEventSynchronize(b));
    float ms = 0;
    CUDA_OK(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CUDA_OK(cudaGetLastError());
    *ms_per_launch = ms / reps;
    CUDA_OK(cudaMemcpyAsync(e.posq.p, keep_pos.p, sizeof(float4) * e.N, cudaMemcpyDeviceToDevice, e.stream));
    CUDA_OK(cudaMemcpyAsync(e.vel.p, keep_vel.p, sizeof(float4) * e.N, cudaMemcpyDeviceToDevice, e.stream));
    CUDA_OK(cudaMemcpyAsync(e.spos.p, keep_spos.p, sizeof(float4) * e.N, cudaMemcpyDeviceToDevice, e.stream));
    e.evaluate(true, false);
    e.sync();
    for (auto &h : e.hs) h.steps_since_rebuild = 0;
    keep_pos.release();
    keep_vel.release();
    keep_spos.release();
  });
}

rmd_status rmd_debug_draws(uint32_t seed, uint32_t atom0, int32_t count, uint32_t step, float *uniforms,
                           float *normals) {
  if (count < 0 || (count > 0 && (!uniforms || !normals))) return RMD_ERR_INVALID;
  return guarded(nullptr, [&]() {
    if (count == 0) return;
    rmd::DevArray<float> u, g;
    u.alloc((size_t)count * 4);
    g.alloc((size_t)count * 3);
    rmd::launch_draws(seed, atom0, count, step, u.p, g.p, nullptr);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaMemcpy(uniforms, u.p, u.bytes(), cudaMemcpyDeviceToHost));
    CUDA_OK(cudaMemcpy(normals, g.p, g.bytes(), cudaMemcpyDeviceToHost));
    u.release();
    g.release();
  });
}

int64_t rmd_debug_kernel_launches(const rmd_sim *sim) { return sim ? sim->engine.kernel_launches : 0; }

int32_t rmd_debug_plane_pass(int32_t nx, int32_t ny) {
  return nx > 0 && ny > 0 ? rmd::fft_plane_split(nx, ny) : 0;
}

rmd_status rmd_surrogate_report_at(rmd_sim *sim, int32_t s, rmd_surrogate_report *out) {
  if (rmd_status c = check_index(sim, s)) return c;
  if (!out) return RMD_ERR_INVALID;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    e.sync();
    std::vector<double> b(rmd::N_BARO);
    CUDA_OK(cudaMemcpy(b.data(), e.baro.p + (size_t)s * rmd::N_BARO, sizeof(double) * rmd::N_BARO,
                       cudaMemcpyDeviceToHost));
    memset(out, 0, sizeof *out);
    out->samples = (int64_t)b[rmd::B_REPLAY_N];
    out->train_steps = (int64_t)b[rmd::B_TRAIN_STEPS];
    out->loss = b[rmd::B_LOSS];
    out->prediction_error_kT = b[rmd::B_PRED_ERR];
    out->screening = b[rmd::B_LEARNED] != 0.0 && b[rmd::B_REPLAY_N] >= b[rmd::B_WARMUP];
    out->attempts = (int64_t)b[rmd::B_ATTEMPTS];
    out->exact_evaluations = (int64_t)b[rmd::B_EXACT_EVALS];
    out->screened = (int64_t)b[rmd::B_SCREENED_TOTAL];
    out->accepted = (int64_t)b[rmd::B_ACCEPTED];
    out->exact_passes = e.exact_passes;
    out->skipped_passes = e.skipped_passes;
  });
}

rmd_status rmd_surrogate_weights(rmd_sim *sim, int32_t s, float *params) {
  if (rmd_status c = check_index(sim, s)) return c;
  if (!params) return RMD_ERR_INVALID;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    if (!e.learned) throw rmd::Error(RMD_ERR_INVALID, "the learned barostat is not enabled");
    e.sync();
    CUDA_OK(cudaMemcpy(params, e.mlp_master.p + (size_t)s * rmd::MLP_STRIDE, sizeof(float) * rmd::MLP_PARAMS,
                       cudaMemcpyDeviceToHost));
  });
}

rmd_status rmd_surrogate_evaluate(const float *params, const float *inputs, const float *targets, int32_t count,
                                  float *outputs, float *grads, double *loss) {
  if (!params || !inputs || count <= 0 || count > rmd::MLP_BATCH || (grads && (!targets || !loss)))
    return RMD_ERR_INVALID;
  return guarded(nullptr, [&]() {
    rmd::DevArray<float> p, x, t, o, g, l;
    p.upload(std::vector<float>(params, params + rmd::MLP_PARAMS));
    x.upload(std::vector<float>(inputs, inputs + (size_t)count * rmd::MLP_IN));
    if (targets) t.upload(std::vector<float>(targets, targets + count));
    o.alloc(count);
    if (grads) {
      g.alloc(rmd::MLP_PARAMS);
      l.alloc(1);
    }
    rmd::surrogate_predict(p.p, x.p, count, o.p, nullptr);
    if (grads) rmd::surrogate_gradients(p.p, x.p, t.p, count, g.p, l.p, nullptr);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaDeviceSynchronize());
    if (outputs) CUDA_OK(cudaMemcpy(outputs, o.p, sizeof(float) * count, cudaMemcpyDeviceToHost));
    if (grads) {
      CUDA_OK(cudaMemcpy(grads, g.p, sizeof(float) * rmd::MLP_PARAMS, cudaMemcpyDeviceToHost));
      float lf = 0;
      CUDA_OK(cudaMemcpy(&lf, l.p, sizeof(float), cudaMemcpyDeviceToHost));
      *loss = lf;
    }
    for (auto *a : {&p, &x, &t, &o, &g, &l}) a->release();
  });
}

rmd_status rmd_kernel_shapes(const rmd_sim *sim, int32_t shapes[3], double tune_ms[9]) {
  if (!sim) return RMD_ERR_INVALID;
  const auto &e = sim->engine;
  if (shapes) {
    shapes[0] = e.group_atoms;
    shapes[1] = e.nb_lanes;
    shapes[2] = e.spread_atoms;
  }
  if (tune_ms)
    for (int k = 0; k < 9; ++k) tune_ms[k] = e.tune_ms[k];
  return RMD_OK;
}

rmd_status rmd_set_kernel_shapes(rmd_sim *sim, int32_t group_atoms, int32_t nonbonded_lanes,
                                 int32_t spread_atoms) {
  if (!sim) return RMD_ERR_INVALID;
  auto ok = [](int v, int a, int b, int c) { return v == 0 || v == a || v == b || v == c; };
  if (!(ok(group_atoms, 4, 8, 16) || group_atoms == 32) || !(ok(nonbonded_lanes, 8, 16, 32) || ok(nonbonded_lanes, 32, 64, 128)) ||
      !ok(spread_atoms, 4, 8, 16))
    return RMD_ERR_INVALID;
  auto &e = sim->engine;
  if (e.pair_list != 1 && ((group_atoms && group_atoms != rmd::GROUP_ATOMS) ||
                            (nonbonded_lanes && nonbonded_lanes != 32 && nonbonded_lanes != 64 &&
                             nonbonded_lanes != 128))) {
    e.last_error = "with group-pair rows the search groups hold 4 atoms and a row is shared by 32, 64 or 128 lanes";
    return RMD_ERR_INVALID;
  }
  if (e.pair_list == 1 && nonbonded_lanes > 32) {
    e.last_error = "per-atom rows take 8, 16 or 32 lanes an atom";
    return RMD_ERR_INVALID;
  }
  if (group_atoms) e.group_atoms = group_atoms;
  if (nonbonded_lanes) e.nb_lanes = nonbonded_lanes;
  if (spread_atoms) e.spread_atoms = spread_atoms;
  e.drop_graphs();
  return RMD_OK;
}

rmd_status rmd_debug_set_nonbonded(rmd_sim *sim, int32_t lanes, int32_t pair_fixed) {
  if (!sim || (lanes != 8 && lanes != 16 && lanes != 32)) return RMD_ERR_INVALID;
  auto &e = sim->engine;
  if (e.pair_list != 1) {
    e.last_error = "the pair-loop shape and accumulation form can only be changed on per-atom rows (pair_list 1)";
    return RMD_ERR_INVALID;
  }
  e.nb_lanes = lanes;
  e.pair_fixed = pair_fixed ? 1 : 0;
  for (auto &kv : e.graphs) cudaGraphExecDestroy(kv.second);
  e.graphs.clear();
  e.graph_launches.clear();
  return RMD_OK;
}

rmd_status rmd_debug_fft(rmd_sim *sim, int32_t s, const double *data, double *half_spectrum, double *round_trip) {
  if (rmd_status c = check_index(sim, s)) return c;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    const auto &h = e.hs[s];
    const auto &ds = e.h_sys[s];
    const int nx = h.grid[0], ny = h.grid[1], nz = h.grid[2], nzh = nz / 2 + 1;
    const size_t pts = (size_t)nx * ny * nz, hp = (size_t)nx * ny * nzh;
    e.sync();
    std::vector<long long> fx(pts);
    for (size_t k = 0; k < pts; ++k) fx[k] = (long long)std::llround(data[k] * rmd::FORCE_SCALE);
    CUDA_OK(cudaMemsetAsync(e.fixed_grid.p, 0, e.fixed_grid.bytes(), e.stream));
    CUDA_OK(cudaMemcpyAsync(e.fixed_grid.p + ds.grid_base, fx.data(), sizeof(long long) * pts,
                            cudaMemcpyHostToDevice, e.stream));
    const rmd::LaunchCtx c = e.ctx();
    rmd::launch_fft_forward(c, e.stream);
    e.sync();
    std::vector<float2> hs_(hp);
    CUDA_OK(cudaMemcpy(hs_.data(), e.half.p + ds.half_base, sizeof(float2) * hp, cudaMemcpyDeviceToHost));
    for (size_t k = 0; k < hp; ++k) {
      half_spectrum[2 * k] = hs_[k].x;
      half_spectrum[2 * k + 1] = hs_[k].y;
    }
    rmd::launch_fft_inverse(c, e.stream);
    e.sync();
    std::vector<float> rg(pts);
    CUDA_OK(cudaMemcpy(rg.data(), e.real_grid.p + ds.grid_base, sizeof(float) * pts, cudaMemcpyDeviceToHost));
    for (size_t k = 0; k < pts; ++k) round_trip[k] = rg[k];
  });
}

}  // extern "C"


// ----------------------------------------------------------------- trajectory output
// ECMAScript x.toExponential(7) (rst7.js:69): eight significant digits of the exact binary
// value, the larger on a tie, "e", the exponent's sign and its digits without padding.
static std::string script_exponential7(double x) {
  if (x == 0.0) return "0.0000000e+0";
  std::string sign = x < 0 ? "-" : "";
  const double a = std::fabs(x);
  // 40 exact significant digits (glibc prints the exact decimal expansion, rounded only at
  // the last digit shown), then the tie-up rounding at the eighth by hand
  char buf[64];
  snprintf(buf, sizeof buf, "%.39e", a);
  std::string digits;
  const char *p = buf;
  for (; *p && *p != 'e'; ++p)
    if (*p >= '0' && *p <= '9') digits.push_back(*p);
  int exponent = atoi(p + 1);
  std::string head = digits.substr(0, 8);
  bool up = digits[8] >= '5';
  if (up) {
    int k = 7;
    while (k >= 0 && head[k] == '9') head[k--] = '0';
    if (k < 0) {
      head = "1" + head.substr(0, 7);
      exponent += 1;
    } else {
      head[k] = (char)(head[k] + 1);
    }
  }
  return sign + head.substr(0, 1) + "." + head.substr(1) + "e" + (exponent < 0 ? "-" : "+") +
         std::to_string(std::abs(exponent));
}

static std::string pad_start(const std::string &s, size_t width) {
  return s.size() >= width ? s : std::string(width - s.size(), ' ') + s;
}

rmd_status rmd_image_molecules_at(rmd_sim *sim, int32_t s, double *out) {
  if (rmd_status c = check_index(sim, s)) return c;
  if (!out) return RMD_ERR_INVALID;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    const rmd::TrajArgs t = e.traj_args(s, true);
    rmd::DevArray<double> wrapped;
    wrapped.alloc(3 * (size_t)t.atom_count);
    rmd::launch_traj_image(t, wrapped.p, e.stream);
    CUDA_OK(cudaGetLastError());
    CUDA_OK(cudaMemcpyAsync(out, wrapped.p, sizeof(double) * wrapped.n, cudaMemcpyDeviceToHost, e.stream));
    e.sync();
    wrapped.release();
  });
}

int64_t rmd_dcd_frame_bytes(int32_t atom_count, int32_t periodic) {
  if (atom_count < 0) return -1;
  return (periodic ? 56 : 0) + 3 * (4 * (int64_t)atom_count + 8);
}

rmd_status rmd_dcd_frame_at(rmd_sim *sim, int32_t s, int32_t periodic, int32_t image, uint8_t *out) {
  if (rmd_status c = check_index(sim, s)) return c;
  if (!out) return RMD_ERR_INVALID;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    rmd::TrajArgs t = e.traj_args(s, image != 0);
    const size_t bytes = (size_t)rmd_dcd_frame_bytes(t.atom_count, periodic);
    if (e.traj_out.n < bytes) e.traj_out.alloc(bytes);
    t.out = e.traj_out.p;
    rmd::launch_dcd_pack(t, periodic ? 1 : 0, e.stream);
    CUDA_OK(cudaGetLastError());
    int status[2];
    CUDA_OK(cudaMemcpyAsync(status, e.traj_status.p, sizeof status, cudaMemcpyDeviceToHost, e.stream));
    e.sync();
    if (status[0] != INT_MAX)  // dcd.js:112-128
      throw rmd::Error(RMD_ERR_NON_FINITE,
                       "the simulation is no longer a number: a coordinate handed to the DCD writer (atom " +
                           std::to_string(status[0]) + ") is not finite. The frame was refused, so the file "
                           "holds the frames written before it and is still readable.");
    CUDA_OK(cudaMemcpy(out, e.traj_out.p, bytes, cudaMemcpyDeviceToHost));
  });
}

rmd_status rmd_dcd_header(int32_t atom_count, int32_t frames, int32_t first_step, int32_t interval, double timestep,
                          int32_t periodic, const char *title, const char *created, uint8_t out[276]) {
  if (!out || atom_count < 0 || frames < 0) return RMD_ERR_INVALID;
  memset(out, 0, 276);
  auto put32 = [&](int offset, int32_t v) { memcpy(out + offset, &v, 4); };
  put32(0, 84);
  memcpy(out + 4, "CORD", 4);
  put32(8, frames);
  put32(12, first_step);
  put32(16, interval);
  put32(20, std::max(0, frames - 1) * interval);  // the last frame's step, as OpenMM fills it
  const float delta = (float)(timestep / 0.04888821);  // AKMA time units (dcd.js:56)
  memcpy(out + 44, &delta, 4);
  put32(48, periodic ? 1 : 0);
  put32(84, 24);
  put32(88, 84);
  put32(92, 164);
  put32(96, 2);
  auto text = [&](int offset, const char *s) {  // NUL-padded, non-ASCII as '?' (dcd.js:243-254)
    for (int k = 0; s && k < 80 && s[k]; ++k) {
      const unsigned char c = (unsigned char)s[k];
      out[offset + k] = c < 128 ? c : 0x3f;
    }
  };
  text(100, title ? title : "Created by RainMD");
  text(180, created);
  put32(260, 164);
  put32(264, 4);
  put32(268, atom_count);
  put32(272, 4);
  return RMD_OK;
}

rmd_status rmd_restart_at(rmd_sim *sim, int32_t s, const char *title, double time, int32_t velocities, int32_t box,
                          char *out, int64_t capacity, int64_t *bytes) {
  if (rmd_status c = check_index(sim, s)) return c;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    const auto &h = e.hs[s];
    const std::string head = std::string(title ? title : "RainMD restart") + "\n" +
                             pad_start(std::to_string(h.n), 5) + pad_start(script_exponential7(time), 15) + "\n";
    const long long n3 = 3ll * h.n;
    const long long total = (long long)head.size() + rmd::rst7_block_size(n3) * (velocities ? 2 : 1) +
                            (box ? rmd::rst7_block_size(6) : 0);
    if (bytes) *bytes = total;
    if (!out) return;
    if (capacity < total) throw rmd::Error(RMD_ERR_INVALID, "the restart needs " + std::to_string(total) + " bytes");
    rmd::Rst7Box b{};
    b.velocity_unit = 20.455 * 0.1;  // units.js:24, 44; rst7.js:87-89
    if (box) {  // boxFromVectors (web/app.js:326-343) of the live box
      rmd::DevSysD d;
      CUDA_OK(cudaMemcpy(&d, e.sysd.p + s, sizeof d, cudaMemcpyDeviceToHost));
      const double *v = d.box;
      const double la = rmd::script_hypot(v[0], v[1], v[2]), lb = rmd::script_hypot(v[3], v[4], v[5]),
                   lc = rmd::script_hypot(v[6], v[7], v[8]);
      auto dot = [](const double *u, const double *w) { return u[0] * w[0] + u[1] * w[1] + u[2] * w[2]; };
      auto degrees = [](double c) { return (std::acos(std::max(-1.0, std::min(1.0, c))) * 180) / M_PI; };
      b.values[0] = la / 0.1;
      b.values[1] = lb / 0.1;
      b.values[2] = lc / 0.1;
      b.values[3] = degrees(dot(v + 3, v + 6) / (lb * lc));
      b.values[4] = degrees(dot(v, v + 6) / (la * lc));
      b.values[5] = degrees(dot(v, v + 3) / (la * lb));
    }
    rmd::TrajArgs t = e.traj_args(s, false);
    if (e.traj_out.n < (size_t)total) e.traj_out.alloc((size_t)total);
    t.out = e.traj_out.p;
    CUDA_OK(cudaMemcpyAsync(e.traj_out.p, head.data(), head.size(), cudaMemcpyHostToDevice, e.stream));
    rmd::launch_rst7_format(t, (long long)head.size(), velocities ? 1 : 0, box ? 1 : 0, b, e.stream);
    CUDA_OK(cudaGetLastError());
    int status[2];
    CUDA_OK(cudaMemcpyAsync(status, e.traj_status.p, sizeof status, cudaMemcpyDeviceToHost, e.stream));
    e.sync();
    // the first failing value in file order decides, as the reference's loop does (rst7.js:27-55)
    if (status[0] != INT_MAX && status[0] < status[1])
      throw rmd::Error(RMD_ERR_NON_FINITE,
                       "the simulation is no longer a number: a coordinate handed to the restart writer (value " +
                           std::to_string(status[0]) + ") is not finite. No restart was written. A restart is the "
                           "one output that is fed straight back into a simulation, so writing a non-finite one "
                           "would carry the blow-up into whatever ran next.");
    if (status[1] != INT_MAX)
      throw rmd::Error(RMD_ERR_INVALID,
                       "coordinate " + std::to_string(status[1]) + " does not fit the 12-column restart format. "
                       "An atom has left the box, which means the simulation blew up rather than that the "
                       "writer is wrong.");
    CUDA_OK(cudaMemcpy(out, e.traj_out.p, (size_t)total, cudaMemcpyDeviceToHost));
  });
}

// ----------------------------------------------------------------- headless rendering
namespace {
// Every check a frame's inputs get before anything reaches the device.
void validate_render(bool have_positions, int32_t atom_count, const rmd_camera *camera, const float *styles,
                     const float *guides, int32_t guide_count, const uint32_t *segments, int32_t segment_count,
                     int32_t draw_spheres, int32_t draw_ribbon, int32_t width, int32_t height, const uint8_t *rgba) {
  if (!camera || !rgba || width <= 0 || height <= 0 || width > 16384 || height > 16384 || atom_count < 0)
    throw rmd::Error(RMD_ERR_INVALID, "a frame needs a camera, an output image and a size of 1-16384 pixels a side");
  if (draw_spheres && atom_count > 0 && !styles)
    throw rmd::Error(RMD_ERR_INVALID, "drawing spheres needs a style (colour, radius) per atom");
  if (draw_ribbon && segment_count > 0) {
    if (!guides || !segments || guide_count <= 0)
      throw rmd::Error(RMD_ERR_INVALID, "drawing the ribbon needs its guides and segments");
    for (long long k = 0; k < 4ll * segment_count; ++k)
      if (segments[k] >= (uint32_t)guide_count)
        throw rmd::Error(RMD_ERR_INVALID, "a ribbon segment names guide " + std::to_string(segments[k]) +
                                              " of " + std::to_string(guide_count));
  }
  if (draw_spheres && atom_count > 0 && !have_positions)
    throw rmd::Error(RMD_ERR_INVALID, "drawing spheres needs positions");
}

rmd_status render_frame(const float4 *positions, int32_t atom_count, const rmd_camera *camera,
                        const float *styles, const float *guides, int32_t guide_count, const uint32_t *segments,
                        int32_t segment_count, int32_t draw_spheres, int32_t draw_ribbon, int32_t width,
                        int32_t height, uint8_t *rgba, cudaStream_t stream) {
  rmd::RenderArgs a{};
  static_assert(sizeof(rmd::RenderCamera) == sizeof(rmd_camera), "the camera uniform is 36 floats");
  memcpy(&a.camera, camera, sizeof a.camera);
  a.atom_count = draw_spheres ? atom_count : 0;
  a.segment_count = draw_ribbon ? segment_count : 0;
  a.draw_spheres = draw_spheres && atom_count > 0 ? 1 : 0;
  a.draw_ribbon = draw_ribbon && segment_count > 0 ? 1 : 0;
  a.width = width;
  a.height = height;
  a.positions = positions;
  rmd::DevArray<float4> d_styles, corners;
  rmd::DevArray<float> d_guides, verts;
  rmd::DevArray<uint4> d_segments;
  rmd::DevArray<unsigned long long> keys;
  rmd::DevArray<uchar4> image;
  if (a.draw_spheres) {
    d_styles.alloc(atom_count);
    CUDA_OK(cudaMemcpyAsync(d_styles.p, styles, sizeof(float4) * atom_count, cudaMemcpyHostToDevice, stream));
    corners.alloc(4 * (size_t)atom_count);
    a.styles = d_styles.p;
    a.sphere_corners = corners.p;
  }
  if (a.draw_ribbon) {
    d_guides.alloc(12 * (size_t)guide_count);
    CUDA_OK(cudaMemcpyAsync(d_guides.p, guides, sizeof(float) * 12 * guide_count, cudaMemcpyHostToDevice, stream));
    d_segments.alloc(segment_count);
    CUDA_OK(cudaMemcpyAsync(d_segments.p, segments, sizeof(uint4) * segment_count, cudaMemcpyHostToDevice, stream));
    verts.alloc(12 * 24 * 8 * (size_t)segment_count);
    a.guides = d_guides.p;
    a.segments = d_segments.p;
    a.ribbon_vertices = verts.p;
  }
  keys.alloc((size_t)width * height);
  image.alloc((size_t)width * height);
  a.keys = keys.p;
  a.image = image.p;
  rmd::launch_render(a, stream);
  CUDA_OK(cudaGetLastError());
  CUDA_OK(cudaMemcpyAsync(rgba, image.p, sizeof(uchar4) * (size_t)width * height, cudaMemcpyDeviceToHost, stream));
  CUDA_OK(cudaStreamSynchronize(stream));
  return RMD_OK;
}
}  // namespace

rmd_status rmd_render_at(rmd_sim *sim, int32_t s, const rmd_camera *camera, const float *styles,
                         const float *guides, int32_t guide_count, const uint32_t *segments, int32_t segment_count,
                         int32_t draw_spheres, int32_t draw_ribbon, int32_t width, int32_t height, uint8_t *rgba) {
  if (rmd_status c = check_index(sim, s)) return c;
  return guarded(sim, [&]() {
    auto &e = sim->engine;
    const auto &h = e.hs[s];
    validate_render(true, h.n, camera, styles, guides, guide_count, segments, segment_count, draw_spheres,
                    draw_ribbon, width, height, rgba);
    render_frame(e.posq.p + h.atom_start, h.n, camera, styles, guides, guide_count, segments, segment_count,
                 draw_spheres, draw_ribbon, width, height, rgba, e.stream);
  });
}

rmd_status rmd_render_positions(const float *positions, int32_t atom_count, const rmd_camera *camera,
                                const float *styles, const float *guides, int32_t guide_count,
                                const uint32_t *segments, int32_t segment_count, int32_t draw_spheres,
                                int32_t draw_ribbon, int32_t width, int32_t height, uint8_t *rgba) {
  return guarded(nullptr, [&]() {
    validate_render(positions != nullptr, atom_count, camera, styles, guides, guide_count, segments,
                    segment_count, draw_spheres, draw_ribbon, width, height, rgba);
    rmd::DevArray<float4> p;
    if (atom_count > 0 && positions) {
      std::vector<float4> host(atom_count);
      for (int i = 0; i < atom_count; ++i)
        host[i] = make_float4(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2], 0.0f);
      p.upload(host);
    }
    render_frame(p.p, atom_count, camera, styles, guides, guide_count, segments, segment_count,
                 draw_spheres, draw_ribbon, width, height, rgba, cudaStreamLegacy);
  });
}
