// Shared device-side definitions for the B200 RainMD step engine (sm_100a).
//
// Every kernel works on a BATCH of independent systems: atoms, cells, neighbour rows,
// PME grids and bonded terms of all systems are concatenated, and a per-system
// descriptor (DevSys) gives each system's offsets, box and cut-offs. A single system is
// a batch of one. Kernels read the box from DevSys rather than from a baked constant so
// the on-device barostat can change it inside a CUDA graph.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rmd {

constexpr double ONE_4PI_EPS0 = 138.935456;      // shared/units.js:47
constexpr double BOLTZMANN = 0.008314462618;     // shared/units.js:50
constexpr double BAR_TO_KJ_PER_MOL_NM3 = 0.06022140857;  // shared/units.js:53

// Forces are accumulated as 64-bit two's-complement fixed point with 2^32 units per
// kJ/mol/nm: integer addition is associative, so any order of atomics gives the same
// bits. The PME charge grid uses the same format with 2^32 units per elementary charge.
constexpr double FORCE_SCALE = 4294967296.0;
constexpr float FORCE_SCALE_F = 4294967296.0f;
constexpr float FORCE_UNSCALE_F = 2.3283064365386963e-10f;  // 2^-32, exact

constexpr int MAX_CLUSTER_ATOMS = 8;
constexpr int MAX_CLUSTER_CONSTRAINTS = 12;
constexpr int MAX_ORDER = 5;

// Per-system descriptor, resident in device memory.
struct DevSys {
  float box[9];       // reduced box rows a, b, c (nm)
  float recip[9];     // rows of the inverse box (recip[3*i + d])
  float inv_diag[3];  // 1/a_x, 1/b_y, 1/c_z for the minimum image
  float cutoff, cutoff2, list_cutoff, list_cutoff2;
  float alpha;
  int atom_start, atom_count;
  int type_count, lj_base;
  int cell_counts[3];
  int cell_base;        // offset into per-cell arrays (count/cursor)
  int cell_start_base;  // offset into cell_start ((cells + 1) per system)
  int cell_capacity;    // cells allocated for this system
  int group_base;       // first neighbour-search group slot of this system
  long long nbr_base;   // offset of row 0 in the neighbour array
  int nbr_capacity;     // entries a row holds (per-atom rows and group rows alike)
  long long gnbr_base;  // offset of group slot 0's row in the group-pair array
  int grid[3];
  long long grid_base;  // real grid offset (K^3)
  long long half_base;  // complex half-spectrum offset (Kx*Ky*(Kz/2+1))
  int moduli_base;      // moduli[x][y][z] concatenated (Kx+Ky+Kz)
  int order;
  int molecule_start, molecule_count;  // into molecule CSR
  // Lattice shifts S = ka*a + kb*b + kc*c for ka, kb, kc in {-1, 0, 1}, indexed by
  // code = (ka+1)*9 + (kb+1)*3 + (kc+1): a neighbour entry carries the code of the image of
  // its partner that was nearest when the list was built (d = x_i - x_j - S).
  float4 shift[27];
};

// FP64 per-system state owned by the device (box for the barostat, energies, counters).
struct DevSysD {
  double box[9];
  double volume;
  double q2_sum, q_sum;       // for the self and net-charge terms
  double disp_a, disp_b;      // dispersion coefficients (dispersion.js:37)
  double cutoff, alpha;
  double list_cutoff;
  double saved_box[9];
  double saved_volume;
  int dispersion_on;
  int max_counts[3];    // cells allocated per axis; the device never plans more
  int saved_counts[3];
  int pad0;
};

// ---------------------------------------------------- programmatic dependent launch
// The kernels of the step's serial chains (integrator, spreading, FFT passes, gather) are
// launched with programmatic stream serialisation (launch_chained): a kernel's blocks may be
// scheduled while its predecessor in the stream is still running, which hides the launch
// latency between short dependent kernels. Such a kernel must start with chain_begin(): it
// waits until every predecessor grid has completed and its memory is visible, before any
// memory access, then lets its own successor be scheduled. In a plain launch both are no-ops.
__device__ __forceinline__ void chain_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KernelArgs, typename... Args>
inline void launch_kernel(bool chained, void (*kernel)(KernelArgs...), dim3 grid, dim3 block, size_t smem,
                          cudaStream_t stream, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr;
  attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr.val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = chained ? 1 : 0;
  (void)cudaLaunchKernelEx(&cfg, kernel, static_cast<KernelArgs>(args)...);  // errors surface in cudaGetLastError
}

template <typename... KernelArgs, typename... Args>
inline void launch_chained(void (*kernel)(KernelArgs...), dim3 grid, dim3 block, size_t smem,
                           cudaStream_t stream, Args... args) {
  launch_kernel(true, kernel, grid, block, smem, stream, args...);
}

// ---------------------------------------------------------------- fixed point
__device__ __forceinline__ unsigned long long to_fixed(float v) {
  return (unsigned long long)__float2ll_rn(v * FORCE_SCALE_F);
}
__device__ __forceinline__ float from_fixed(unsigned long long v) {
  return __ll2float_rn((long long)v) * FORCE_UNSCALE_F;
}
__device__ __forceinline__ void add_fixed(unsigned long long *p, float v) {
  atomicAdd(p, to_fixed(v));
}

// ---------------------------------------------------------------- warp helpers
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ long long warp_sum(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ---------------------------------------------------------------- counter RNG
// shared/random.js:24-87: integer mixing is exact on every device; the uniform keeps the
// top 23 bits so (state>>9)+0.5 is exact in f32 and bit-identical to the f64 host draw.
__device__ __forceinline__ uint32_t rng_mix(uint32_t s) {
  s ^= s >> 16;
  s *= 0x7feb352du;
  s ^= s >> 15;
  s *= 0x846ca68bu;
  s ^= s >> 16;
  return s;
}
__device__ __forceinline__ float rng_uniform(uint32_t seed, uint32_t a, uint32_t b, uint32_t c) {
  uint32_t s = rng_mix(seed ^ (a * 0x9e3779b1u));
  s = rng_mix(s ^ (b * 0x85ebca6bu));
  s = rng_mix(s ^ (c * 0xc2b2ae35u));
  return ((float)(s >> 9) + 0.5f) * 1.1920928955078125e-7f;
}
__device__ __forceinline__ double rng_uniform_d(uint32_t seed, uint32_t a, uint32_t b, uint32_t c) {
  uint32_t s = rng_mix(seed ^ (a * 0x9e3779b1u));
  s = rng_mix(s ^ (b * 0x85ebca6bu));
  s = rng_mix(s ^ (c * 0xc2b2ae35u));
  return ((double)(s >> 9) + 0.5) * (1.0 / 8388608.0);
}
__device__ __forceinline__ float3 rng_gaussian3(uint32_t seed, uint32_t atom, uint32_t step) {
  float u1 = rng_uniform(seed, atom, step, 0), u2 = rng_uniform(seed, atom, step, 1);
  float u3 = rng_uniform(seed, atom, step, 2), u4 = rng_uniform(seed, atom, step, 3);
  float r1 = sqrtf(-2.0f * logf(u1)), r2 = sqrtf(-2.0f * logf(u3));
  float s2, c2, s4, c4;
  sincospif(2.0f * u2, &s2, &c2);
  sincospif(2.0f * u4, &s4, &c4);
  return make_float3(r1 * c2, r1 * s2, r2 * c4);
}

// ---------------------------------------------------------------- erfc
// erfc(z) = t * P(t) * exp(-z^2), t = 1/(1 + z/2). P is this project's own degree-8 fit
// (rainmd_b200/fit_erfc.py: relative error 2.0e-8 in exact arithmetic over z in [0, 5],
// 3e-7 at f32 evaluation). Returns erfc and leaves exp(-z^2) in `gauss` for the force.
// Hardware approximate reciprocal (one MUFU instruction, within 1 ulp).
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ float erfc_and_gauss(float z, float &gauss) {
  gauss = __expf(-z * z);
  // t in (0, 1]: a 1-ulp reciprocal moves erfc by ~1e-7 relative, well inside the f32 pair
  // arithmetic's own error, at a fraction of the correctly rounded division's cost
  float t = rcp_approx(fmaf(0.5f, z, 1.0f));
  float p = -4.967514911e-02f;
  p = fmaf(p, t, 2.366592171e-01f);
  p = fmaf(p, t, -3.827331461e-01f);
  p = fmaf(p, t, 1.511331490e-01f);
  p = fmaf(p, t, 6.722758340e-02f);
  p = fmaf(p, t, 1.595169610e-01f);
  p = fmaf(p, t, 2.551498949e-01f);
  p = fmaf(p, t, 2.805130003e-01f);
  p = fmaf(p, t, 2.822084696e-01f);
  return t * p * gauss;
}

// 1/sqrt(x) for x > 0: the hardware approximation plus one Newton-Raphson step
// y <- y (1.5 - 0.5 x y^2), which leaves only the unbiased rounding of three f32 operations.
// The pair kernel raises this to the 6th and 12th power and sums millions of LJ terms whose
// repulsive and dispersive halves nearly cancel, so the approximation's own bias (not its
// size) would otherwise set the error of the LJ total.
__device__ __forceinline__ float rsqrt_refined(float x) {
  const float y = rsqrtf(x);
  return y * fmaf(-0.5f * x * y, y, 1.5f);
}

// ---------------------------------------------------------------- geometry
// Minimum image for a reduced box, c then b then a (cpu/forces/geometry.js:27-43). The
// force kernels use rint(d/L); at an exact half-box tie it may pick the other image of an
// equidistant pair, which changes no energy.
__device__ __forceinline__ float3 min_image(float3 d, const DevSys &s) {
  float k = rintf(d.z * s.inv_diag[2]);
  d.x = fmaf(-k, s.box[6], d.x);
  d.y = fmaf(-k, s.box[7], d.y);
  d.z = fmaf(-k, s.box[8], d.z);
  k = rintf(d.y * s.inv_diag[1]);
  d.x = fmaf(-k, s.box[3], d.x);
  d.y = fmaf(-k, s.box[4], d.y);
  k = rintf(d.x * s.inv_diag[0]);
  d.x = fmaf(-k, s.box[0], d.x);
  return d;
}

// The exact-rounding forms used by the cell and neighbour-list build, so that the lists
// are bit-identical to the f32 restatement of wgsl-common.js:81-123 (no FMA contraction,
// a true division, floor(x + 0.5)).
__device__ __forceinline__ float3 min_image_exact(float3 d, const DevSys &s) {
  float k = floorf(__fadd_rn(__fdiv_rn(d.z, s.box[8]), 0.5f));
  d.x = __fsub_rn(d.x, __fmul_rn(k, s.box[6]));
  d.y = __fsub_rn(d.y, __fmul_rn(k, s.box[7]));
  d.z = __fsub_rn(d.z, __fmul_rn(k, s.box[8]));
  k = floorf(__fadd_rn(__fdiv_rn(d.y, s.box[4]), 0.5f));
  d.x = __fsub_rn(d.x, __fmul_rn(k, s.box[3]));
  d.y = __fsub_rn(d.y, __fmul_rn(k, s.box[4]));
  d.z = __fsub_rn(d.z, __fmul_rn(k, s.box[5]));
  k = floorf(__fadd_rn(__fdiv_rn(d.x, s.box[0]), 0.5f));
  d.x = __fsub_rn(d.x, __fmul_rn(k, s.box[0]));
  d.y = __fsub_rn(d.y, __fmul_rn(k, s.box[1]));
  d.z = __fsub_rn(d.z, __fmul_rn(k, s.box[2]));
  return d;
}
__device__ __forceinline__ float dot_exact(float3 d) {
  return __fadd_rn(__fadd_rn(__fmul_rn(d.x, d.x), __fmul_rn(d.y, d.y)), __fmul_rn(d.z, d.z));
}
__device__ __forceinline__ float frac_exact(float3 p, const DevSys &s, int d) {
  return __fadd_rn(__fadd_rn(__fmul_rn(p.x, s.recip[d]), __fmul_rn(p.y, s.recip[3 + d])),
                   __fmul_rn(p.z, s.recip[6 + d]));
}
__device__ __forceinline__ int3 cell_coord(float3 p, const DevSys &s) {
  int c[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    float f = frac_exact(p, s, d);
    float wrapped = __fsub_rn(f, floorf(f));
    float scaled = __fmul_rn(wrapped, (float)s.cell_counts[d]);
    int v = (int)scaled;
    c[d] = min(v, s.cell_counts[d] - 1);
  }
  return make_int3(c[0], c[1], c[2]);
}

// ---------------------------------------------------------------- B-splines
// Cardinal B-spline weights and derivatives at a fractional offset; the derivative is
// read at order-1 before the final recursion step (shared/pme/parameters.js:121-149).
template <int ORDER>
__device__ __forceinline__ void bspline(float u, float *w, float *dw) {
  // The derivative below reads w[ORDER-1] before the last recursion step sets it: the
  // weights of order ORDER-1 padded with a zero, so every entry starts at zero.
#pragma unroll
  for (int k = 0; k < ORDER; ++k) w[k] = 0.0f;
  w[0] = 1.0f - u;
  w[1] = u;
#pragma unroll
  for (int k = 3; k < ORDER; ++k) {
    const float div = 1.0f / (float)(k - 1);
    w[k - 1] = div * u * w[k - 2];
#pragma unroll
    for (int j = 1; j < k - 1; ++j)
      w[k - j - 1] = div * ((u + (float)j) * w[k - j - 2] + ((float)(k - j) - u) * w[k - j - 1]);
    w[0] = div * (1.0f - u) * w[0];
  }
  dw[0] = -w[0];
#pragma unroll
  for (int j = 1; j < ORDER; ++j) dw[j] = w[j - 1] - w[j];
  const float div = 1.0f / (float)(ORDER - 1);
  w[ORDER - 1] = div * u * w[ORDER - 2];
#pragma unroll
  for (int j = 1; j < ORDER - 1; ++j)
    w[ORDER - j - 1] =
        div * ((u + (float)j) * w[ORDER - j - 2] + ((float)(ORDER - j) - u) * w[ORDER - j - 1]);
  w[0] = div * (1.0f - u) * w[0];
}

__device__ __forceinline__ int shift_code(int ka, int kb, int kc) { return (ka + 1) * 9 + (kb + 1) * 3 + (kc + 1); }
constexpr int NBR_SLOT_BITS = 27;
constexpr int NBR_SLOT_MASK = (1 << NBR_SLOT_BITS) - 1;

// Group-pair rows (pair_list 0/2): atoms are taken GROUP_ATOMS at a time (a search group: spatially
// close atoms of one cell in sub-cell order); a group's row lists each partner atom once, as
// slot | image code << 23 | mask << 28, where bit a of the 4-bit mask says that the group's atom
// a must skip this partner (an excluded pair, or a pair inside the group seen from its other
// atom). A pair of atoms in different groups is listed only in the row of the group that comes
// first in search order, so every pair is evaluated once.
constexpr int GROUP_ATOMS = 4;
constexpr int GROUP_SLOT_BITS = 23;
constexpr int GROUP_SLOT_MASK = (1 << GROUP_SLOT_BITS) - 1;
constexpr int GROUP_CODE_SHIFT = 23;
constexpr int GROUP_MASK_SHIFT = 28;

__device__ __forceinline__ int wrap_index(int v, int n) {
  int r = v % n;
  return r < 0 ? r + n : r;
}

// Float bit-pattern max for non-negative floats (NaN and Inf win: shared/finite.js:1-35).
__device__ __forceinline__ void atomic_max_nonneg(unsigned int *slot, float v) {
  atomicMax(slot, __float_as_uint(v));
}

}  // namespace rmd
