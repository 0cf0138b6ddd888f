// On-device trajectory output: whole-molecule imaging and the DCD and AMBER-restart byte
// layouts, written straight from the position buffer into a device staging buffer, so a frame
// crosses PCIe once, already packed.
//
// The byte layouts and the arithmetic are the reference writers' (shared/traj/imaging.js:
// 39-91, shared/traj/dcd.js:96-240, shared/traj/rst7.js:20-101), including the float64
// evaluation order of the JavaScript they run in: every FP64 operation below is an explicitly
// rounded intrinsic, so no fused multiply-add changes a bit, and the restart's decimal fields
// follow ECMAScript's Number.prototype.toFixed exactly (the integer n nearest to x * 10^7 on
// the double's exact binary value, the larger n on a tie), computed in 128-bit integers.
#include <climits>
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "kernels.h"

namespace rmd {

// ---------------------------------------------------------------- imaging
// One thread per molecule: the FP64 centroid of its atoms in atom order (the order the
// reference's single pass over atoms accumulates in), then the integer lattice translation
// taking it into the cell, c then b then a (imaging.js:60-82).
__global__ void k_traj_shifts(TrajArgs t) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= t.mol_count) return;
  const DevSysD &d = t.sysd[t.sys];
  const double ax = d.box[0], bx = d.box[3], by = d.box[4], cx = d.box[6], cy = d.box[7], cz = d.box[8];
  // -0.0 leaves every coordinate's bits as they are, a -0.0 included (x + -0.0 == x)
  double3 shift = make_double3(-0.0, -0.0, -0.0);
  const int g = t.mol_first + m;
  const int begin = t.mol_start[g], end = t.mol_start[g + 1];
  if (ax > 0.0 && by > 0.0 && cz > 0.0 && end > begin) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int k = begin; k < end; ++k) {
      const float4 p = t.posq[t.mol_atoms[k]];
      sx = __dadd_rn(sx, (double)p.x);
      sy = __dadd_rn(sy, (double)p.y);
      sz = __dadd_rn(sz, (double)p.z);
    }
    const double size = (double)(end - begin);
    const double x = __ddiv_rn(sx, size), y = __ddiv_rn(sy, size), z = __ddiv_rn(sz, size);
    const double nc = floor(__ddiv_rn(z, cz));
    const double y_c = __dsub_rn(y, __dmul_rn(nc, cy));
    const double nb = floor(__ddiv_rn(y_c, by));
    const double x_cb = __dsub_rn(__dsub_rn(x, __dmul_rn(nc, cx)), __dmul_rn(nb, bx));
    const double na = floor(__ddiv_rn(x_cb, ax));
    shift.x = -__dadd_rn(__dadd_rn(__dmul_rn(na, ax), __dmul_rn(nb, bx)), __dmul_rn(nc, cx));
    shift.y = -__dadd_rn(__dmul_rn(nb, by), __dmul_rn(nc, cy));
    shift.z = -__dmul_rn(nc, cz);
  }
  t.shift[m] = shift;
}

__device__ __forceinline__ bool finite3(float4 p) { return isfinite(p.x) && isfinite(p.y) && isfinite(p.z); }

// The wrapped FP64 coordinates (imaging.js:84-89): position + the molecule's translation.
__global__ void k_traj_image(TrajArgs t, double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= t.atom_count) return;
  const int a = t.atom_start + i;
  const float4 p = t.posq[a];
  const double3 s = t.image ? t.shift[t.mol_of_atom[a] - t.mol_first] : make_double3(-0.0, -0.0, -0.0);
  out[3 * (long long)i] = __dadd_rn((double)p.x, s.x);
  out[3 * (long long)i + 1] = __dadd_rn((double)p.y, s.y);
  out[3 * (long long)i + 2] = __dadd_rn((double)p.z, s.z);
}

// ---------------------------------------------------------------- DCD
// Separately rounded FP64 operations on both sides (the host compiler targets x86-64 without
// FMA, so plain operators are already separately rounded there).
#ifdef __CUDA_ARCH__
#define TRAJ_MUL(a, b) __dmul_rn((a), (b))
#define TRAJ_ADD(a, b) __dadd_rn((a), (b))
#define TRAJ_SUB(a, b) __dsub_rn((a), (b))
#else
#define TRAJ_MUL(a, b) ((a) * (b))
#define TRAJ_ADD(a, b) ((a) + (b))
#define TRAJ_SUB(a, b) ((a) - (b))
#endif

// The hypotenuse as an ECMAScript engine computes Math.hypot: the arguments scaled by the
// largest magnitude, their squares summed with Kahan compensation in argument order, then the
// square root times the scale. Exact for the axis-aligned vectors of a rectangular box.
__host__ __device__ inline double script_hypot3(double x, double y, double z) {
  const double v[3] = {fabs(x), fabs(y), fabs(z)};
  double top = 0.0;
  for (double a : v)
    if (a > top) top = a;
  if (top == 0.0) return 0.0;
  double sum = 0.0, carry = 0.0;
  for (double a : v) {
    const double n = a / top;
    const double term = TRAJ_SUB(TRAJ_MUL(n, n), carry);
    const double next = TRAJ_ADD(sum, term);
    carry = TRAJ_SUB(TRAJ_SUB(next, sum), term);
    sum = next;
  }
  return TRAJ_MUL(sqrt(sum), top);
}

// dcd.js:214-230: [a, cos(gamma), b, cos(beta), cos(alpha), c], lengths in angstroms.
__host__ __device__ inline void dcd_cell(const double *v, double cell[6]) {
  const double la = script_hypot3(v[0], v[1], v[2]), lb = script_hypot3(v[3], v[4], v[5]),
               lc = script_hypot3(v[6], v[7], v[8]);
  auto dot = [](const double *u, const double *w) {
    return TRAJ_ADD(TRAJ_ADD(TRAJ_MUL(u[0], w[0]), TRAJ_MUL(u[1], w[1])), TRAJ_MUL(u[2], w[2]));
  };
  const double bc = TRAJ_MUL(lb, lc), ac = TRAJ_MUL(la, lc), ab = TRAJ_MUL(la, lb);
  const double cos_alpha = bc > 0 ? dot(v + 3, v + 6) / bc : 0.0;
  const double cos_beta = ac > 0 ? dot(v, v + 6) / ac : 0.0;
  const double cos_gamma = ab > 0 ? dot(v, v + 3) / ab : 0.0;
  cell[0] = TRAJ_MUL(la, 10.0);
  cell[1] = cos_gamma;
  cell[2] = TRAJ_MUL(lb, 10.0);
  cell[3] = cos_beta;
  cell[4] = cos_alpha;
  cell[5] = TRAJ_MUL(lc, 10.0);
}

__device__ __forceinline__ void put_u32(unsigned char *p, unsigned v) {
  *reinterpret_cast<unsigned *>(p) = v;  // every field of a frame starts on a 4-byte boundary
}

// One thread per atom: the imaged coordinate in angstroms rounded to f32 (dcd.js:136-141),
// written into its axis record; thread 0 also writes the record markers and the cell record.
// A non-finite input coordinate is recorded (its atom index) and the frame refused.
__global__ void k_dcd_pack(TrajArgs t, int periodic) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = t.atom_count;
  const long long base = periodic ? 56 : 0, axis = 4 * n + 8;
  if (i == 0) {
    for (int k = 0; k < 3; ++k) {
      put_u32(t.out + base + k * axis, (unsigned)(4 * n));
      put_u32(t.out + base + k * axis + 4 + 4 * n, (unsigned)(4 * n));
    }
    if (periodic) {
      double cell[6];
      dcd_cell(t.sysd[t.sys].box, cell);
      put_u32(t.out, 48u);
      for (int k = 0; k < 6; ++k) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(cell[k]);
        put_u32(t.out + 4 + 8 * k, (unsigned)(b & 0xffffffffull));
        put_u32(t.out + 8 + 8 * k, (unsigned)(b >> 32));
      }
      put_u32(t.out + 52, 48u);
    }
  }
  if (i >= n) return;
  const int a = t.atom_start + i;
  const float4 p = t.posq[a];
  if (!finite3(p)) atomicMin(t.status, i);
  const double3 s = t.image ? t.shift[t.mol_of_atom[a] - t.mol_first] : make_double3(-0.0, -0.0, -0.0);
  const float x = __double2float_rn(__dmul_rn(__dadd_rn((double)p.x, s.x), 10.0));
  const float y = __double2float_rn(__dmul_rn(__dadd_rn((double)p.y, s.y), 10.0));
  const float z = __double2float_rn(__dmul_rn(__dadd_rn((double)p.z, s.z), 10.0));
  put_u32(t.out + base + 4 + 4 * i, __float_as_uint(x));
  put_u32(t.out + base + axis + 4 + 4 * i, __float_as_uint(y));
  put_u32(t.out + base + 2 * axis + 4 + 4 * i, __float_as_uint(z));
}

// ---------------------------------------------------------------- AMBER restart
// ECMAScript x.toFixed(7) right-aligned in 12 columns (rst7.js:45-50). Returns the field's
// length before padding (> 12 means it does not fit and nothing is meaningful in `field`).
__host__ __device__ inline int fixed7_field(double x, char field[12]) {
  const bool neg = x < 0.0;
  const double a = neg ? -x : x;
  if (!(a < 1048576.0)) return 13;  // 2^20: at least seven integer digits, never fits
  unsigned long long n = 0;
  if (a > 0.0) {
    unsigned long long bits;
    memcpy(&bits, &a, 8);
    const int ex = (int)(bits >> 52);
    unsigned long long m = bits & ((1ull << 52) - 1);
    int e;
    if (ex == 0) {
      e = -1074;  // subnormal
    } else {
      m |= 1ull << 52;
      e = ex - 1075;
    }
    // a * 10^7 = m * 10^7 / 2^k exactly, k = -e >= 32 for a < 2^20
    const int k = -e;
    const unsigned __int128 P = (unsigned __int128)m * 10000000u;
    if (k < 127) {
      const unsigned __int128 q = P >> k, r = P - (q << k), half = (unsigned __int128)1 << (k - 1);
      n = (unsigned long long)q + (r >= half ? 1u : 0u);
    }
  }
  const unsigned long long ip = n / 10000000ull, frac = n % 10000000ull;
  char digits[24];
  int nd = 0;
  unsigned long long v = ip;
  do {
    digits[nd++] = (char)('0' + v % 10);
    v /= 10;
  } while (v);
  const int len = (neg ? 1 : 0) + nd + 8;
  if (len > 12) return len;
  int c = 0;
  for (; c < 12 - len; ++c) field[c] = ' ';
  if (neg) field[c++] = '-';
  for (int d = nd - 1; d >= 0; --d) field[c++] = digits[d];
  field[c++] = '.';
  unsigned long long f = frac;
  for (int d = 6; d >= 0; --d) {
    field[c + d] = (char)('0' + f % 10);
    f /= 10;
  }
  return len;
}

// Bytes of a block of `values` fields, six to a line, each line ending in a newline.
__host__ __device__ inline long long rst7_block_bytes(long long values) {
  return (values / 6) * 73 + (values % 6 ? (values % 6) * 12 + 1 : 0);
}

// One thread per value: positions in angstroms (x / 0.1), then velocities in angstroms per
// AMBER time unit (v / (20.455 * 0.1)), then the six box numbers; each formatted into its
// fixed place. The first value (in file order) that is non-finite or too wide is recorded.
__global__ void k_rst7_format(TrajArgs t, long long header, int velocities, int box, Rst7Box b) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n3 = 3ll * t.atom_count;
  const long long total = n3 * (velocities ? 2 : 1) + (box ? 6 : 0);
  if (k >= total) return;
  long long j = k, start = header, count = n3;
  double v;
  if (k < n3) {
    const float4 p = t.posq[t.atom_start + k / 3];
    const float c = k % 3 == 0 ? p.x : (k % 3 == 1 ? p.y : p.z);
    v = __ddiv_rn((double)c, 0.1);
  } else if (velocities && k < 2 * n3) {
    j = k - n3;
    start = header + rst7_block_bytes(n3);
    const float4 u = t.vel[t.atom_start + j / 3];
    const float c = j % 3 == 0 ? u.x : (j % 3 == 1 ? u.y : u.z);
    v = __ddiv_rn((double)c, b.velocity_unit);
  } else {
    j = k - n3 * (velocities ? 2 : 1);
    start = header + rst7_block_bytes(n3) * (velocities ? 2 : 1);
    count = 6;
    v = b.values[j];
  }
  char *dst = reinterpret_cast<char *>(t.out) + start + (j / 6) * 73 + (j % 6) * 12;
  if (!isfinite(v)) {
    atomicMin(t.status, (int)k);
    return;
  }
  char field[12];
  if (fixed7_field(v, field) > 12) {
    atomicMin(t.status + 1, (int)k);
    return;
  }
  for (int c = 0; c < 12; ++c) dst[c] = field[c];
  if (j % 6 == 5 || j == count - 1) dst[12] = '\n';
}

// ---------------------------------------------------------------- launchers
void launch_traj_shifts(const TrajArgs &t, cudaStream_t stream) {
  if (t.mol_count > 0) k_traj_shifts<<<(t.mol_count + 127) / 128, 128, 0, stream>>>(t);
}
void launch_traj_image(const TrajArgs &t, double *out, cudaStream_t stream) {
  k_traj_image<<<(t.atom_count + 255) / 256, 256, 0, stream>>>(t, out);
}
void launch_dcd_pack(const TrajArgs &t, int periodic, cudaStream_t stream) {
  k_dcd_pack<<<(t.atom_count + 255) / 256, 256, 0, stream>>>(t, periodic);
}
void launch_rst7_format(const TrajArgs &t, long long header, int velocities, int box, const Rst7Box &b,
                        cudaStream_t stream) {
  const long long total = 3ll * t.atom_count * (velocities ? 2 : 1) + (box ? 6 : 0);
  k_rst7_format<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(t, header, velocities, box, b);
}

// ---------------------------------------------------------------- host helpers
int fixed7_text(double x, char field[12]) { return fixed7_field(x, field); }
long long rst7_block_size(long long values) { return rst7_block_bytes(values); }
void dcd_cell_host(const double *box, double cell[6]) { dcd_cell(box, cell); }
double script_hypot(double x, double y, double z) { return script_hypot3(x, y, z); }

}  // namespace rmd
