// Particle-mesh Ewald reciprocal space for a batch of systems.
//
// Same mathematics and conventions as RainMD's pme.js:137-345 / cpu/forces/pme.js:76-259:
// B-spline spreading with grid index (floor(u) + k - order + 1) mod K, signed frequencies,
// wave vectors from the ROWS of the inverse box, moduli dividing the kernel, the factor 2
// folded into the convolved grid, an unnormalised inverse transform, and no 1/2 in the
// force gather. The spline order is a template parameter (4 or 5).
//
// B200 design (not the reference's pass structure):
//   spread   ORDER^2 threads per atom, 64-bit fixed-point integer atomics (deterministic);
//   z pass   R2C: two real z-lines packed as one complex line, FFT in shared memory,
//            split into two half spectra; also converts fixed point -> f32 and zeroes the
//            fixed grid for the next step (no separate clear/convert kernels);
//   y pass   complex FFT along y on the half spectrum, in place;
//   x pass   forward FFT along x, the Ewald convolution and the FP64 energy partial, and
//            the inverse FFT along x, all while the lines are in shared memory;
//   y pass   inverse; z pass C2R back to a real f32 grid; gather four threads per atom.
//   planes   where a kz plane fits shared memory, the y pass, the x pass and the inverse y
//            pass are one kernel over whole planes: one block a plane for small planes, a
//            thread-block cluster a plane (distributed shared memory) for larger ones.
// Lines filled by a transpose (y and x passes) are padded to n + 1 in shared memory.
// The FFT is a mixed-radix (4, 2, 3, 5) Stockham autosort over lines held in shared
// memory; a host-built task table gives each block a set of lines of one system, so
// systems with different grid sizes run in the same launch.
#include <algorithm>

#include <cooperative_groups.h>

#include "common.cuh"
#include "kernels.h"

namespace rmd {

namespace cg = cooperative_groups;

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// multiply by -i (forward) or +i (inverse)
__device__ __forceinline__ float2 rot(float2 a, bool inverse) {
  return inverse ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <int R>
__device__ __forceinline__ void dft_small(float2 *v, bool inv) {
  if (R == 2) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (R == 4) {
    float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    float2 a2 = cadd(v[1], v[3]), a3 = rot(csub(v[1], v[3]), inv);
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    v[1] = cadd(a1, a3);
    v[3] = csub(a1, a3);
  } else if (R == 3) {
    const float h = 0.86602540378443864676f;  // sqrt(3)/2
    float2 t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    float2 b = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
    float2 r = rot(make_float2(h * t2.x, h * t2.y), inv);  // -i*h*t2 forward
    v[0] = cadd(v[0], t1);
    v[1] = cadd(b, r);
    v[2] = csub(b, r);
  } else if (R == 5) {
    const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
    const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
    float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    float2 b1 = make_float2(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
    float2 b2 = make_float2(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
    float2 q1 = rot(make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y), inv);
    float2 q2 = rot(make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y), inv);
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(b1, q1);
    v[4] = csub(b1, q1);
    v[2] = cadd(b2, q2);
    v[3] = csub(b2, q2);
  }
}

__device__ __forceinline__ int fast_div(int x, FastDiv f) {
  return (int)((__umulhi((uint32_t)x, f.magic) + (uint32_t)x) >> f.shift);
}

template <int R>
__device__ __forceinline__ void stockham_stage(const float2 *__restrict__ in, float2 *__restrict__ out,
                                               int lines, int N, int ld, int Ns, const float2 *tw,
                                               bool inv, FastDiv per_line_div, FastDiv span_div) {
  const int per_line = N / R;
  const int stride_tw = N / (Ns * R);
  for (int idx = threadIdx.x; idx < lines * per_line; idx += blockDim.x) {
    const int line = fast_div(idx, per_line_div), j = idx - line * per_line;
    const float2 *src = in + line * ld;
    float2 v[R];
    const int jq = fast_div(j, span_div);
    const int k = j - jq * Ns;
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[j + r * per_line];
#pragma unroll
    for (int r = 1; r < R; ++r) {
      float2 w = tw[k * r * stride_tw];
      if (inv) w.y = -w.y;
      v[r] = cmul(v[r], w);
    }
    dft_small<R>(v, inv);
    float2 *dst = out + line * ld + jq * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[r * Ns] = v[r];
  }
}

// Transform `lines` lines of length N held in a, line l starting at a + l * ld (ld >= N;
// lines filled by a transpose use ld = N + 1 so that the transposing accesses, which step
// by ld, fall in different shared-memory banks); returns the buffer holding the result. The
// twiddles tw are read as given (global or shared memory).
__device__ float2 *fft_stages(float2 *a, float2 *b, int lines, int N, int ld, const FftAxis &ax,
                              const float2 *tw, bool inv) {
  int Ns = 1;
  for (int st = 0; st < ax.nstages; ++st) {
    const int R = ax.radix[st];
    __syncthreads();
    const FastDiv pl = ax.per_line[st], sp = ax.span[st];
    if (R == 4) stockham_stage<4>(a, b, lines, N, ld, Ns, tw, inv, pl, sp);
    else if (R == 2) stockham_stage<2>(a, b, lines, N, ld, Ns, tw, inv, pl, sp);
    else if (R == 3) stockham_stage<3>(a, b, lines, N, ld, Ns, tw, inv, pl, sp);
    else stockham_stage<5>(a, b, lines, N, ld, Ns, tw, inv, pl, sp);
    Ns *= R;
    float2 *t = a;
    a = b;
    b = t;
  }
  __syncthreads();
  return a;
}

// Twiddle tables up to this length are read from shared memory.
constexpr int TW_CACHE = 512;

// fft_stages with the axis's twiddles first copied to shared memory, so the stages read them
// without a global round trip after each barrier (longer tables stay in global memory).
__device__ float2 *fft_lines(float2 *a, float2 *b, int lines, int N, int ld, const FftAxis &ax,
                             const float2 *tw, bool inv) {
  __shared__ float2 tw_cache[TW_CACHE];
  if (N <= TW_CACHE) {
    __syncthreads();  // a previous transform in this block has finished with the cache
    for (int k = threadIdx.x; k < N; k += blockDim.x) tw_cache[k] = tw[k];
    tw = tw_cache;    // visible after the barrier that opens the first stage
  }
  return fft_stages(a, b, lines, N, ld, ax, tw, inv);
}

constexpr int FFT_SMEM = 2048;  // complex values per buffer per block

// ------------------------------------------------------------------------ spreading
// ORDER*ORDER threads per atom: thread (kx, ky) adds the ORDER points of one z-row. Each
// thread recomputes the atom's splines (cheap) so no cross-thread exchange is needed, and
// the atom's p^3 atomics are issued by many threads at once instead of serially.
template <int ORDER>
__global__ void k_spread(const float4 *__restrict__ posq, const int *__restrict__ sys_of_atom,
                         const DevSys *__restrict__ sys, unsigned long long *__restrict__ fixed_grid,
                         int n_atoms) {
  chain_begin();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(t / (ORDER * ORDER));
  if (i >= n_atoms) return;
  const int kx = (int)(t % (ORDER * ORDER)) / ORDER, ky = (int)(t % ORDER);
  const float4 p = posq[i];
  if (p.w == 0.f) return;
  const DevSys &s = sys[sys_of_atom[i]];
  float w[3][ORDER], dw[3][ORDER];
  int base[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float f = p.x * s.recip[d] + p.y * s.recip[3 + d] + p.z * s.recip[6 + d];
    const float scaled = (f - floorf(f)) * (float)s.grid[d];
    const float fl = floorf(scaled);
    base[d] = (int)fl;
    bspline<ORDER>(scaled - fl, w[d], dw[d]);
  }
  const int nx = s.grid[0], ny = s.grid[1], nz = s.grid[2];
  const int ix = wrap_index(base[0] + kx - ORDER + 1, nx);
  const int iy = wrap_index(base[1] + ky - ORDER + 1, ny);
  float wx = 0.f, wy = 0.f;
#pragma unroll
  for (int k = 0; k < ORDER; ++k) {
    if (k == kx) wx = w[0][k];
    if (k == ky) wy = w[1][k];
  }
  const float wxy = p.w * wx * wy;
  unsigned long long *rowp = fixed_grid + s.grid_base + ((long long)ix * ny + iy) * nz;
#pragma unroll
  for (int kz = 0; kz < ORDER; ++kz) {
    const int iz = wrap_index(base[2] + kz - ORDER + 1, nz);
    atomicAdd(rowp + iz, to_fixed(wxy * w[2][kz]));
  }
}

// -------------------------------------------------------------- z pass, forward (R2C)
__global__ void __launch_bounds__(256) k_fft_z_r2c(const FftTask *__restrict__ tasks,
                                                   const DevSys *__restrict__ sys,
                                                   const FftPlan *__restrict__ plans,
                                                   const float2 *__restrict__ twiddles,
                                                   unsigned long long *__restrict__ fixed_grid,
                                                   float2 *__restrict__ half) {
  chain_begin();
  __shared__ float2 bufa[FFT_SMEM], bufb[FFT_SMEM];
  const FftTask t = tasks[blockIdx.x];
  const DevSys &s = sys[t.sys];
  const FftPlan &pl = plans[t.sys];
  const int N = s.grid[2], nzh = N / 2 + 1;
  const int nlines = s.grid[0] * s.grid[1];
  const int M = t.count;
  unsigned long long *g = fixed_grid + s.grid_base;
  for (int idx = threadIdx.x; idx < M * N; idx += blockDim.x) {
    const int p = fast_div(idx, pl.axis[2].n_div), k = idx - p * N;
    const int l = 2 * (t.first + p);
    unsigned long long *ra = g + (long long)l * N + k;
    const bool two = l + 1 < nlines;
    // both values read before either is cleared for the next step's spreading
    const unsigned long long va = ra[0];
    const unsigned long long vb = two ? ra[N] : 0ull;
    ra[0] = 0ull;
    if (two) ra[N] = 0ull;
    bufa[idx] = make_float2(from_fixed(va), two ? from_fixed(vb) : 0.f);
  }
  float2 *r = fft_lines(bufa, bufb, M, N, N, pl.axis[2], twiddles + pl.axis[2].tw_base, false);
  float2 *h = half + s.half_base;
  for (int idx = threadIdx.x; idx < M * nzh; idx += blockDim.x) {
    const int p = fast_div(idx, pl.axis[2].half_div), k = idx - p * nzh;
    const int l = 2 * (t.first + p);
    const float2 z = r[p * N + k];
    const float2 zc = r[p * N + (N - k) % N];
    // A = (Z + conj(Zc))/2, B = -i (Z - conj(Zc))/2
    const float2 a = make_float2(0.5f * (z.x + zc.x), 0.5f * (z.y - zc.y));
    const float2 b = make_float2(0.5f * (z.y + zc.y), -0.5f * (z.x - zc.x));
    h[(long long)l * nzh + k] = a;
    if (l + 1 < nlines) h[(long long)(l + 1) * nzh + k] = b;
  }
}

// -------------------------------------------------------------- z pass, inverse (C2R)
__global__ void __launch_bounds__(256) k_fft_z_c2r(const FftTask *__restrict__ tasks,
                                                   const DevSys *__restrict__ sys,
                                                   const FftPlan *__restrict__ plans,
                                                   const float2 *__restrict__ twiddles,
                                                   const float2 *__restrict__ half,
                                                   float *__restrict__ real_grid) {
  chain_begin();
  __shared__ float2 bufa[FFT_SMEM], bufb[FFT_SMEM];
  const FftTask t = tasks[blockIdx.x];
  const DevSys &s = sys[t.sys];
  const FftPlan &pl = plans[t.sys];
  const int N = s.grid[2], nzh = N / 2 + 1;
  const int nlines = s.grid[0] * s.grid[1];
  const int M = t.count;
  const float2 *h = half + s.half_base;
  for (int idx = threadIdx.x; idx < M * N; idx += blockDim.x) {
    const int p = fast_div(idx, pl.axis[2].n_div), k = idx - p * N;
    const int l = 2 * (t.first + p);
    const bool has_b = l + 1 < nlines;
    float2 a, b;
    if (k < nzh) {
      a = h[(long long)l * nzh + k];
      b = has_b ? h[(long long)(l + 1) * nzh + k] : make_float2(0.f, 0.f);
      if (k == 0 || 2 * k == N) {
        a.y = 0.f;
        b.y = 0.f;
      }
    } else {
      a = h[(long long)l * nzh + (N - k)];
      b = has_b ? h[(long long)(l + 1) * nzh + (N - k)] : make_float2(0.f, 0.f);
      a.y = -a.y;
      b.y = -b.y;
    }
    bufa[idx] = make_float2(a.x - b.y, a.y + b.x);  // A + iB
  }
  float2 *r = fft_lines(bufa, bufb, M, N, N, pl.axis[2], twiddles + pl.axis[2].tw_base, true);
  float *g = real_grid + s.grid_base;
  for (int idx = threadIdx.x; idx < M * N; idx += blockDim.x) {
    const int p = fast_div(idx, pl.axis[2].n_div), k = idx - p * N;
    const int l = 2 * (t.first + p);
    const float2 z = r[idx];
    g[(long long)l * N + k] = z.x;
    if (l + 1 < nlines) g[(long long)(l + 1) * N + k] = z.y;
  }
}

// ------------------------------------------------------ y pass (either direction, in place)
__global__ void __launch_bounds__(256) k_fft_y(const FftTask *__restrict__ tasks,
                                               const DevSys *__restrict__ sys,
                                               const FftPlan *__restrict__ plans,
                                               const float2 *__restrict__ twiddles,
                                               float2 *__restrict__ half, int inverse) {
  chain_begin();
  __shared__ float2 bufa[FFT_SMEM], bufb[FFT_SMEM];
  const FftTask t = tasks[blockIdx.x];
  const DevSys &s = sys[t.sys];
  const FftPlan &pl = plans[t.sys];
  const int ny = s.grid[1], nzh = s.grid[2] / 2 + 1;
  const int x = t.fixed, kz0 = t.first, M = t.count;
  float2 *h = half + s.half_base + (long long)x * ny * nzh + kz0;
  const int ld = ny + 1;  // padded lines (bank-conflict-free transpose)
  for (int idx = threadIdx.x; idx < ny * M; idx += blockDim.x) {
    const int y = idx / M, m = idx - y * M;
    bufa[m * ld + y] = h[(long long)y * nzh + m];
  }
  float2 *r = fft_lines(bufa, bufb, M, ny, ld, pl.axis[1], twiddles + pl.axis[1].tw_base, inverse != 0);
  for (int idx = threadIdx.x; idx < ny * M; idx += blockDim.x) {
    const int y = idx / M, m = idx - y * M;
    h[(long long)y * nzh + m] = r[m * ld + y];
  }
}

// ------------------------------ x pass: forward FFT, Ewald convolution + energy, inverse
template <bool ENERGY>
__global__ void __launch_bounds__(256) k_fft_x_convolve(const FftTask *__restrict__ tasks,
                                                        const DevSys *__restrict__ sys,
                                                        const DevSysD *__restrict__ sysd,
                                                        const FftPlan *__restrict__ plans,
                                                        const float2 *__restrict__ twiddles,
                                                        const float *__restrict__ moduli,
                                                        float2 *__restrict__ half,
                                                        double *__restrict__ e_pme,
                                                        double *__restrict__ e_pme_vir) {
  chain_begin();
  __shared__ float2 bufa[FFT_SMEM], bufb[FFT_SMEM];
  __shared__ double red[2][256 / 32];
  const FftTask t = tasks[blockIdx.x];
  const DevSys &s = sys[t.sys];
  const FftPlan &pl = plans[t.sys];
  const int nx = s.grid[0], ny = s.grid[1], nz = s.grid[2], nzh = nz / 2 + 1;
  const int y = t.fixed, kz0 = t.first, M = t.count;
  const long long stride = (long long)ny * nzh;
  float2 *h = half + s.half_base + (long long)y * nzh + kz0;
  const int ld = nx + 1;  // padded lines (bank-conflict-free transpose)
  for (int idx = threadIdx.x; idx < nx * M; idx += blockDim.x) {
    const int x = idx / M, m = idx - x * M;
    bufa[m * ld + x] = h[x * stride + m];
  }
  float2 *r = fft_lines(bufa, bufb, M, nx, ld, pl.axis[0], twiddles + pl.axis[0].tw_base, false);
  const double volume = sysd[t.sys].volume;
  const double alpha = sysd[t.sys].alpha;
  const float factor = (float)(M_PI * M_PI / (alpha * alpha));
  const float two_pref = (float)(2.0 * ONE_4PI_EPS0 / (2.0 * M_PI * volume));
  const float *modx = moduli + s.moduli_base, *mody = modx + nx, *modz = mody + ny;
  const int ky = y <= ny / 2 ? y : y - ny;
  double energy = 0.0, virial = 0.0;
  for (int idx = threadIdx.x; idx < nx * M; idx += blockDim.x) {
    const int m = idx / nx, mx = idx - m * nx;
    const int kz = kz0 + m;
    const int kx = mx <= nx / 2 ? mx : mx - nx;
    const int at = m * ld + mx;
    float2 v = r[at];
    if (kx == 0 && ky == 0 && kz == 0) {
      r[at] = make_float2(0.f, 0.f);
      continue;
    }
    const float fx = (float)kx, fy = (float)ky, fz = (float)kz;
    const float cx = fx * s.recip[0] + fy * s.recip[1] + fz * s.recip[2];
    const float cy = fx * s.recip[3] + fy * s.recip[4] + fz * s.recip[5];
    const float cz = fx * s.recip[6] + fy * s.recip[7] + fz * s.recip[8];
    const float m2 = cx * cx + cy * cy + cz * cz;
    const float kernel = __expf(-factor * m2) / (m2 * modx[mx] * mody[y] * modz[kz]);
    if (ENERGY) {
      const double weight = (kz == 0 || 2 * kz == nz) ? 1.0 : 2.0;
      const double ek = weight * 0.5 * (double)two_pref * (double)kernel * ((double)v.x * v.x + (double)v.y * v.y);
      energy += ek;
      virial += ek * (1.0 + (double)factor * (double)m2);
    }
    const float sc = kernel * two_pref;
    r[at] = make_float2(v.x * sc, v.y * sc);
  }
  float2 *other = (r == bufa) ? bufb : bufa;
  float2 *q = fft_lines(r, other, M, nx, ld, pl.axis[0], twiddles + pl.axis[0].tw_base, true);
  for (int idx = threadIdx.x; idx < nx * M; idx += blockDim.x) {
    const int x = idx / M, m = idx - x * M;
    h[x * stride + m] = q[m * ld + x];
  }
  if (ENERGY) {
    energy = warp_sum(energy);
    virial = warp_sum(virial);
    if ((threadIdx.x & 31) == 0) {
      red[0][threadIdx.x >> 5] = energy;
      red[1][threadIdx.x >> 5] = virial;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double total = 0, total_vir = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        total += red[0][w];
        total_vir += red[1][w];
      }
      e_pme[blockIdx.x] = total;
      e_pme_vir[blockIdx.x] = total_vir;
    }
  }
}

// ------------------------------------------------------------------------- gather
template <int ORDER>
__global__ void k_gather(const float4 *__restrict__ posq, const int *__restrict__ sys_of_atom,
                         const DevSys *__restrict__ sys, const float *__restrict__ real_grid,
                         unsigned long long *__restrict__ force, int n_atoms) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_atoms) return;
  const float4 p = posq[i];
  if (p.w == 0.f) return;
  const DevSys &s = sys[sys_of_atom[i]];
  float w[3][ORDER], dw[3][ORDER];
  int base[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float f = p.x * s.recip[d] + p.y * s.recip[3 + d] + p.z * s.recip[6 + d];
    const float scaled = (f - floorf(f)) * (float)s.grid[d];
    const float fl = floorf(scaled);
    base[d] = (int)fl;
    bspline<ORDER>(scaled - fl, w[d], dw[d]);
  }
  const int nx = s.grid[0], ny = s.grid[1], nz = s.grid[2];
  const float *g = real_grid + s.grid_base;
  float gu = 0.f, gv = 0.f, gw = 0.f;
#pragma unroll
  for (int kx = 0; kx < ORDER; ++kx) {
    const int ix = wrap_index(base[0] + kx - ORDER + 1, nx);
#pragma unroll
    for (int ky = 0; ky < ORDER; ++ky) {
      const int iy = wrap_index(base[1] + ky - ORDER + 1, ny);
      const float *rowp = g + ((long long)ix * ny + iy) * nz;
      const float wxy = w[0][kx] * w[1][ky], dxy = dw[0][kx] * w[1][ky], wdy = w[0][kx] * dw[1][ky];
#pragma unroll
      for (int kz = 0; kz < ORDER; ++kz) {
        const int iz = wrap_index(base[2] + kz - ORDER + 1, nz);
        const float v = __ldg(rowp + iz);
        gu = fmaf(dxy * w[2][kz], v, gu);
        gv = fmaf(wdy * w[2][kz], v, gv);
        gw = fmaf(wxy * dw[2][kz], v, gw);
      }
    }
  }
  const float su = gu * (float)nx * p.w, sv = gv * (float)ny * p.w, sw = gw * (float)nz * p.w;
  add_fixed(force + i, -(su * s.recip[0] + sv * s.recip[1] + sw * s.recip[2]));
  add_fixed(force + n_atoms + i, -(su * s.recip[3] + sv * s.recip[4] + sw * s.recip[5]));
  add_fixed(force + 2 * (long long)n_atoms + i, -(su * s.recip[6] + sv * s.recip[7] + sw * s.recip[8]));
}

// Force gather with four threads per atom (atoms in cell order, for locality of the grid
// reads): thread q sums the x-planes kx = q, q + 4 (< ORDER), the four partial gradients are
// combined with shuffles, and the first thread adds the force. One thread per atom leaves
// most of the GPU idle at these sizes (23,558 atoms are 185 blocks of 128).
template <int ORDER>
__global__ void k_gather4(const float4 *__restrict__ posq, const int *__restrict__ sorted_orig,
                          const int *__restrict__ sys_of_atom, const DevSys *__restrict__ sys,
                          const float *__restrict__ real_grid, unsigned long long *__restrict__ force,
                          int n_atoms) {
  chain_begin();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int slot = t >> 2, q = t & 3;
  const bool valid = slot < n_atoms;
  const int i = valid ? sorted_orig[slot] : 0;
  const float4 p = valid ? posq[i] : make_float4(0.f, 0.f, 0.f, 0.f);
  float gu = 0.f, gv = 0.f, gw = 0.f;
  const DevSys &s = sys[sys_of_atom[i]];
  if (valid && p.w != 0.f) {
    float w[3][ORDER], dw[3][ORDER];
    int base[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float f = p.x * s.recip[d] + p.y * s.recip[3 + d] + p.z * s.recip[6 + d];
      const float scaled = (f - floorf(f)) * (float)s.grid[d];
      const float fl = floorf(scaled);
      base[d] = (int)fl;
      bspline<ORDER>(scaled - fl, w[d], dw[d]);
    }
    const int nx = s.grid[0], ny = s.grid[1], nz = s.grid[2];
    const float *g = real_grid + s.grid_base;
    int iz[ORDER];
#pragma unroll
    for (int kz = 0; kz < ORDER; ++kz) iz[kz] = wrap_index(base[2] + kz - ORDER + 1, nz);
    // this thread's x-planes: kx = q (and q + 4 for order 5), weights selected without
    // branching so the four threads of an atom run the y and z loops in step
    for (int kx = q; kx < ORDER; kx += 4) {
      float wx = w[0][0], dwx = dw[0][0];
#pragma unroll
      for (int k = 1; k < ORDER; ++k) {
        wx = (kx == k) ? w[0][k] : wx;
        dwx = (kx == k) ? dw[0][k] : dwx;
      }
      const int ix = wrap_index(base[0] + kx - ORDER + 1, nx);
#pragma unroll
      for (int ky = 0; ky < ORDER; ++ky) {
        const int iy = wrap_index(base[1] + ky - ORDER + 1, ny);
        const float *rowp = g + ((long long)ix * ny + iy) * nz;
        const float wxy = wx * w[1][ky], dxy = dwx * w[1][ky], wdy = wx * dw[1][ky];
#pragma unroll
        for (int kz = 0; kz < ORDER; ++kz) {
          const float v = __ldg(rowp + iz[kz]);
          gu = fmaf(dxy * w[2][kz], v, gu);
          gv = fmaf(wdy * w[2][kz], v, gv);
          gw = fmaf(wxy * dw[2][kz], v, gw);
        }
      }
    }
  }
#pragma unroll
  for (int o = 1; o < 4; o <<= 1) {
    gu += __shfl_xor_sync(0xffffffffu, gu, o);
    gv += __shfl_xor_sync(0xffffffffu, gv, o);
    gw += __shfl_xor_sync(0xffffffffu, gw, o);
  }
  if (!valid || q != 0 || p.w == 0.f) return;
  // the convolved grid already carries the Coulomb prefactor (and the factor 2)
  const float su = gu * (float)s.grid[0] * p.w, sv = gv * (float)s.grid[1] * p.w, sw = gw * (float)s.grid[2] * p.w;
  add_fixed(force + i, -(su * s.recip[0] + sv * s.recip[1] + sw * s.recip[2]));
  add_fixed(force + n_atoms + i, -(su * s.recip[3] + sv * s.recip[4] + sw * s.recip[5]));
  add_fixed(force + 2 * (long long)n_atoms + i, -(su * s.recip[6] + sv * s.recip[7] + sw * s.recip[8]));
}

static void launch_gather(const LaunchCtx &c, cudaStream_t stream) {
  const int n = c.n_atoms, tb = 128;
  const int blocks = (int)(((long long)n * 4 + tb - 1) / tb);
  if (c.pme_order == 4)
    launch_chained(k_gather4<4>, blocks, tb, 0, stream, c.posq, c.sorted_orig, c.sys_of_atom, c.sys, c.real_grid, c.force, n);
  else
    launch_chained(k_gather4<5>, blocks, tb, 0, stream, c.posq, c.sorted_orig, c.sys_of_atom, c.sys, c.real_grid, c.force, n);
}

// Forward transform of the spread grid to the half spectrum (z and y; x is left to the caller).
static void launch_forward_zy(const LaunchCtx &c, cudaStream_t stream, bool all = false) {
  // A plain launch: the first FFT pass waits for the spreading's last atomics like any kernel
  // boundary. Chained after the spreading it was slower on one B200 at 64^3 (the seven
  // reciprocal kernels 0.067 against 0.049 ms, the 23,558-atom step 0.1394 against 0.1358 ms)
  // and no faster at 32^3 or 100^3. It still lets the next pass be scheduled early.
  k_fft_z_r2c<<<c.n_tasks_z, 256, 0, stream>>>(c.tasks_z, c.sys, c.fft_plans, c.twiddles, c.fixed_grid, c.half);
  const FftTask *ty = all ? c.tasks_y_all : c.tasks_y;
  const int n = all ? c.n_tasks_y_all : c.n_tasks_y;
  if (n > 0) launch_kernel(c.chain_pme, k_fft_y, n, 256, 0, stream, ty, c.sys, c.fft_plans, c.twiddles, c.half, 0);
}

static void launch_inverse_yz(const LaunchCtx &c, cudaStream_t stream, bool all = false) {
  const FftTask *ty = all ? c.tasks_y_all : c.tasks_y;
  const int n = all ? c.n_tasks_y_all : c.n_tasks_y;
  if (n > 0) launch_kernel(c.chain_pme, k_fft_y, n, 256, 0, stream, ty, c.sys, c.fft_plans, c.twiddles, c.half, 1);
  launch_kernel(c.chain_pme, k_fft_z_c2r, c.n_tasks_z, 256, 0, stream, c.tasks_z, c.sys, c.fft_plans, c.twiddles, c.half,
                c.real_grid);
}

// A plane pass's per-axis tables in shared memory: the y and x twiddles and B-spline moduli,
// copied once when the plane is loaded (in the same round trip as the plane) instead of before
// each of the four transforms. Planes on these passes have nx, ny <= TW_CACHE.
struct PlaneTables {
  float2 tw_y[TW_CACHE], tw_x[TW_CACHE];
  float mod_x[TW_CACHE], mod_y[TW_CACHE];
};

// Fill the tables (visible after the barrier that opens the first transform stage); returns
// the z moduli, read from global memory (one value a plane).
__device__ __forceinline__ const float *stage_plane_tables(PlaneTables &tab, const FftPlan &pl,
                                                           const float2 *__restrict__ twiddles,
                                                           const float *__restrict__ mod, int nx, int ny) {
  for (int k = threadIdx.x; k < ny; k += blockDim.x) {
    tab.tw_y[k] = twiddles[pl.axis[1].tw_base + k];
    tab.mod_y[k] = mod[nx + k];
  }
  for (int k = threadIdx.x; k < nx; k += blockDim.x) {
    tab.tw_x[k] = twiddles[pl.axis[0].tw_base + k];
    tab.mod_x[k] = mod[k];
  }
  return mod + nx + ny;
}

// The Ewald convolution of one half-spectrum point (x index mx, y index my, plane kz) in place,
// with its energy and virial terms added when ENERGY: the per-point arithmetic of
// k_fft_x_convolve, shared by the fused plane passes.
template <bool ENERGY>
__device__ __forceinline__ void convolve_point(float2 &v, int mx, int my, int kz, int nx, int ny, int nz,
                                               const DevSys &s, const float *modx, const float *mody,
                                               const float *modz, float factor, float two_pref,
                                               double &energy, double &virial) {
  const int kx = mx <= nx / 2 ? mx : mx - nx;
  const int ky = my <= ny / 2 ? my : my - ny;
  if (kx == 0 && ky == 0 && kz == 0) {
    v = make_float2(0.f, 0.f);
    return;
  }
  const float fx = (float)kx, fy = (float)ky, fz = (float)kz;
  const float cx = fx * s.recip[0] + fy * s.recip[1] + fz * s.recip[2];
  const float cy = fx * s.recip[3] + fy * s.recip[4] + fz * s.recip[5];
  const float cz = fx * s.recip[6] + fy * s.recip[7] + fz * s.recip[8];
  const float m2 = cx * cx + cy * cy + cz * cz;
  const float kernel = __expf(-factor * m2) / (m2 * modx[mx] * mody[my] * modz[kz]);
  if (ENERGY) {
    const double weight = (kz == 0 || 2 * kz == nz) ? 1.0 : 2.0;
    const double ek = weight * 0.5 * (double)two_pref * (double)kernel * ((double)v.x * v.x + (double)v.y * v.y);
    energy += ek;
    virial += ek * (1.0 + (double)factor * (double)m2);
  }
  const float sc = kernel * two_pref;
  v = make_float2(v.x * sc, v.y * sc);
}

// Block sum of a thread's energy and virial terms, written by thread 0 to e[slot], ev[slot].
__device__ __forceinline__ void block_energy(double energy, double virial, double *e, double *ev, int slot) {
  __shared__ double red[2][256 / 32];
  energy = warp_sum(energy);
  virial = warp_sum(virial);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = energy;
    red[1][threadIdx.x >> 5] = virial;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double total = 0, total_vir = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      total += red[0][w];
      total_vir += red[1][w];
    }
    e[slot] = total;
    ev[slot] = total_vir;
  }
}

// ----------------- y and x passes of one kz plane fused: forward y, forward x, the Ewald
// convolution (and energy), inverse x, inverse y, with the whole plane in shared memory. One
// block per (system, kz) plane of the half spectrum, for systems with small planes (see
// fft_plane_split): three launches and two trips of the half spectrum through L2 become
// one. The energy partial is the plane's, so a system's partials are grouped the same way in a
// batch as alone.
template <bool ENERGY>
__global__ void __launch_bounds__(256) k_fft_plane(const FftTask *__restrict__ tasks,
                                                   const DevSys *__restrict__ sys,
                                                   const DevSysD *__restrict__ sysd,
                                                   const FftPlan *__restrict__ plans,
                                                   const float2 *__restrict__ twiddles,
                                                   const float *__restrict__ moduli,
                                                   float2 *__restrict__ half, int plane_stride,
                                                   double *__restrict__ e_pme, double *__restrict__ e_pme_vir) {
  chain_begin();
  extern __shared__ float2 plane_smem[];
  __shared__ PlaneTables tab;
  float2 *bufa = plane_smem, *bufb = plane_smem + plane_stride;
  const FftTask t = tasks[blockIdx.x];
  const DevSys &s = sys[t.sys];
  const FftPlan &pl = plans[t.sys];
  const int nx = s.grid[0], ny = s.grid[1], nz = s.grid[2], nzh = nz / 2 + 1;
  const int kz = t.fixed;
  const int ldy = ny + 1, ldx = nx + 1;  // padded lines (bank-conflict-free transposes)
  float2 *h = half + s.half_base + kz;  // element (x, y) at h[(x * ny + y) * nzh]
  for (int idx = threadIdx.x; idx < nx * ny; idx += blockDim.x) {
    const int x = fast_div(idx, pl.axis[1].n_div), y = idx - x * ny;
    bufa[x * ldy + y] = h[(long long)idx * nzh];
  }
  const float *modz = stage_plane_tables(tab, pl, twiddles, moduli + s.moduli_base, nx, ny);
  // forward y: nx lines of ny
  float2 *r = fft_stages(bufa, bufb, nx, ny, ldy, pl.axis[1], tab.tw_y, false);
  float2 *o = (r == bufa) ? bufb : bufa;
  for (int idx = threadIdx.x; idx < nx * ny; idx += blockDim.x) {
    const int x = fast_div(idx, pl.axis[1].n_div), y = idx - x * ny;
    o[y * ldx + x] = r[x * ldy + y];
  }
  // forward x: ny lines of nx
  r = fft_stages(o, r, ny, nx, ldx, pl.axis[0], tab.tw_x, false);
  const double volume = sysd[t.sys].volume;
  const double alpha = sysd[t.sys].alpha;
  const float factor = (float)(M_PI * M_PI / (alpha * alpha));
  const float two_pref = (float)(2.0 * ONE_4PI_EPS0 / (2.0 * M_PI * volume));
  double energy = 0.0, virial = 0.0;
  for (int idx = threadIdx.x; idx < nx * ny; idx += blockDim.x) {
    const int y = fast_div(idx, pl.axis[0].n_div), mx = idx - y * nx;
    convolve_point<ENERGY>(r[y * ldx + mx], mx, y, kz, nx, ny, nz, s, tab.mod_x, tab.mod_y, modz, factor,
                           two_pref, energy, virial);
  }
  // inverse x
  o = (r == bufa) ? bufb : bufa;
  r = fft_stages(r, o, ny, nx, ldx, pl.axis[0], tab.tw_x, true);
  o = (r == bufa) ? bufb : bufa;
  for (int idx = threadIdx.x; idx < nx * ny; idx += blockDim.x) {
    const int x = fast_div(idx, pl.axis[1].n_div), y = idx - x * ny;
    o[x * ldy + y] = r[y * ldx + x];
  }
  // inverse y
  r = fft_stages(o, r, nx, ny, ldy, pl.axis[1], tab.tw_y, true);
  for (int idx = threadIdx.x; idx < nx * ny; idx += blockDim.x) {
    const int x = fast_div(idx, pl.axis[1].n_div), y = idx - x * ny;
    h[(long long)idx * nzh] = r[x * ldy + y];
  }
  if (ENERGY) block_energy(energy, virial, e_pme, e_pme_vir, blockIdx.x);
}

// The same fused pass for larger planes, shared by a thread-block cluster of PLANE_CLUSTER
// blocks so that a plane is not one block's serial chain. Block r of a cluster owns the x rows
// [r * rows_per, ...) for the y transforms and the y columns [r * cols_per, ...) for the x
// transforms and the convolution; between them each block gathers its lines from the other
// blocks' shared memory (distributed shared memory), with three cluster barriers: after the
// forward y pass (rows complete), after the inverse x pass (columns complete, and every block
// done reading the rows), and after the gather back (every block done reading the columns, so
// none exits while another still reads it). Every line goes through the same transform as in
// k_fft_plane; the energy partials are one per block of the cluster.
template <bool ENERGY>
__global__ void __cluster_dims__(PLANE_CLUSTER, 1, 1) __launch_bounds__(256)
    k_fft_plane_cluster(const FftTask *__restrict__ tasks, const DevSys *__restrict__ sys,
                        const DevSysD *__restrict__ sysd, const FftPlan *__restrict__ plans,
                        const float2 *__restrict__ twiddles, const float *__restrict__ moduli,
                        float2 *__restrict__ half, int row_stride, int col_stride,
                        double *__restrict__ e_pme, double *__restrict__ e_pme_vir) {
  chain_begin();
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  extern __shared__ float2 plane_smem[];
  __shared__ PlaneTables tab;
  float2 *ra = plane_smem, *rb = ra + row_stride, *ca = rb + row_stride, *cb = ca + col_stride;
  const FftTask t = tasks[blockIdx.x / PLANE_CLUSTER];
  const DevSys &s = sys[t.sys];
  const FftPlan &pl = plans[t.sys];
  const int nx = s.grid[0], ny = s.grid[1], nz = s.grid[2], nzh = nz / 2 + 1;
  const int kz = t.fixed;
  const int ldy = ny + 1, ldx = nx + 1;
  const int rows_per = (nx + PLANE_CLUSTER - 1) / PLANE_CLUSTER, cols_per = (ny + PLANE_CLUSTER - 1) / PLANE_CLUSTER;
  const int x0 = min(nx, rank * rows_per), nr = min(nx, x0 + rows_per) - x0;
  const int y0 = min(ny, rank * cols_per), nc = min(ny, y0 + cols_per) - y0;
  float2 *h = half + s.half_base + kz;  // element (x, y) at h[(x * ny + y) * nzh]
  for (int idx = threadIdx.x; idx < nr * ny; idx += blockDim.x) {
    const int xl = fast_div(idx, pl.axis[1].n_div), y = idx - xl * ny;
    ra[xl * ldy + y] = h[((long long)(x0 + xl) * ny + y) * nzh];
  }
  const float *modz = stage_plane_tables(tab, pl, twiddles, moduli + s.moduli_base, nx, ny);
  // forward y over this block's rows; every block runs the same stages, so the result sits
  // at the same offset in each block's shared memory
  const float2 *rows = fft_stages(ra, rb, nr, ny, ldy, pl.axis[1], tab.tw_y, false);
  cluster.sync();
  for (int idx = threadIdx.x; idx < nc * nx; idx += blockDim.x) {
    const int yl = fast_div(idx, pl.axis[0].n_div), x = idx - yl * nx;
    const int owner = x / rows_per;
    const float2 *src = cluster.map_shared_rank(rows, owner);
    ca[yl * ldx + x] = src[(x - owner * rows_per) * ldy + y0 + yl];
  }
  // forward x over this block's columns, the convolution, inverse x
  float2 *c = fft_stages(ca, cb, nc, nx, ldx, pl.axis[0], tab.tw_x, false);
  const double volume = sysd[t.sys].volume;
  const double alpha = sysd[t.sys].alpha;
  const float factor = (float)(M_PI * M_PI / (alpha * alpha));
  const float two_pref = (float)(2.0 * ONE_4PI_EPS0 / (2.0 * M_PI * volume));
  double energy = 0.0, virial = 0.0;
  for (int idx = threadIdx.x; idx < nc * nx; idx += blockDim.x) {
    const int yl = fast_div(idx, pl.axis[0].n_div), mx = idx - yl * nx;
    convolve_point<ENERGY>(c[yl * ldx + mx], mx, y0 + yl, kz, nx, ny, nz, s, tab.mod_x, tab.mod_y, modz, factor,
                           two_pref, energy, virial);
  }
  const float2 *cols = fft_stages(c, c == ca ? cb : ca, nc, nx, ldx, pl.axis[0], tab.tw_x, true);
  cluster.sync();
  for (int idx = threadIdx.x; idx < nr * ny; idx += blockDim.x) {
    const int xl = fast_div(idx, pl.axis[1].n_div), y = idx - xl * ny;
    const int owner = y / cols_per;
    const float2 *src = cluster.map_shared_rank(cols, owner);
    ra[xl * ldy + y] = src[(y - owner * cols_per) * ldx + x0 + xl];
  }
  cluster.sync();
  // inverse y over this block's rows
  const float2 *r = fft_stages(ra, rb, nr, ny, ldy, pl.axis[1], tab.tw_y, true);
  for (int idx = threadIdx.x; idx < nr * ny; idx += blockDim.x) {
    const int xl = fast_div(idx, pl.axis[1].n_div), y = idx - xl * ny;
    h[((long long)(x0 + xl) * ny + y) * nzh] = r[xl * ldy + y];
  }
  if (ENERGY) block_energy(energy, virial, e_pme, e_pme_vir, blockIdx.x);
}

// Planes of at most this many points go to one block each. A block's plane is one serial
// chain, so larger grids run faster shared by a cluster: measured on one B200 (the seven
// reciprocal kernels) one block a plane is faster than the separate passes at 32^3 (0.037
// against 0.041 ms) and for 64 grids of 22^3-50^3 together (0.30 against 0.34 ms), slower at
// 64^3 (0.071 against 0.056 ms) and 100^3 (0.194 against 0.152 ms). A cluster a plane for
// those 64 small grids too was slower again (0.375 ms): their 1,150 planes fill the GPU already.
constexpr long long PLANE_SINGLE_MAX = 52 * 52;

void fft_plane_buffers(int nx, int ny, int split, int *rows, int *cols) {
  if (split == 1) {
    *rows = *cols = std::max(nx * (ny + 1), ny * (nx + 1));
    return;
  }
  *rows = (nx + split - 1) / split * (ny + 1);
  *cols = (ny + split - 1) / split * (nx + 1);
}

// The rule depends on the system alone, so a system takes the same pass in a batch as alone.
// A cluster block's row and column buffers are each held to half the limit, so that the
// largest rows and the largest columns of different systems in one launch still fit together.
int fft_plane_split(int nx, int ny) {
  int rows, cols;
  fft_plane_buffers(nx, ny, 1, &rows, &cols);
  if (nx > TW_CACHE || ny > TW_CACHE) return 0;
  if ((long long)nx * ny <= PLANE_SINGLE_MAX && 2LL * rows * (long long)sizeof(float2) <= FFT_PLANE_SMEM_MAX) return 1;
  if (nx < PLANE_CLUSTER || ny < PLANE_CLUSTER) return 0;
  fft_plane_buffers(nx, ny, PLANE_CLUSTER, &rows, &cols);
  const long long half_limit = FFT_PLANE_SMEM_MAX / 2;
  if (2LL * rows * (long long)sizeof(float2) <= half_limit && 2LL * cols * (long long)sizeof(float2) <= half_limit)
    return PLANE_CLUSTER;
  return 0;
}

// The largest dynamic shared memory the plane kernels may take, set once per device before any
// launch (and never lowered, so engines with different grids cannot undercut each other).
cudaError_t fft_plane_prepare() {
  const void *fns[4] = {(const void *)k_fft_plane<true>, (const void *)k_fft_plane<false>,
                        (const void *)k_fft_plane_cluster<true>, (const void *)k_fft_plane_cluster<false>};
  for (const void *f : fns) {
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FFT_PLANE_SMEM_MAX);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

static void launch_planes(const LaunchCtx &c, bool energy, cudaStream_t stream) {
  // partials after the x tasks': the planes' one each, then the clusters' PLANE_CLUSTER each
  double *e = c.e_pme + c.n_tasks_x, *ev = c.e_pme_vir + c.n_tasks_x;
  if (c.n_tasks_plane > 0) {
    const size_t smem = 2 * (size_t)c.plane_stride * sizeof(float2);
    launch_kernel(c.chain_pme, energy ? k_fft_plane<true> : k_fft_plane<false>, c.n_tasks_plane, 256, smem, stream,
                   c.tasks_plane, c.sys, c.sysd, c.fft_plans, c.twiddles, c.moduli, c.half, c.plane_stride, e, ev);
  }
  if (c.n_tasks_cluster > 0) {
    e += c.n_tasks_plane;
    ev += c.n_tasks_plane;
    const size_t smem = 2 * ((size_t)c.cluster_rows + c.cluster_cols) * sizeof(float2);
    launch_kernel(c.chain_pme, energy ? k_fft_plane_cluster<true> : k_fft_plane_cluster<false>,
                  c.n_tasks_cluster * PLANE_CLUSTER,
                   256, smem, stream, c.tasks_cluster, c.sys, c.sysd, c.fft_plans, c.twiddles, c.moduli, c.half,
                   c.cluster_rows, c.cluster_cols, e, ev);
  }
}

int pme_launches(const LaunchCtx &c) {
  if (!c.pme_on) return 0;
  return 4 + (c.n_tasks_plane > 0 ? 1 : 0) + (c.n_tasks_cluster > 0 ? 1 : 0) + (c.n_tasks_x > 0 ? 3 : 0);
}

// Everything up to the convolved real grid: spreading, forward transform, convolution (and
// energy), inverse transform.
static void launch_transform_convolve(const LaunchCtx &c, bool energy, cudaStream_t stream) {
  launch_forward_zy(c, stream);
  launch_planes(c, energy, stream);
  if (c.n_tasks_x > 0)
    launch_kernel(c.chain_pme, energy ? k_fft_x_convolve<true> : k_fft_x_convolve<false>, c.n_tasks_x, 256, 0, stream,
                   c.tasks_x, c.sys, c.sysd, c.fft_plans, c.twiddles, c.moduli, c.half, c.e_pme, c.e_pme_vir);
  launch_inverse_yz(c, stream);
}

void launch_pme_grid(const LaunchCtx &c, bool energy, cudaStream_t stream) {
  if (!c.pme_on) return;
  launch_spread_only(c, stream);
  launch_transform_convolve(c, energy, stream);
}

void launch_pme_gather(const LaunchCtx &c, cudaStream_t stream) {
  if (c.pme_on) launch_gather(c, stream);
}

void launch_pme(const LaunchCtx &c, bool energy, cudaStream_t stream) {
  if (!c.pme_on) return;
  launch_spread_only(c, stream);
  launch_transform_convolve(c, energy, stream);
  launch_gather(c, stream);
}

// Debug: forward R2C then C2R of a given real grid (already in real_grid as f32 values
// converted to fixed point by the caller), without the convolution. Used to check the FFT
// against a DFT.
__global__ void k_fft_x_plain(const FftTask *__restrict__ tasks, const DevSys *__restrict__ sys,
                              const FftPlan *__restrict__ plans, const float2 *__restrict__ twiddles,
                              float2 *__restrict__ half, int inverse) {
  __shared__ float2 bufa[FFT_SMEM], bufb[FFT_SMEM];
  const FftTask t = tasks[blockIdx.x];
  const DevSys &s = sys[t.sys];
  const FftPlan &pl = plans[t.sys];
  const int nx = s.grid[0], ny = s.grid[1], nzh = s.grid[2] / 2 + 1;
  const int y = t.fixed, kz0 = t.first, M = t.count;
  const long long stride = (long long)ny * nzh;
  float2 *h = half + s.half_base + (long long)y * nzh + kz0;
  const int ld = nx + 1;
  for (int idx = threadIdx.x; idx < nx * M; idx += blockDim.x) {
    const int x = idx / M, m = idx - x * M;
    bufa[m * ld + x] = h[x * stride + m];
  }
  float2 *r = fft_lines(bufa, bufb, M, nx, ld, pl.axis[0], twiddles + pl.axis[0].tw_base, inverse != 0);
  for (int idx = threadIdx.x; idx < nx * M; idx += blockDim.x) {
    const int x = idx / M, m = idx - x * M;
    h[x * stride + m] = r[m * ld + x];
  }
}

void launch_spread_only(const LaunchCtx &c, cudaStream_t stream) {
  const int n = c.n_atoms;
  const int per_block = c.spread_atoms > 0 ? c.spread_atoms : 8;
  const int blocks = (n + per_block - 1) / per_block;
  if (c.pme_order == 4)
    launch_kernel(c.chain_pme, k_spread<4>, blocks, per_block * 16, 0, stream, c.posq, c.sys_of_atom, c.sys,
                  c.fixed_grid, n);
  else
    launch_kernel(c.chain_pme, k_spread<5>, blocks, per_block * 25, 0, stream, c.posq, c.sys_of_atom, c.sys,
                  c.fixed_grid, n);
}

// (the debug transforms run the separate passes over every system)
void launch_fft_forward(const LaunchCtx &c, cudaStream_t stream) {
  launch_forward_zy(c, stream, true);
  k_fft_x_plain<<<c.n_tasks_x_all, 256, 0, stream>>>(c.tasks_x_all, c.sys, c.fft_plans, c.twiddles, c.half, 0);
}

void launch_fft_inverse(const LaunchCtx &c, cudaStream_t stream) {
  k_fft_x_plain<<<c.n_tasks_x_all, 256, 0, stream>>>(c.tasks_x_all, c.sys, c.fft_plans, c.twiddles, c.half, 1);
  launch_inverse_yz(c, stream, true);
}

}  // namespace rmd
