// BAOAB Langevin integration with SHAKE/RATTLE (or SETTLE for rigid 3-site water), fused.
//
// The step is RainMD's (integrate.js:523-558, cpu/integrate/langevin.js:30-135):
//     B R  A S  O R  A S  [forces]  B R
// B = half kick, R = RATTLE, A = half drift, S = SHAKE with the velocity corrected by the
// accumulated position correction / h, O = Ornstein-Uhlenbeck with the counter RNG.
// Every operation is per atom or per constraint cluster, and clusters share no atom, so
// one thread owning a unit (a free atom or a whole cluster) can apply the entire sequence
// to its atoms in registers with no synchronisation. The reference launches eight passes
// per step for this; here it is one kernel, and the closing "B R" of step n is fused into
// the same launch as the opening "B R A S O R A S" of step n+1 (both use the same forces).
// The same launch records the skin displacement (max |x - x_build|^2 per system, as float
// bits so NaN/Inf win; displacement.js:43-107) and, when asked, per-atom kinetic energies.
#include "common.cuh"
#include "kernels.h"

namespace rmd {

// A unit's atoms, held in registers when CAP is small and every index is static (free
// atoms: CAP 1, SETTLE waters: CAP 3); generic SHAKE clusters use CAP = MAX_CLUSTER_ATOMS.
template <int CAP>
struct UnitState {
  int n;
  int atom[CAP];
  float x[CAP][3], v[CAP][3], im[CAP], f[CAP][3];
  float ref[CAP][3], corr[CAP][3];
};

struct ConstraintSet {
  int n;
  int a[MAX_CLUSTER_CONSTRAINTS], b[MAX_CLUSTER_CONSTRAINTS];
  float d[MAX_CLUSTER_CONSTRAINTS];
};

struct SolverDiag {
  int max_iterations;
  int shake_cap, rattle_cap;
  float stalled_residual;
};

template <int CAP>
__device__ __forceinline__ void kick(UnitState<CAP> &u, float h) {
#pragma unroll
  for (int k = 0; k < CAP; ++k) {
    if (k >= u.n || u.im[k] <= 0.f) continue;
    const float sc = h * u.im[k];
#pragma unroll
    for (int c = 0; c < 3; ++c) u.v[k][c] = fmaf(sc, u.f[k][c], u.v[k][c]);
  }
}

// integrate.js:337-395
__device__ void rattle(UnitState<MAX_CLUSTER_ATOMS> &u, const ConstraintSet &cs, const DevInteg &p, SolverDiag &dg) {
  if (cs.n == 0) return;
  bool converged = false, stalled = false;
  float previous = 1e30f;
  for (int it = 0; it < p.max_iterations; ++it) {
    float worst = 0.f;
    for (int k = 0; k < cs.n; ++k) {
      const int a = cs.a[k], b = cs.b[k];
      const float bx = u.x[a][0] - u.x[b][0], by = u.x[a][1] - u.x[b][1], bz = u.x[a][2] - u.x[b][2];
      const float rx = u.v[a][0] - u.v[b][0], ry = u.v[a][1] - u.v[b][1], rz = u.v[a][2] - u.v[b][2];
      const float proj = bx * rx + by * ry + bz * rz;
      const float scaled = fabsf(proj) / (cs.d[k] * cs.d[k]);
      worst = fmaxf(worst, scaled);
      if (scaled <= p.tolerance) continue;
      const float ia = u.im[a], ib = u.im[b];
      const float den = (ia + ib) * (bx * bx + by * by + bz * bz);
      if (den < 1e-20f) continue;
      const float lam = -proj / den;
      u.v[a][0] += lam * ia * bx; u.v[a][1] += lam * ia * by; u.v[a][2] += lam * ia * bz;
      u.v[b][0] -= lam * ib * bx; u.v[b][1] -= lam * ib * by; u.v[b][2] -= lam * ib * bz;
    }
    if (worst <= p.tolerance) { converged = true; break; }
    if (it >= 2 && worst >= previous * 0.99f) { stalled = true; break; }
    previous = worst;
  }
  if (!converged && !stalled) dg.rattle_cap = 1;
}

// integrate.js:188-335: SHAKE along the pre-drift bond vectors, corrections accumulated so
// the velocity update v += correction / h never subtracts two box-spanning coordinates.
__device__ void shake(UnitState<MAX_CLUSTER_ATOMS> &u, const ConstraintSet &cs, const DevInteg &p, SolverDiag &dg) {
  if (cs.n == 0) return;
  for (int k = 0; k < u.n; ++k) u.corr[k][0] = u.corr[k][1] = u.corr[k][2] = 0.f;
  bool converged = false, stalled = false;
  float previous = 1e30f, achieved = 0.f;
  int iterations = 0;
  for (int it = 0; it < p.max_iterations; ++it) {
    float worst = 0.f;
    for (int k = 0; k < cs.n; ++k) {
      const int a = cs.a[k], b = cs.b[k];
      const float dx = u.x[a][0] - u.x[b][0], dy = u.x[a][1] - u.x[b][1], dz = u.x[a][2] - u.x[b][2];
      const float rest2 = cs.d[k] * cs.d[k];
      const float err = dx * dx + dy * dy + dz * dz - rest2;
      const float rel = fabsf(err) / rest2;
      worst = fmaxf(worst, rel);
      if (rel <= p.tolerance) continue;
      const float ox = u.ref[a][0] - u.ref[b][0], oy = u.ref[a][1] - u.ref[b][1], oz = u.ref[a][2] - u.ref[b][2];
      const float proj = dx * ox + dy * oy + dz * oz;
      const float ia = u.im[a], ib = u.im[b];
      const float den = 2.0f * (ia + ib) * proj;
      if (fabsf(den) < 1e-20f) continue;
      const float lam = -err / den;
      const float sax = lam * ia * ox, say = lam * ia * oy, saz = lam * ia * oz;
      const float sbx = lam * ib * ox, sby = lam * ib * oy, sbz = lam * ib * oz;
      u.x[a][0] += sax; u.x[a][1] += say; u.x[a][2] += saz;
      u.x[b][0] -= sbx; u.x[b][1] -= sby; u.x[b][2] -= sbz;
      u.corr[a][0] += sax; u.corr[a][1] += say; u.corr[a][2] += saz;
      u.corr[b][0] -= sbx; u.corr[b][1] -= sby; u.corr[b][2] -= sbz;
    }
    iterations = it + 1;
    achieved = worst;
    if (worst <= p.tolerance) { converged = true; break; }
    if (it >= 2 && worst >= previous * 0.99f) { stalled = true; break; }
    previous = worst;
  }
  const float inv_h = 1.0f / p.half_step;
  for (int k = 0; k < u.n; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) u.v[k][c] = fmaf(u.corr[k][c], inv_h, u.v[k][c]);
  dg.max_iterations = max(dg.max_iterations, iterations);
  if (!converged && !stalled) dg.shake_cap = 1;
  dg.stalled_residual = fmaxf(dg.stalled_residual, achieved);
}

template <int CAP>
__device__ __forceinline__ void drift(UnitState<CAP> &u, float h) {
#pragma unroll
  for (int k = 0; k < CAP; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (k >= u.n) continue;
      u.ref[k][c] = u.x[k][c];
      u.x[k][c] = fmaf(h, u.v[k][c], u.x[k][c]);
    }
}

template <int CAP>
__device__ __forceinline__ void thermostat(UnitState<CAP> &u, const DevInteg &p, uint32_t step,
                                           const float *__restrict__ noise, int local_base) {
#pragma unroll
  for (int k = 0; k < CAP; ++k) {
    if (k >= u.n || u.im[k] <= 0.f) continue;
    float3 g;
    if (p.supplied_noise) {
      const float *nz = noise + 3 * (long long)u.atom[k];
      g = make_float3(nz[0], nz[1], nz[2]);
    } else {
      g = rng_gaussian3(p.seed, (uint32_t)(u.atom[k] - local_base), step);
    }
    const float amp = p.noise_scale * sqrtf(p.kT * u.im[k]);
    u.v[k][0] = fmaf(p.decay, u.v[k][0], amp * g.x);
    u.v[k][1] = fmaf(p.decay, u.v[k][1], amp * g.y);
    u.v[k][2] = fmaf(p.decay, u.v[k][2], amp * g.z);
  }
}

// SETTLE (Miyamoto & Kollman 1992) for a rigid 3-site water: atom 0 the heavy apex,
// atoms 1 and 2 the light pair. Positions: the closed-form solution that restores the
// triangle from the pre-drift one (reference `ref`) by a rigid motion conserving linear
// and angular momentum; velocities (the RATTLE analogue): the 3x3 linear system for the
// three bond-direction impulses, solved exactly.
__device__ void settle_positions(UnitState<3> &u, const DevSettle &w, float inv_h) {
  const float mO = w.m_o, mH = w.m_h;
  const float wt = mO + 2.f * mH;
  const float ra = w.ra, rb = w.rb, rc = w.rc;  // geometry constants
  // Everything below is relative to the old apex position o: the new positions are within
  // a drift of it, so x - o is exact and the centre of mass, the frame and the rebuilt
  // triangle are all formed from numbers of ~0.1 nm. Formed from absolute coordinates
  // (several nm) instead, the f32 rounding of the centre of mass and the frame feeds back
  // through the velocity correction into a kinetic energy that grows exponentially.
  float o[3], xl[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    o[c] = u.ref[0][c];
#pragma unroll
    for (int k = 0; k < 3; ++k) xl[k][c] = u.x[k][c] - o[c];
  }
  float com[3], b0[3], c0[3], a1[3], b1[3], c1[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    b0[c] = u.ref[1][c] - o[c];
    c0[c] = u.ref[2][c] - o[c];
    com[c] = (mO * xl[0][c] + mH * (xl[1][c] + xl[2][c])) / wt;
    a1[c] = xl[0][c] - com[c];
    b1[c] = xl[1][c] - com[c];
    c1[c] = xl[2][c] - com[c];
  }
  // frame: Z along the normal of the old plane, X in the new apex direction
  float n0[3] = {b0[1] * c0[2] - b0[2] * c0[1], b0[2] * c0[0] - b0[0] * c0[2], b0[0] * c0[1] - b0[1] * c0[0]};
  float ax[3] = {a1[1] * n0[2] - a1[2] * n0[1], a1[2] * n0[0] - a1[0] * n0[2], a1[0] * n0[1] - a1[1] * n0[0]};
  float ay[3] = {n0[1] * ax[2] - n0[2] * ax[1], n0[2] * ax[0] - n0[0] * ax[2], n0[0] * ax[1] - n0[1] * ax[0]};
  const float nz = rsqrt_refined(n0[0] * n0[0] + n0[1] * n0[1] + n0[2] * n0[2]);
  const float nx = rsqrt_refined(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]);
  const float ny = rsqrt_refined(ay[0] * ay[0] + ay[1] * ay[1] + ay[2] * ay[2]);
#pragma unroll
  for (int c = 0; c < 3; ++c) { n0[c] *= nz; ax[c] *= nx; ay[c] *= ny; }
  auto proj = [&](const float *v, const float *e) { return v[0] * e[0] + v[1] * e[1] + v[2] * e[2]; };
  const float b0x = proj(b0, ax), b0y = proj(b0, ay);
  const float c0x = proj(c0, ax), c0y = proj(c0, ay);
  const float a1z = proj(a1, n0), b1x = proj(b1, ax), b1y = proj(b1, ay), b1z = proj(b1, n0);
  const float c1x = proj(c1, ax), c1y = proj(c1, ay), c1z = proj(c1, n0);
  float sinphi = a1z / ra;
  sinphi = fminf(1.f, fmaxf(-1.f, sinphi));
  const float cosphi = sqrtf(fmaxf(0.f, 1.f - sinphi * sinphi));
  float sinpsi = (b1z - c1z) / (2.f * rc * cosphi);
  sinpsi = fminf(1.f, fmaxf(-1.f, sinpsi));
  const float cospsi = sqrtf(fmaxf(0.f, 1.f - sinpsi * sinpsi));
  const float ya2 = ra * cosphi;
  const float xb2 = -rc * cospsi;
  const float t1 = -rb * cosphi;
  const float t2 = rc * sinpsi * sinphi;
  const float yb2 = t1 - t2, yc2 = t1 + t2;
  const float alpha_ = xb2 * (b0x - c0x) + b0y * yb2 + c0y * yc2;
  const float beta_ = xb2 * (c0y - b0y) + b0x * yb2 + c0x * yc2;
  const float gamma_ = b0x * b1y - b1x * b0y + c0x * c1y - c1x * c0y;
  const float a2b2 = alpha_ * alpha_ + beta_ * beta_;
  const float sintheta = (alpha_ * gamma_ - beta_ * sqrtf(fmaxf(0.f, a2b2 - gamma_ * gamma_))) / a2b2;
  const float costheta = sqrtf(fmaxf(0.f, 1.f - sintheta * sintheta));
  const float a3x = -ya2 * sintheta, a3y = ya2 * costheta, a3z = a1z;
  const float b3x = xb2 * costheta - yb2 * sintheta, b3y = xb2 * sintheta + yb2 * costheta, b3z = b1z;
  const float c3x = -xb2 * costheta - yc2 * sintheta, c3y = -xb2 * sintheta + yc2 * costheta, c3z = c1z;
  float na[3], nb[3], nc[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    na[c] = com[c] + a3x * ax[c] + a3y * ay[c] + a3z * n0[c];
    nb[c] = com[c] + b3x * ax[c] + b3y * ay[c] + b3z * n0[c];
    nc[c] = com[c] + c3x * ax[c] + c3y * ay[c] + c3z * n0[c];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float da = na[c] - xl[0][c], db = nb[c] - xl[1][c], dc = nc[c] - xl[2][c];
    u.x[0][c] = o[c] + na[c];
    u.x[1][c] = o[c] + nb[c];
    u.x[2][c] = o[c] + nc[c];
    u.v[0][c] = fmaf(da, inv_h, u.v[0][c]);
    u.v[1][c] = fmaf(db, inv_h, u.v[1][c]);
    u.v[2][c] = fmaf(dc, inv_h, u.v[2][c]);
  }
}

// Remove the bond-direction relative velocity of the three water bonds exactly: solve
// A tau = -(e_ij . v_ij) for the impulses along the unit bond vectors.
__device__ void settle_velocities(UnitState<3> &u, const DevSettle &w) {
  const int P[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  float e[3][3], rhs[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int a = P[k][0], b = P[k][1];
    float d[3] = {u.x[a][0] - u.x[b][0], u.x[a][1] - u.x[b][1], u.x[a][2] - u.x[b][2]};
    const float inv = rsqrt_refined(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
#pragma unroll
    for (int c = 0; c < 3; ++c) e[k][c] = d[c] * inv;
    rhs[k] = -(e[k][0] * (u.v[a][0] - u.v[b][0]) + e[k][1] * (u.v[a][1] - u.v[b][1]) +
               e[k][2] * (u.v[a][2] - u.v[b][2]));
  }
  const float im0 = 1.0f / w.m_o, imh = 1.0f / w.m_h;
  const float ima[3] = {im0, im0, imh}, imb[3] = {imh, imh, imh};
  // A[k][l] = e_k . (dv_k/dtau_l): tau_l changes v_a(l) by +im*e_l and v_b(l) by -im*e_l
  float A[3][3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      const int ak = P[k][0], bk = P[k][1], al = P[l][0], bl = P[l][1];
      const float iml_a = (al == 0) ? im0 : imh, iml_b = imh;
      float coef = 0.f;  // d(v_ak - v_bk)/dtau_l along e_l
      if (ak == al) coef += iml_a;
      if (ak == bl) coef -= iml_b;
      if (bk == al) coef -= iml_a;
      if (bk == bl) coef += iml_b;
      A[k][l] = coef * (e[k][0] * e[l][0] + e[k][1] * e[l][1] + e[k][2] * e[l][2]);
    }
  (void)ima; (void)imb;
  const float det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                    A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                    A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
  if (fabsf(det) < 1e-30f) return;
  const float id = 1.0f / det;
  float tau[3];
  tau[0] = id * (rhs[0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (rhs[1] * A[2][2] - A[1][2] * rhs[2]) +
                 A[0][2] * (rhs[1] * A[2][1] - A[1][1] * rhs[2]));
  tau[1] = id * (A[0][0] * (rhs[1] * A[2][2] - A[1][2] * rhs[2]) - rhs[0] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                 A[0][2] * (A[1][0] * rhs[2] - rhs[1] * A[2][0]));
  tau[2] = id * (A[0][0] * (A[1][1] * rhs[2] - rhs[1] * A[2][1]) - A[0][1] * (A[1][0] * rhs[2] - rhs[1] * A[2][0]) +
                 rhs[0] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]));
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    const int a = P[l][0], b = P[l][1];
    const float ia = (a == 0) ? im0 : imh, ib = imh;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      u.v[a][c] += tau[l] * ia * e[l][c];
      u.v[b][c] -= tau[l] * ib * e[l][c];
    }
  }
}

struct UnitResult {
  int sidx;
  unsigned worst_bits;
  SolverDiag dg;
};

// Apply this launch's part of the step to one unit. KIND: 0 free atom, 1 SHAKE cluster,
// 2 SETTLE water; CAP is the unit's static capacity.
template <int MODE, int KIND, int CAP>
__device__ __forceinline__ void process_unit(const IntegrateArgs &g, int index, UnitResult &res) {
  UnitState<CAP> u;
  ConstraintSet cs;
  cs.n = 0;
  int settle_index = -1;
  if (KIND == 0) {
    u.n = 1;
    u.atom[0] = g.free_atoms[index];
  } else if (KIND == 1) {
    const int ab = g.cl_atom_start[index], ae = g.cl_atom_start[index + 1];
    u.n = ae - ab;
    for (int k = 0; k < u.n; ++k) u.atom[k] = g.cl_atoms[ab + k];
    const int cb = g.cl_con_start[index], ce = g.cl_con_start[index + 1];
    cs.n = ce - cb;
    for (int k = 0; k < cs.n; ++k) {
      const int2 pr = g.cl_con_pair[cb + k];
      cs.a[k] = pr.x;
      cs.b[k] = pr.y;
      cs.d[k] = g.cl_con_dist[cb + k];
    }
  } else {
    settle_index = index;
    const int3 w = g.settle_atoms[index];
    u.n = 3;
    u.atom[0] = w.x;
    u.atom[1] = w.y;
    u.atom[2] = w.z;
  }
  const int sidx = g.sys_of_atom[u.atom[0]];
  res.sidx = sidx;
  const DevInteg p = g.integ[sidx];
  SolverDiag dg = {0, 0, 0, 0.f};
  if (MODE & INT_CONSTRAIN) {
    // minimiser: project the displaced positions back onto the constraints along the
    // pre-displacement geometry (encodeConstrainPositions, integrate.js:672-688)
    if (KIND == 0) return;
#pragma unroll
    for (int k = 0; k < CAP; ++k) {
      if (k >= u.n) continue;
      const int a = u.atom[k];
      const float4 x = g.posq[a], r = g.saved_posq[a];
      u.x[k][0] = x.x; u.x[k][1] = x.y; u.x[k][2] = x.z;
      u.ref[k][0] = r.x; u.ref[k][1] = r.y; u.ref[k][2] = r.z;
      u.v[k][0] = u.v[k][1] = u.v[k][2] = 0.f;
      u.im[k] = g.vel[a].w;
    }
    if constexpr (KIND == 1) shake(u, cs, p, dg);
    if constexpr (KIND == 2) settle_positions(u, g.settle_param[settle_index], 1.0f);
#pragma unroll
    for (int k = 0; k < CAP; ++k) {
      if (k >= u.n) continue;
      const float4 old = g.posq[u.atom[k]];
      g.posq[u.atom[k]] = make_float4(u.x[k][0], u.x[k][1], u.x[k][2], old.w);
    }
    return;
  }
#pragma unroll
  for (int k = 0; k < CAP; ++k) {
    if (k >= u.n) continue;
    const int a = u.atom[k];
    const float4 x = g.posq[a];
    const float4 v = g.vel[a];
    u.x[k][0] = x.x; u.x[k][1] = x.y; u.x[k][2] = x.z;
    u.v[k][0] = v.x; u.v[k][1] = v.y; u.v[k][2] = v.z;
    u.im[k] = v.w;  // inverse mass (0 for a massless site)
    u.f[k][0] = from_fixed(g.force[a]);
    u.f[k][1] = from_fixed(g.force[g.n_atoms + a]);
    u.f[k][2] = from_fixed(g.force[2 * (long long)g.n_atoms + a]);
  }
  const float h = p.half_step;
  const int local_base = g.sys_atom_start[sidx];
  const uint32_t step = (uint32_t)(g.step_base[sidx] + g.step_offset);
  DevSettle sw;
  if constexpr (KIND == 2) sw = g.settle_param[settle_index];
  auto velocity_constraint = [&]() {
    if constexpr (KIND == 1) rattle(u, cs, p, dg);
    if constexpr (KIND == 2) settle_velocities(u, sw);
  };
  auto position_constraint = [&]() {
    if constexpr (KIND == 1) shake(u, cs, p, dg);
    if constexpr (KIND == 2) settle_positions(u, sw, 1.0f / h);
  };
  if (MODE & INT_CLOSE) {
    kick(u, h);
    velocity_constraint();
  }
  if (MODE & INT_CLOSE_KINETIC) {
#pragma unroll
    for (int k = 0; k < CAP; ++k) {
      if (k >= u.n) continue;
      const float m = u.im[k] > 0.f ? 1.0f / u.im[k] : 0.f;
      g.ke_post[u.atom[k]] = 0.5 * (double)m *
          ((double)u.v[k][0] * u.v[k][0] + (double)u.v[k][1] * u.v[k][1] + (double)u.v[k][2] * u.v[k][2]);
    }
  }
  if (MODE & INT_OPEN) {
    kick(u, h);
    velocity_constraint();
    drift(u, h);
    position_constraint();
    thermostat(u, p, step, g.noise, local_base);
    velocity_constraint();
    drift(u, h);
    position_constraint();
  }
  if (MODE & INT_OPEN_KINETIC) {
#pragma unroll
    for (int k = 0; k < CAP; ++k) {
      if (k >= u.n) continue;
      const float m = u.im[k] > 0.f ? 1.0f / u.im[k] : 0.f;
      g.ke_early[u.atom[k]] = 0.5 * (double)m *
          ((double)u.v[k][0] * u.v[k][0] + (double)u.v[k][1] * u.v[k][1] + (double)u.v[k][2] * u.v[k][2]);
    }
  }
  unsigned worst = 0u;
#pragma unroll
  for (int k = 0; k < CAP; ++k) {
    if (k >= u.n) continue;
    const int a = u.atom[k];
    if (MODE & INT_OPEN) {
      const float4 old = g.posq[a];
      g.posq[a] = make_float4(u.x[k][0], u.x[k][1], u.x[k][2], old.w);
      // keep the cell-ordered copy current: same wrap shift as at the last rebuild
      const float4 w = g.wrap[a];
      g.spos[g.rank[a]] = make_float4(u.x[k][0] - w.x, u.x[k][1] - w.y, u.x[k][2] - w.z, old.w);
      const float4 o = g.origin[a];
      const float dx = u.x[k][0] - o.x, dy = u.x[k][1] - o.y, dz = u.x[k][2] - o.z;
      worst = max(worst, __float_as_uint(dx * dx + dy * dy + dz * dz));
    }
    g.vel[a] = make_float4(u.v[k][0], u.v[k][1], u.v[k][2], u.im[k]);
  }
  res.worst_bits = worst;
  res.dg = dg;
}

template <int MODE>
__global__ void __launch_bounds__(64) k_integrate(IntegrateArgs g) {
  chain_begin();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool active = t < g.n_units;
  UnitResult res = {0, 0u, {0, 0, 0, 0.f}};
  if (active) {
    if (t < g.n_free) process_unit<MODE, 0, 1>(g, t, res);
    else if (t < g.n_free + g.n_clusters) process_unit<MODE, 1, MAX_CLUSTER_ATOMS>(g, t - g.n_free, res);
    else process_unit<MODE, 2, 3>(g, t - g.n_free - g.n_clusters, res);
  }
  if (MODE & INT_CONSTRAIN) return;  // every thread of the launch leaves here together
  // --- skin displacement and solver diagnostics, aggregated per warp when it is one system
  const int sidx = res.sidx;
  unsigned worst_bits = res.worst_bits;
  const int sref = __shfl_sync(0xffffffffu, sidx, 0);
  const bool uniform = __all_sync(0xffffffffu, !active || sidx == sref);
  int diag_iter = res.dg.max_iterations, diag_shake = res.dg.shake_cap, diag_rattle = res.dg.rattle_cap;
  unsigned diag_res = __float_as_uint(res.dg.stalled_residual);
  if (uniform) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      worst_bits = max(worst_bits, __shfl_xor_sync(0xffffffffu, worst_bits, o));
      diag_iter = max(diag_iter, __shfl_xor_sync(0xffffffffu, diag_iter, o));
      diag_shake |= __shfl_xor_sync(0xffffffffu, diag_shake, o);
      diag_rattle |= __shfl_xor_sync(0xffffffffu, diag_rattle, o);
      diag_res = max(diag_res, __shfl_xor_sync(0xffffffffu, diag_res, o));
    }
  }
  if (active && (!uniform || lane == 0)) {
    const int s2 = uniform ? sref : sidx;
    if ((MODE & INT_OPEN) && worst_bits) {
      atomicMax(&g.disp[s2], worst_bits);
      atomicMax(&g.disp[g.n_systems + s2], worst_bits);
    }
    if (diag_iter) atomicMax(&g.diag[4 * s2], diag_iter);
    if (diag_shake) atomicMax(&g.diag[4 * s2 + 1], 1);
    if (diag_rattle) atomicMax(&g.diag[4 * s2 + 2], 1);
    if (diag_res) atomicMax((unsigned *)&g.diag[4 * s2 + 3], diag_res);
  }
}

void launch_integrate(const IntegrateArgs &a, int mode, cudaStream_t stream) {
  if (a.n_units == 0) return;
  const int tb = 64, blocks = (a.n_units + tb - 1) / tb;
  void (*kernel)(IntegrateArgs);
  switch (mode) {
    case INT_OPEN: kernel = k_integrate<INT_OPEN>; break;
    case INT_OPEN | INT_OPEN_KINETIC: kernel = k_integrate<INT_OPEN | INT_OPEN_KINETIC>; break;
    case INT_CLOSE | INT_OPEN: kernel = k_integrate<INT_CLOSE | INT_OPEN>; break;
    case INT_CLOSE | INT_OPEN | INT_OPEN_KINETIC: kernel = k_integrate<INT_CLOSE | INT_OPEN | INT_OPEN_KINETIC>; break;
    case INT_CLOSE: kernel = k_integrate<INT_CLOSE>; break;
    case INT_CLOSE | INT_CLOSE_KINETIC: kernel = k_integrate<INT_CLOSE | INT_CLOSE_KINETIC>; break;
    case INT_CONSTRAIN: kernel = k_integrate<INT_CONSTRAIN>; break;
    default: kernel = k_integrate<INT_CLOSE_KINETIC>; break;
  }
  launch_chained(kernel, blocks, tb, 0, stream, a);
}

// The thermostat's draws for atoms [atom0, atom0 + count) at `step`, through the same device
// functions k_integrate calls (random.js:59 uniformAt for c = 0..3, and the Box-Muller triple
// built from them): four uniforms and three normals per atom.
__global__ void k_draws(uint32_t seed, uint32_t atom0, int count, uint32_t step, float *__restrict__ uniforms,
                        float *__restrict__ normals) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const uint32_t atom = atom0 + (uint32_t)k;
#pragma unroll
  for (uint32_t c = 0; c < 4; ++c) uniforms[4 * (long long)k + c] = rng_uniform(seed, atom, step, c);
  const float3 g = rng_gaussian3(seed, atom, step);
  normals[3 * (long long)k] = g.x;
  normals[3 * (long long)k + 1] = g.y;
  normals[3 * (long long)k + 2] = g.z;
}

void launch_draws(uint32_t seed, uint32_t atom0, int count, uint32_t step, float *uniforms, float *normals,
                  cudaStream_t stream) {
  if (count <= 0) return;
  k_draws<<<(count + 127) / 128, 128, 0, stream>>>(seed, atom0, count, step, uniforms, normals);
}

}  // namespace rmd
