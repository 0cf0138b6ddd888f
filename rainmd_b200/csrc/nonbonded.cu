// Direct-space Lennard-Jones + Ewald-screened Coulomb over the neighbour list, fused with
// the exception pass (1-4 pairs and the erf correction of every excluded pair).
//
// Physics as RainMD's nonbonded.js:30-200 / cpu/forces/nonbonded.js:24-162: a full
// (both-direction) list, so each atom's force is a gather and needs no atomics; energies
// are halved because each pair is seen from both atoms; the screened-Coulomb force carries
// the Gaussian term 2a exp(-a^2 r^2)/sqrt(pi); exceptions have no cutoff and the erf
// correction uses the atoms' full charges.
//
// B200 shape: LANES lanes per atom (32 = one warp; 16 or 8 = 2 or 4 atoms per warp, chosen
// by the autotuner). Lanes stride the atom's neighbour row, so the row read is coalesced
// and the j positions (float4 x,y,z,q) are gathered through L1. exp(-z^2) is computed
// once per pair and shared by erfc and the Gaussian. Per-lane partial forces are converted
// to 64-bit fixed point and reduced with integer shuffles, so the sum is exact and
// order-independent; lane 0 stores the atom's force (this kernel is the first writer of
// the force array in every evaluation). Energies, and the pair virial sum F.r over the
// list pairs (the barostat surrogate's input), are only computed in the ENERGY variant.
#include "common.cuh"
#include "kernels.h"

namespace rmd {

template <int LANES>
__device__ __forceinline__ long long group_sum(long long v) {
#pragma unroll
  for (int o = LANES / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <int LANES>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = LANES / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// PAIR_FIXED (the precision form): each pair force (and, in the ENERGY variant, each pair
// energy) is quantised to 64-bit fixed point (2^32 per unit) before it is summed, so the
// atom's sums are exact integers and do not depend on the order of its neighbour row or on
// the lanes per atom (a rebuilt list, a resumed run, a different batch or launch shape all
// give the same bits). Without it (the plain form) lanes sum in f32 and convert once.
template <bool ENERGY, int LANES, bool PAIR_FIXED>
__global__ void __launch_bounds__(128) k_nonbonded(
    const float4 *__restrict__ posq, const float4 *__restrict__ spos, const int *__restrict__ sorted_orig,
    const int *__restrict__ sorted_type, const int *__restrict__ sys_of_atom, const DevSys *__restrict__ sys,
    const float2 *__restrict__ lj, const int *__restrict__ nbr, const int *__restrict__ nbr_count,
    const int *__restrict__ exc_start, const int *__restrict__ exc_partner,
    const float4 *__restrict__ exc_param, unsigned long long *__restrict__ force,
    double *__restrict__ e_lj, double *__restrict__ e_coul, double *__restrict__ e_vir, int n_atoms,
    int lj_entries) {
  // the type tables in shared memory when they fit (the launch sizes the buffer), so the
  // pair's LJ parameters are one shared-memory read after its partner's type
  extern __shared__ float2 lj_shared[];
  const bool lj_in_smem = lj_entries > 0;
  for (int k = threadIdx.x; k < lj_entries; k += blockDim.x) lj_shared[k] = lj[k];
  if (lj_in_smem) __syncthreads();
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  // A warp may hold a group past the last atom (LANES < 32): it works on a clamped atom
  // with an empty row and stores nothing, so every lane reaches the shuffles.
  const bool valid = gid / LANES < n_atoms;
  if (!valid && LANES == 32) return;
  const int si = valid ? gid / LANES : n_atoms - 1;  // atoms are visited in cell order
  const int lane = gid % LANES;
  const int i = sorted_orig[si];
  const DevSys &s = sys[sys_of_atom[i]];
  const float4 pw = spos[si];
  const int ti = sorted_type[si];
  const float2 *ljrow = (lj_in_smem ? lj_shared : lj) + s.lj_base + ti * s.type_count;
  const float alpha = s.alpha;
  const float gauss_k = 2.0f * alpha * 0.5641895835477563f;  // 2a/sqrt(pi)
  const float cut2 = s.cutoff2;
  const int count = valid ? nbr_count[si] : 0;
  const int *row = nbr + s.nbr_base + (long long)(si - s.atom_start) * s.nbr_capacity;

  float fx = 0.f, fy = 0.f, fz = 0.f, elj = 0.f, ecoul = 0.f, evir = 0.f;
  long long qx = 0, qy = 0, qz = 0, qlj = 0, qcoul = 0, qvir = 0;
  // Software pipeline over the lane's entries: the row word two entries ahead and the
  // partner record (position, type, image shift) one entry ahead are in flight while this
  // entry's pair is computed, so the gathers' latency overlaps the arithmetic.
  int k = lane;
  unsigned e1 = 0, e2 = 0;
  float4 pj1 = make_float4(0.f, 0.f, 0.f, 0.f), S1 = pj1;
  int tj1 = 0;
  if (k < count) {
    e1 = (unsigned)__ldg(row + k);
    const int g = (int)(e1 & NBR_SLOT_MASK);
    pj1 = __ldg(spos + g);
    tj1 = __ldg(sorted_type + g);
    S1 = s.shift[e1 >> NBR_SLOT_BITS];  // the partner's image (code 0..26), fixed at the rebuild
  }
  if (k + LANES < count) e2 = (unsigned)__ldg(row + k + LANES);
  for (; k < count; k += LANES) {
    const float4 pj = pj1, S = S1;
    const int tj = tj1;
    if (k + LANES < count) {
      e1 = e2;
      const int g = (int)(e1 & NBR_SLOT_MASK);
      pj1 = __ldg(spos + g);
      tj1 = __ldg(sorted_type + g);
      S1 = s.shift[e1 >> NBR_SLOT_BITS];
      if (k + 2 * LANES < count) e2 = (unsigned)__ldg(row + k + 2 * LANES);
    }
    const float3 d = make_float3(pw.x - pj.x - S.x, pw.y - pj.y - S.y, pw.z - pj.z - S.z);
    const float r2 = fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z));
    if (r2 <= cut2) {
      const float inv_r = rsqrt_refined(r2);
      const float inv_r2 = inv_r * inv_r;
      const float inv_r6 = inv_r2 * inv_r2 * inv_r2;
      const float2 ab = ljrow[tj];
      const float a12 = ab.x * inv_r6 * inv_r6, b6 = ab.y * inv_r6;
      float scalar = (12.0f * a12 - 6.0f * b6) * inv_r2;
      const float qq = (float)ONE_4PI_EPS0 * (pw.w * pj.w);  // symmetric in i and j
      const float r = r2 * inv_r;
      float gauss;
      const float screened = erfc_and_gauss(alpha * r, gauss);
      scalar = fmaf(qq * fmaf(screened, inv_r, gauss_k * gauss), inv_r2, scalar);
      if (PAIR_FIXED) {
        qx += (long long)to_fixed(scalar * d.x);
        qy += (long long)to_fixed(scalar * d.y);
        qz += (long long)to_fixed(scalar * d.z);
      } else {
        fx = fmaf(scalar, d.x, fx);
        fy = fmaf(scalar, d.y, fy);
        fz = fmaf(scalar, d.z, fz);
      }
      if (ENERGY) {
        if (PAIR_FIXED) {
          qlj += (long long)to_fixed(a12 - b6);
          qcoul += (long long)to_fixed(qq * screened * inv_r);
          qvir += (long long)to_fixed(scalar * r2);
        } else {
          elj += a12 - b6;
          ecoul = fmaf(qq * screened, inv_r, ecoul);
          evir = fmaf(scalar, r2, evir);
        }
      }
    }
  }
  // Exceptions: 1-4 scaled LJ/Coulomb and -q_i q_j erf(a r)/r, no cutoff.
  const int eb = exc_start[i], ee = valid ? exc_start[i + 1] : eb;
  const float4 pi = posq[i];
  for (int e = eb + lane; e < ee; e += LANES) {
    float pair_lj = 0.f, pair_coul = 0.f;
    const int j = exc_partner[e];
    const float4 prm = exc_param[e];  // chargeProduct, ljA, ljB, fullProduct
    const float4 pj = posq[j];
    float3 d = min_image(make_float3(pi.x - pj.x, pi.y - pj.y, pi.z - pj.z), s);
    const float r2 = fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z));
    const float inv_r = rsqrt_refined(r2);
    const float inv_r2 = inv_r * inv_r, inv_r6 = inv_r2 * inv_r2 * inv_r2;
    float scalar = 0.f;
    if (prm.y != 0.f || prm.z != 0.f) {
      const float a12 = prm.y * inv_r6 * inv_r6, b6 = prm.z * inv_r6;
      scalar += (12.0f * a12 - 6.0f * b6) * inv_r2;
      if (ENERGY) pair_lj += a12 - b6;
    }
    if (prm.x != 0.f) {
      const float qq = (float)ONE_4PI_EPS0 * prm.x;
      scalar += qq * inv_r * inv_r2;
      if (ENERGY) pair_coul += qq * inv_r;
    }
    if (alpha > 0.f && prm.w != 0.f) {
      const float qq = (float)ONE_4PI_EPS0 * prm.w;
      float gauss;
      const float r = r2 * inv_r;
      const float unscreened = 1.0f - erfc_and_gauss(alpha * r, gauss);
      scalar -= qq * (unscreened * inv_r - gauss_k * gauss) * inv_r2;
      if (ENERGY) pair_coul -= qq * unscreened * inv_r;
    }
    if (ENERGY) {
      if (PAIR_FIXED) {
        qlj += (long long)to_fixed(pair_lj);
        qcoul += (long long)to_fixed(pair_coul);
        qvir += (long long)to_fixed(scalar * r2);
      } else {
        elj += pair_lj;
        ecoul += pair_coul;
        evir = fmaf(scalar, r2, evir);
      }
    }
    if (PAIR_FIXED) {
      qx += (long long)to_fixed(scalar * d.x);
      qy += (long long)to_fixed(scalar * d.y);
      qz += (long long)to_fixed(scalar * d.z);
    } else {
      fx = fmaf(scalar, d.x, fx);
      fy = fmaf(scalar, d.y, fy);
      fz = fmaf(scalar, d.z, fz);
    }
  }
  if (!PAIR_FIXED) {
    qx = (long long)to_fixed(fx);
    qy = (long long)to_fixed(fy);
    qz = (long long)to_fixed(fz);
  }
  const long long gx = group_sum<LANES>(qx);
  const long long gy = group_sum<LANES>(qy);
  const long long gz = group_sum<LANES>(qz);
  double dl = 0, dc = 0, dv = 0;
  if (ENERGY) {
    if (PAIR_FIXED) {  // exact integer sums: the energy, like the force, is order-independent
      dl = (double)group_sum<LANES>(qlj) / FORCE_SCALE;
      dc = (double)group_sum<LANES>(qcoul) / FORCE_SCALE;
      dv = (double)group_sum<LANES>(qvir) / FORCE_SCALE;
    } else {
      dl = group_sum<LANES>((double)elj);
      dc = group_sum<LANES>((double)ecoul);
      dv = group_sum<LANES>((double)evir);
    }
  }
  if (lane == 0 && valid) {
    force[i] = (unsigned long long)gx;
    force[n_atoms + i] = (unsigned long long)gy;
    force[2 * (long long)n_atoms + i] = (unsigned long long)gz;
    if (ENERGY) {
      e_lj[i] = 0.5 * dl;
      e_coul[i] = 0.5 * dc;
      e_vir[i] = 0.5 * dv;
    }
  }
}

// ------------------------------------------------------------------ group-pair kernel
// The same pair physics over the group-pair rows (lists.cu k_group_rows). A row's entries are
// dealt to the lanes of `split` warps, one partner a lane. A lane first tests its partner's
// squared distances to the group's GROUP_ATOMS atoms (their records are in the warp's shared
// memory); the entries with an unmasked atom within the cutoff queue in a per-warp ring, and
// each batch of 32 queued entries is evaluated one entry a lane, the partner against the four
// atoms in turn, so a batch evaluates 128 pairs of which none belongs to an entry beyond the
// cutoff of all four (about half the rows' entries). Each pair is evaluated once, from the
// group that lists it. Its force is quantised to 64-bit fixed point
// (as the atom-row kernel's precision form does) and added to two integer sums in the lane's
// registers: the group atom's (one per group atom, reduced over the warp once, at the end of
// the row) and the partner's (its negation, added to the force array with one 64-bit atomic per
// component at the end of the lane's entry). Because the pair force is computed from the same
// f32 operands in the same order as the atom-row kernel computes it from either atom (the
// charge product is symmetric, the image shifts of opposite codes are exact negatives, and
// rounding to nearest is odd), every atom's force is the same sum of the same integers as
// there, bit for bit. Energies (ENERGY) are accumulated the same way into per-atom integer sums
// that hold each pair's full energy for both of its atoms, then halved, which is the atom-row
// kernel's per-atom value exactly. The force array (and, for ENERGY, the energy sums) must be
// zero when the kernel starts. The exceptions of each group atom are evaluated by 8 lanes of the
// row's first warp, as in the atom-row kernel.

// Warp sum of 16 64-bit values (v[0..15]): returns in lane l the sum over all 32 lanes of
// v[(l >> 1) & 15] (the lane pair 2k, 2k + 1 holds value k). Five exchange levels that halve the
// values each lane carries, 16 + 8 + 4 + 2 + 1 shuffles of 64-bit words instead of 80.
__device__ __forceinline__ long long warp_sum_sixteen(long long (&v)[16], int lane) {
#pragma unroll
  for (int level = 0, width = 16; level < 4; ++level, width >>= 1) {
    const int bit = 4 - level;  // exchange across lane bit 4, then 3, 2, 1
    const bool hi = (lane >> bit) & 1;
#pragma unroll
    for (int k = 0; k < width / 2; ++k) {
      const long long send = hi ? v[k] : v[k + width / 2];
      const long long keep = hi ? v[k + width / 2] : v[k];
      v[k] = keep + __shfl_xor_sync(0xffffffffu, send, 1 << bit);
    }
  }
  return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}

// One row entry against the group's GROUP_ATOMS atoms: the four pairs are evaluated without
// branches (a pair that is masked or beyond the cutoff is evaluated at r = 1 nm and contributes
// zero), so their chains can interleave. Each pair force is quantised (the scale folded into
// the scalar factor: a power of two, so the product rounds exactly as the scaled force does)
// and added to the group atom's integer sums in `acc`; the partner gets the negated sum with
// one 64-bit atomic per component (energies as they are).
template <bool ENERGY>
__device__ __forceinline__ void group_pair_entry(const unsigned e, const float4 pj, const int2 info_j,
                                                 const float4 *__restrict__ gpos, const int *__restrict__ glj,
                                                 const float2 *__restrict__ ljtab, const DevSys &s, float alpha,
                                                 float gauss_k, float cut2, long long (&acc)[GROUP_ATOMS][ENERGY ? 6 : 3],
                                                 unsigned long long *__restrict__ force,
                                                 unsigned long long *__restrict__ e_acc, int n_atoms) {
  const float4 S = s.shift[(e >> GROUP_CODE_SHIFT) & 31u];
  long long jx = 0, jy = 0, jz = 0, jl = 0, jc = 0, jv = 0;
#pragma unroll
  for (int a = 0; a < GROUP_ATOMS; ++a) {
    const float4 pw = gpos[a];
    const float3 d = make_float3(pw.x - pj.x - S.x, pw.y - pj.y - S.y, pw.z - pj.z - S.z);
    const float r2d = fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z));
    const bool in = !((e >> (GROUP_MASK_SHIFT + a)) & 1u) && r2d <= cut2;
    const float r2 = in ? r2d : 1.0f;
    const float inv_r = rsqrt_refined(r2);
    const float inv_r2 = inv_r * inv_r;
    const float inv_r6 = inv_r2 * inv_r2 * inv_r2;
    const float2 ab = ljtab[glj[a] + info_j.x];
    const float a12 = ab.x * inv_r6 * inv_r6, b6 = ab.y * inv_r6;
    float scalar = (12.0f * a12 - 6.0f * b6) * inv_r2;
    const float qq = (float)ONE_4PI_EPS0 * (pw.w * pj.w);
    const float r = r2 * inv_r;
    float gauss;
    const float screened = erfc_and_gauss(alpha * r, gauss);
    scalar = fmaf(qq * fmaf(screened, inv_r, gauss_k * gauss), inv_r2, scalar);
    scalar = in ? scalar * FORCE_SCALE_F : 0.0f;
    const long long fx = __float2ll_rn(scalar * d.x);
    const long long fy = __float2ll_rn(scalar * d.y);
    const long long fz = __float2ll_rn(scalar * d.z);
    acc[a][0] += fx;
    acc[a][1] += fy;
    acc[a][2] += fz;
    jx += fx;
    jy += fy;
    jz += fz;
    if (ENERGY) {
      const long long el = in ? (long long)to_fixed(a12 - b6) : 0;
      const long long ec = in ? (long long)to_fixed(qq * screened * inv_r) : 0;
      const long long ev = __float2ll_rn(scalar * r2);
      acc[a][ENERGY ? 3 : 0] += el;
      acc[a][ENERGY ? 4 : 0] += ec;
      acc[a][ENERGY ? 5 : 0] += ev;
      jl += el;
      jc += ec;
      jv += ev;
    }
  }
  const int j = info_j.y;
  if (jx != 0) atomicAdd(force + j, (unsigned long long)(-jx));
  if (jy != 0) atomicAdd(force + n_atoms + j, (unsigned long long)(-jy));
  if (jz != 0) atomicAdd(force + 2 * (long long)n_atoms + j, (unsigned long long)(-jz));
  if (ENERGY) {
    if (jl != 0) atomicAdd(e_acc + j, (unsigned long long)jl);
    if (jc != 0) atomicAdd(e_acc + n_atoms + j, (unsigned long long)jc);
    if (jv != 0) atomicAdd(e_acc + 2 * (long long)n_atoms + j, (unsigned long long)jv);
  }
}

template <bool ENERGY>
__global__ void __launch_bounds__(128, ENERGY ? 4 : 5) k_group_pairs(
    const float4 *__restrict__ posq, const float4 *__restrict__ spos, const int2 *__restrict__ slot_info,
    const int *__restrict__ group_order, const int *__restrict__ group_sys, const DevSys *__restrict__ sys,
    const float2 *__restrict__ lj, const int *__restrict__ gnbr, const int *__restrict__ gnbr_count,
    const int *__restrict__ gfirst, const int *__restrict__ gsize, const int *__restrict__ exc_start,
    const int *__restrict__ exc_partner, const float4 *__restrict__ exc_param,
    unsigned long long *__restrict__ force, unsigned long long *__restrict__ e_acc, int n_atoms, int n_groups,
    int lj_entries, int split) {
  constexpr int G = GROUP_ATOMS;
  extern __shared__ float2 lj_shared[];
  const bool lj_in_smem = lj_entries > 0;
  for (int k = threadIdx.x; k < lj_entries; k += blockDim.x) lj_shared[k] = lj[k];
  if (lj_in_smem) __syncthreads();
  // `split` warps share a group's row, warp r taking the passes r, r + split, ...
  const int task = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int warp = task / split, part = task - warp * split;  // the group slot, this warp's share
  const int lane = threadIdx.x & 31;
  if (warp >= n_groups) return;
  // the group's records, loaded together before the first branch on them
  const int size = gsize[warp], sys_index = group_sys[warp], first = gfirst[warp], count = gnbr_count[warp];
  if (size == 0) return;  // an unused slot (the whole warp leaves)
  const DevSys &s = sys[sys_index];
  const float2 *ljtab = (lj_in_smem ? lj_shared : lj) + s.lj_base;
  // the group's atoms, the same for every lane (an absent atom is masked by every entry): their
  // records in this warp's shared memory, their original indices in registers
  __shared__ float4 group_pos[4][G];
  __shared__ int group_lj[4][G];
  const int wib = threadIdx.x >> 5;
  int ia[G];
#pragma unroll
  for (int a = 0; a < G; ++a) {
    const int si = group_order[first + (a < size ? a : 0)];
    ia[a] = slot_info[si].y;
    if (lane == a) {
      group_pos[wib][a] = spos[si];
      group_lj[wib][a] = slot_info[si].x * s.type_count;
    }
  }
  __syncwarp();
  const float alpha = s.alpha;
  const float gauss_k = 2.0f * alpha * 0.5641895835477563f;  // 2a/sqrt(pi)
  const float cut2 = s.cutoff2;
  const int *row = gnbr + s.gnbr_base + (long long)(warp - s.group_base) * s.nbr_capacity;
  // per group atom: force x, y, z (and energies lj, coulomb, virial) in fixed point
  long long acc[G][ENERGY ? 6 : 3];
#pragma unroll
  for (int a = 0; a < G; ++a)
#pragma unroll
    for (int c = 0; c < (ENERGY ? 6 : 3); ++c) acc[a][c] = 0;
  const int stride = 32 * split;
  int k = 32 * part + lane;
  // Each pass first tests its 32 entries with the four squared distances alone; an entry with
  // some unmasked group atom within the cutoff joins this warp's ring in shared memory (about
  // half of them: the rows hold every partner within the list cutoff of the group's box), and
  // whenever 32 are queued the warp evaluates them, one entry a lane, so the full pair
  // arithmetic runs on entries that contribute. The queued entries keep their records, so
  // the evaluation reads them from shared memory.
  __shared__ unsigned ring_e[4][64];
  __shared__ float4 ring_p[4][64];
  __shared__ int2 ring_i[4][64];
  int head = 0, queued = 0;
  // software pipeline, two deep: the entries of the pass after next and the partner records of
  // the next pass are loaded while this pass's entries are tested, so no load waits on one
  // issued in the same pass
  constexpr unsigned NO_ENTRY = 0xFu << GROUP_MASK_SHIFT;
  unsigned e1 = k < count ? (unsigned)__ldg(row + k) : NO_ENTRY;
  unsigned e2 = k + stride < count ? (unsigned)__ldg(row + k + stride) : NO_ENTRY;
  float4 pj1 = __ldg(spos + (e1 & GROUP_SLOT_MASK));
  int2 info1 = __ldg(slot_info + (e1 & GROUP_SLOT_MASK));
  float4 S1 = s.shift[(e1 >> GROUP_CODE_SHIFT) & 31u];
  // Exceptions of the group atoms (first warp of the row: lanes 8a .. 8a + 7 for atom a): 1-4
  // scaled LJ/Coulomb and -q_i q_j erf(a r)/r, no cutoff, exactly as the atom-row kernel
  // evaluates them. They come before the row walk, so their chain of dependent loads overlaps
  // the walk's first loads instead of following its last pass.
  {
    const int a = lane >> 3, t = lane & 7;
    const bool vi = a < size && part == 0;
    const int i = vi ? ia[0] : 0;
    int ii = ia[0];
#pragma unroll
    for (int b = 1; b < G; ++b)
      if (a == b) ii = ia[b];
    const int eb = vi ? exc_start[ii] : 0, ee = vi ? exc_start[ii + 1] : 0;
    (void)i;
    const float4 pi = posq[ii];
    long long ex = 0, ey = 0, ez = 0, el = 0, ec = 0, ev = 0;
    for (int e = eb + t; e < ee; e += 8) {
      float pair_lj = 0.f, pair_coul = 0.f;
      const int jj = exc_partner[e];
      const float4 prm = exc_param[e];  // chargeProduct, ljA, ljB, fullProduct
      const float4 pk = posq[jj];
      float3 d = min_image(make_float3(pi.x - pk.x, pi.y - pk.y, pi.z - pk.z), s);
      const float r2 = fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z));
      const float inv_r = rsqrt_refined(r2);
      const float inv_r2 = inv_r * inv_r, inv_r6 = inv_r2 * inv_r2 * inv_r2;
      float scalar = 0.f;
      if (prm.y != 0.f || prm.z != 0.f) {
        const float a12 = prm.y * inv_r6 * inv_r6, b6 = prm.z * inv_r6;
        scalar += (12.0f * a12 - 6.0f * b6) * inv_r2;
        if (ENERGY) pair_lj += a12 - b6;
      }
      if (prm.x != 0.f) {
        const float qq = (float)ONE_4PI_EPS0 * prm.x;
        scalar += qq * inv_r * inv_r2;
        if (ENERGY) pair_coul += qq * inv_r;
      }
      if (alpha > 0.f && prm.w != 0.f) {
        const float qq = (float)ONE_4PI_EPS0 * prm.w;
        float gauss;
        const float r = r2 * inv_r;
        const float unscreened = 1.0f - erfc_and_gauss(alpha * r, gauss);
        scalar -= qq * (unscreened * inv_r - gauss_k * gauss) * inv_r2;
        if (ENERGY) pair_coul -= qq * unscreened * inv_r;
      }
      if (ENERGY) {
        el += (long long)to_fixed(pair_lj);
        ec += (long long)to_fixed(pair_coul);
        ev += (long long)to_fixed(scalar * r2);
      }
      ex += (long long)to_fixed(scalar * d.x);
      ey += (long long)to_fixed(scalar * d.y);
      ez += (long long)to_fixed(scalar * d.z);
    }
#pragma unroll
    for (int b = 0; b < G; ++b) {
      if (a == b) {
        acc[b][0] += ex;
        acc[b][1] += ey;
        acc[b][2] += ez;
        if (ENERGY) {
          acc[b][ENERGY ? 3 : 0] += el;
          acc[b][ENERGY ? 4 : 0] += ec;
          acc[b][ENERGY ? 5 : 0] += ev;
        }
      }
    }
  }
  for (int k0 = 32 * part; k0 < count; k0 += stride, k += stride) {
    const unsigned e = e1;
    const float4 pj = pj1, S = S1;
    const int2 info_j = info1;
    if (k0 + stride < count) {
      e1 = e2;
      pj1 = __ldg(spos + (e1 & GROUP_SLOT_MASK));
      info1 = __ldg(slot_info + (e1 & GROUP_SLOT_MASK));
      S1 = s.shift[(e1 >> GROUP_CODE_SHIFT) & 31u];
      e2 = k + 2 * stride < count ? (unsigned)__ldg(row + k + 2 * stride) : NO_ENTRY;
    }
    bool any = false;
#pragma unroll
    for (int a = 0; a < G; ++a) {
      const float4 pw = group_pos[wib][a];
      const float3 d = make_float3(pw.x - pj.x - S.x, pw.y - pj.y - S.y, pw.z - pj.z - S.z);
      const float r2 = fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z));
      any |= !((e >> (GROUP_MASK_SHIFT + a)) & 1u) && r2 <= cut2;
    }
    const unsigned hits = __ballot_sync(0xffffffffu, any);
    if (any) {
      const int slot = (head + queued + __popc(hits & ((1u << lane) - 1u))) & 63;
      ring_e[wib][slot] = e;
      ring_p[wib][slot] = pj;
      ring_i[wib][slot] = info_j;
    }
    queued += __popc(hits);
    if (queued >= 32) {
      __syncwarp();
      const int slot = (head + lane) & 63;
      group_pair_entry<ENERGY>(ring_e[wib][slot], ring_p[wib][slot], ring_i[wib][slot], group_pos[wib],
                               group_lj[wib], ljtab, s, alpha, gauss_k, cut2, acc, force, e_acc, n_atoms);
      __syncwarp();  // every lane has read its slot before the next pass refills the ring
      head = (head + 32) & 63;
      queued -= 32;
    }
  }
  if (queued > 0) {  // the last, partial batch
    __syncwarp();
    const int slot = (head + lane) & 63;
    const bool mine = lane < queued;
    group_pair_entry<ENERGY>(mine ? ring_e[wib][slot] : NO_ENTRY,
                             mine ? ring_p[wib][slot] : make_float4(0.f, 0.f, 0.f, 0.f),
                             mine ? ring_i[wib][slot] : make_int2(0, 0), group_pos[wib], group_lj[wib], ljtab, s,
                             alpha, gauss_k, cut2, acc, force, e_acc, n_atoms);
  }
  // the group atoms' sums over the warp: value 4a + c (component c of atom a) ends in lanes
  // 2(4a + c) and 2(4a + c) + 1; the lane with the even index adds it to the atom
  {
    long long v[16];
#pragma unroll
    for (int a = 0; a < G; ++a) {
#pragma unroll
      for (int c = 0; c < 3; ++c) v[4 * a + c] = acc[a][c];
      v[4 * a + 3] = 0;
    }
    const long long sum = warp_sum_sixteen(v, lane);
    const int slot = (lane >> 1) & 15, a = slot >> 2, c = slot & 3;
    int ii = ia[0];
#pragma unroll
    for (int b = 1; b < G; ++b)
      if (a == b) ii = ia[b];
    if ((lane & 1) == 0 && c < 3 && a < size && sum != 0)
      atomicAdd(force + c * (long long)n_atoms + ii, (unsigned long long)sum);
    if (ENERGY) {
#pragma unroll
      for (int b = 0; b < G; ++b) {
#pragma unroll
        for (int q = 0; q < 3; ++q) v[4 * b + q] = acc[b][ENERGY ? 3 + q : 0];
        v[4 * b + 3] = 0;
      }
      const long long esum = warp_sum_sixteen(v, lane);
      if ((lane & 1) == 0 && c < 3 && a < size && esum != 0)
        atomicAdd(e_acc + c * (long long)n_atoms + ii, (unsigned long long)esum);
    }
  }
}

// Per-atom pair energies from the integer sums: half of each (every pair's energy was added to
// both of its atoms), as the atom-row kernel stores them.
__global__ void k_group_pair_energies(const unsigned long long *__restrict__ e_acc, double *__restrict__ e_lj,
                                      double *__restrict__ e_coul, double *__restrict__ e_vir, int n_atoms) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_atoms) return;
  e_lj[i] = 0.5 * ((double)(long long)e_acc[i] / FORCE_SCALE);
  e_coul[i] = 0.5 * ((double)(long long)e_acc[n_atoms + i] / FORCE_SCALE);
  e_vir[i] = 0.5 * ((double)(long long)e_acc[2 * (long long)n_atoms + i] / FORCE_SCALE);
}

static void launch_group_pairs(const LaunchCtx &c, bool energy, int lanes, cudaStream_t stream) {
  const int split = lanes >= 128 ? 4 : lanes >= 64 ? 2 : 1;  // lanes per group row: warps sharing it x 32
  // (errors of these calls surface in the caller's cudaGetLastError, as the launches' do)
  if (!c.force_cleared)
    (void)cudaMemsetAsync(c.force, 0, sizeof(unsigned long long) * 3 * (size_t)c.n_atoms, stream);
  if (energy) (void)cudaMemsetAsync(c.e_acc, 0, sizeof(unsigned long long) * 3 * (size_t)c.n_atoms, stream);
  const int threads = 128;
  const int blocks = (int)(((long long)c.n_groups_total * split * 32 + threads - 1) / threads);
  constexpr int LJ_SMEM_MAX = 4096;
  const int lj_entries = c.lj_entries <= LJ_SMEM_MAX ? c.lj_entries : 0;
  const size_t smem = sizeof(float2) * lj_entries;
  if (energy) {
    k_group_pairs<true><<<blocks, threads, smem, stream>>>(
        c.posq, c.spos, c.slot_info, c.group_order, c.group_sys, c.sys, c.lj, c.gnbr, c.gnbr_count, c.gfirst,
        c.gsize, c.exc_start, c.exc_partner, c.exc_param, c.force, c.e_acc, c.n_atoms, c.n_groups_total, lj_entries,
        split);
    k_group_pair_energies<<<(c.n_atoms + 255) / 256, 256, 0, stream>>>(c.e_acc, c.e_lj, c.e_coul, c.e_vir, c.n_atoms);
  } else {
    k_group_pairs<false><<<blocks, threads, smem, stream>>>(
        c.posq, c.spos, c.slot_info, c.group_order, c.group_sys, c.sys, c.lj, c.gnbr, c.gnbr_count, c.gfirst,
        c.gsize, c.exc_start, c.exc_partner, c.exc_param, c.force, c.e_acc, c.n_atoms, c.n_groups_total, lj_entries,
        split);
  }
}

template <bool ENERGY, int LANES, bool PAIR_FIXED>
static void launch_nb(const LaunchCtx &c, cudaStream_t stream) {
  const int threads = 128;
  const long long total = (long long)c.n_atoms * LANES;
  const int blocks = (int)((total + threads - 1) / threads);
  constexpr int LJ_SMEM_MAX = 4096;  // float2 entries (32 KB)
  const int lj_entries = c.lj_entries <= LJ_SMEM_MAX ? c.lj_entries : 0;
  k_nonbonded<ENERGY, LANES, PAIR_FIXED><<<blocks, threads, sizeof(float2) * lj_entries, stream>>>(
      c.posq, c.spos, c.sorted_orig, c.sorted_type, c.sys_of_atom, c.sys, c.lj, c.nbr, c.nbr_count, c.exc_start,
      c.exc_partner, c.exc_param, c.force, c.e_lj, c.e_coul, c.e_vir, c.n_atoms, lj_entries);
}

template <bool PAIR_FIXED>
static void launch_nb_lanes(const LaunchCtx &c, bool energy, int lanes, cudaStream_t stream) {
  if (energy) {
    if (lanes == 8) launch_nb<true, 8, PAIR_FIXED>(c, stream);
    else if (lanes == 16) launch_nb<true, 16, PAIR_FIXED>(c, stream);
    else launch_nb<true, 32, PAIR_FIXED>(c, stream);
  } else {
    if (lanes == 8) launch_nb<false, 8, PAIR_FIXED>(c, stream);
    else if (lanes == 16) launch_nb<false, 16, PAIR_FIXED>(c, stream);
    else launch_nb<false, 32, PAIR_FIXED>(c, stream);
  }
}

void launch_nonbonded(const LaunchCtx &c, bool energy, int lanes, cudaStream_t stream) {
  if (c.pair_list != 1) launch_group_pairs(c, energy, lanes, stream);
  else if (c.pair_fixed) launch_nb_lanes<true>(c, energy, lanes, stream);
  else launch_nb_lanes<false>(c, energy, lanes, stream);
}

int nonbonded_launches(const LaunchCtx &c, bool energy) { return c.pair_list != 1 && energy ? 2 : 1; }

// ------------------------------------------------------------------ bonded + restraints
// One thread per term (bonds | angles | torsions | restraints); forces are added to the
// fixed-point array with 64-bit integer atomics (order-independent, deterministic).
// Functional forms as cpu/forces/bonded.js:22-207 and shared/topology/restraints.js:93-126.
template <bool ENERGY>
__global__ void k_bonded(const float4 *__restrict__ posq, const int *__restrict__ sys_of_atom,
                         const DevSys *__restrict__ sys, const int2 *__restrict__ bond_atoms,
                         const float2 *__restrict__ bond_param, int n_bonds,
                         const int4 *__restrict__ angle_atoms, const float2 *__restrict__ angle_param,
                         int n_angles, const int4 *__restrict__ tor_atoms,
                         const float4 *__restrict__ tor_param, int n_tors,
                         const int *__restrict__ rest_atom, const float4 *__restrict__ rest_param,
                         int n_rest, unsigned long long *__restrict__ force,
                         double *__restrict__ e_term, double *__restrict__ e_term_vir, int n_atoms) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long *fxp = force, *fyp = force + n_atoms, *fzp = force + 2 * (long long)n_atoms;
  const int total = n_bonds + n_angles + n_tors + n_rest;
  if (t >= total) return;
  float energy = 0.f, virial = 0.f;  // virial: sum_k F_k.(r_k - r_ref) over the term's atoms
  if (t < n_bonds) {
    const int2 a = bond_atoms[t];
    const float2 p = bond_param[t];
    const float4 A = posq[a.x], B = posq[a.y];
    const float dx = A.x - B.x, dy = A.y - B.y, dz = A.z - B.z;
    const float r = sqrtf(dx * dx + dy * dy + dz * dz);
    const float stretch = r - p.y;
    energy = 0.5f * p.x * stretch * stretch;
    const float sc = r > 0.f ? p.x * stretch / r : 0.f;
    virial = -sc * r * r;
    add_fixed(fxp + a.x, -sc * dx); add_fixed(fyp + a.x, -sc * dy); add_fixed(fzp + a.x, -sc * dz);
    add_fixed(fxp + a.y, sc * dx); add_fixed(fyp + a.y, sc * dy); add_fixed(fzp + a.y, sc * dz);
  } else if ((t -= n_bonds) < n_angles) {
    const int4 a = angle_atoms[t];
    const float2 p = angle_param[t];
    const float4 A = posq[a.x], B = posq[a.y], Cc = posq[a.z];
    const float v1x = A.x - B.x, v1y = A.y - B.y, v1z = A.z - B.z;
    const float v2x = Cc.x - B.x, v2y = Cc.y - B.y, v2z = Cc.z - B.z;
    const float n1 = v1x * v1x + v1y * v1y + v1z * v1z, n2 = v2x * v2x + v2y * v2y + v2z * v2z;
    const float nx = v1y * v2z - v1z * v2y, ny = v1z * v2x - v1x * v2z, nz = v1x * v2y - v1y * v2x;
    const float cm = sqrtf(nx * nx + ny * ny + nz * nz);
    const float dot = v1x * v2x + v1y * v2y + v1z * v2z;
    const float theta = atan2f(cm, dot), dev = theta - p.y;
    energy = 0.5f * p.x * dev * dev;
    const float dE = p.x * dev, safe = fmaxf(cm, 1e-12f);
    const float s1 = -dE / (n1 * safe), s2 = dE / (n2 * safe);
    const float fax = s1 * (v1y * nz - v1z * ny), fay = s1 * (v1z * nx - v1x * nz), faz = s1 * (v1x * ny - v1y * nx);
    const float fcx = s2 * (v2y * nz - v2z * ny), fcy = s2 * (v2z * nx - v2x * nz), fcz = s2 * (v2x * ny - v2y * nx);
    virial = fax * v1x + fay * v1y + faz * v1z + fcx * v2x + fcy * v2y + fcz * v2z;
    add_fixed(fxp + a.x, fax); add_fixed(fyp + a.x, fay); add_fixed(fzp + a.x, faz);
    add_fixed(fxp + a.z, fcx); add_fixed(fyp + a.z, fcy); add_fixed(fzp + a.z, fcz);
    add_fixed(fxp + a.y, -(fax + fcx)); add_fixed(fyp + a.y, -(fay + fcy)); add_fixed(fzp + a.y, -(faz + fcz));
  } else if ((t -= n_angles) < n_tors) {
    const int4 a = tor_atoms[t];
    const float4 p = tor_param[t];  // k, n, phase
    const float4 A = posq[a.x], B = posq[a.y], Cc = posq[a.z], D = posq[a.w];
    const float b1x = B.x - A.x, b1y = B.y - A.y, b1z = B.z - A.z;
    const float b2x = Cc.x - B.x, b2y = Cc.y - B.y, b2z = Cc.z - B.z;
    const float b3x = D.x - Cc.x, b3y = D.y - Cc.y, b3z = D.z - Cc.z;
    const float n1x = b1y * b2z - b1z * b2y, n1y = b1z * b2x - b1x * b2z, n1z = b1x * b2y - b1y * b2x;
    const float n2x = b2y * b3z - b2z * b3y, n2y = b2z * b3x - b2x * b3z, n2z = b2x * b3y - b2y * b3x;
    const float n1s = n1x * n1x + n1y * n1y + n1z * n1z, n2s = n2x * n2x + n2y * n2y + n2z * n2z;
    const float b2l = sqrtf(b2x * b2x + b2y * b2y + b2z * b2z);
    if (!(n1s < 1e-24f || n2s < 1e-24f || b2l < 1e-12f)) {
      const float dn = n1x * n2x + n1y * n2y + n1z * n2z;
      const float cdb = (n1y * n2z - n1z * n2y) * b2x + (n1z * n2x - n1x * n2z) * b2y +
                        (n1x * n2y - n1y * n2x) * b2z;
      const float phi = atan2f(cdb / b2l, dn);
      const float arg = p.y * phi - p.z;
      float sa, ca;
      sincosf(arg, &sa, &ca);
      energy = p.x * (1.0f + ca);
      const float dEdphi = -p.x * p.y * sa;
      const float fA = dEdphi * b2l / n1s, fD = -dEdphi * b2l / n2s;
      const float inv = 1.0f / (b2l * b2l);
      const float tt = (b1x * b2x + b1y * b2y + b1z * b2z) * inv;
      const float uu = (b3x * b2x + b3y * b2y + b3z * b2z) * inv;
      const float fax = fA * n1x, fay = fA * n1y, faz = fA * n1z;
      const float fdx = fD * n2x, fdy = fD * n2y, fdz = fD * n2z;
      const float fcx = tt * fax - (1.f + uu) * fdx, fcy = tt * fay - (1.f + uu) * fdy,
                  fcz = tt * faz - (1.f + uu) * fdz;
      // about atom B: r_A - r_B = -b1, r_C - r_B = b2, r_D - r_B = b2 + b3
      virial = -(fax * b1x + fay * b1y + faz * b1z) + fcx * b2x + fcy * b2y + fcz * b2z +
               fdx * (b2x + b3x) + fdy * (b2y + b3y) + fdz * (b2z + b3z);
      add_fixed(fxp + a.x, fax); add_fixed(fyp + a.x, fay); add_fixed(fzp + a.x, faz);
      add_fixed(fxp + a.w, fdx); add_fixed(fyp + a.w, fdy); add_fixed(fzp + a.w, fdz);
      add_fixed(fxp + a.y, -(1.f + tt) * fax + uu * fdx);
      add_fixed(fyp + a.y, -(1.f + tt) * fay + uu * fdy);
      add_fixed(fzp + a.y, -(1.f + tt) * faz + uu * fdz);
      add_fixed(fxp + a.z, tt * fax - (1.f + uu) * fdx);
      add_fixed(fyp + a.z, tt * fay - (1.f + uu) * fdy);
      add_fixed(fzp + a.z, tt * faz - (1.f + uu) * fdz);
    }
  } else {
    t -= n_tors;
    const int atom = rest_atom[t];
    const float4 p = rest_param[t];  // reference x, y, z, k
    const DevSys &s = sys[sys_of_atom[atom]];
    const float4 A = posq[atom];
    float3 d = min_image(make_float3(A.x - p.x, A.y - p.y, A.z - p.z), s);
    energy = p.w * (d.x * d.x + d.y * d.y + d.z * d.z);
    const float sc = -2.0f * p.w;
    add_fixed(fxp + atom, sc * d.x); add_fixed(fyp + atom, sc * d.y); add_fixed(fzp + atom, sc * d.z);
    virial = sc * (d.x * A.x + d.y * A.y + d.z * A.z);  // F.r: not translation invariant
  }
  if (ENERGY) {
    e_term[blockIdx.x * blockDim.x + threadIdx.x] = (double)energy;
    e_term_vir[blockIdx.x * blockDim.x + threadIdx.x] = (double)virial;
  }
}

void launch_bonded(const LaunchCtx &c, bool energy, cudaStream_t stream) {
  const int total = c.n_bonds + c.n_angles + c.n_tors + c.n_rest;
  if (total == 0) return;
  const int tb = 128;
  if (energy)
    k_bonded<true><<<(total + tb - 1) / tb, tb, 0, stream>>>(
        c.posq, c.sys_of_atom, c.sys, c.bond_atoms, c.bond_param, c.n_bonds, c.angle_atoms,
        c.angle_param, c.n_angles, c.tor_atoms, c.tor_param, c.n_tors, c.rest_atom, c.rest_param,
        c.n_rest, c.force, c.e_term, c.e_term_vir, c.n_atoms);
  else
    k_bonded<false><<<(total + tb - 1) / tb, tb, 0, stream>>>(
        c.posq, c.sys_of_atom, c.sys, c.bond_atoms, c.bond_param, c.n_bonds, c.angle_atoms,
        c.angle_param, c.n_angles, c.tor_atoms, c.tor_param, c.n_tors, c.rest_atom, c.rest_param,
        c.n_rest, c.force, c.e_term, c.e_term_vir, c.n_atoms);
}

// ------------------------------------------------------------------ molecular virial
// One warp per molecule, after every force term: sum_i F_i.(r_i - R) over the molecule's
// atoms, R its centre of mass (positions are never wrapped, so molecules are whole).
// Added to the atomic virial it turns dU/dlnV for atoms scaled with the box into dU/dlnV
// for molecules scaled rigidly about their centres.
__global__ void k_molecular_virial(const float4 *__restrict__ posq, const float *__restrict__ masses,
                                   const int *__restrict__ mol_start, const int *__restrict__ mol_atoms,
                                   const unsigned long long *__restrict__ force, double *__restrict__ mol_vir,
                                   int n_molecules, int n_atoms) {
  const int m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (m >= n_molecules) return;
  const int begin = mol_start[m], end = mol_start[m + 1];
  const int i0 = mol_atoms[begin];
  const float4 r0 = posq[i0];
  double cx = 0, cy = 0, cz = 0, mt = 0;
  for (int k = begin + lane; k < end; k += 32) {
    const int i = mol_atoms[k];
    const float4 p = posq[i];
    const double w = masses[i];
    cx += w * (double)(p.x - r0.x);
    cy += w * (double)(p.y - r0.y);
    cz += w * (double)(p.z - r0.z);
    mt += w;
  }
  cx = warp_sum(cx);
  cy = warp_sum(cy);
  cz = warp_sum(cz);
  mt = warp_sum(mt);
  if (mt > 0) {
    cx /= mt;
    cy /= mt;
    cz /= mt;
  }
  double v = 0;
  for (int k = begin + lane; k < end; k += 32) {
    const int i = mol_atoms[k];
    const float4 p = posq[i];
    const double fx = (double)(long long)force[i] / FORCE_SCALE;
    const double fy = (double)(long long)force[n_atoms + i] / FORCE_SCALE;
    const double fz = (double)(long long)force[2 * (long long)n_atoms + i] / FORCE_SCALE;
    v += fx * ((double)(p.x - r0.x) - cx) + fy * ((double)(p.y - r0.y) - cy) + fz * ((double)(p.z - r0.z) - cz);
  }
  v = warp_sum(v);
  if (lane == 0) mol_vir[m] = v;
}

void launch_molecular_virial(const LaunchCtx &c, cudaStream_t stream) {
  if (c.n_molecules <= 0) return;
  const int tb = 128;
  k_molecular_virial<<<(int)(((long long)c.n_molecules * 32 + tb - 1) / tb), tb, 0, stream>>>(
      c.posq, c.masses, c.mol_start, c.mol_atoms, c.force, c.mol_vir, c.n_molecules, c.n_atoms);
}

}  // namespace rmd
