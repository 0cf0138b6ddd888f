// Deterministic FP64 energy reductions and the on-device Monte Carlo barostat.
//
// Energies: every energy-producing kernel writes per-item FP64 contributions (per atom,
// per bonded term, per PME block); one block per segment sums its range in a fixed order,
// and one thread per system adds the segments in a fixed order and the volume-dependent
// constants: Ewald self and net-charge terms (cpu/forces/pme.js:270-286) and the LJ
// dispersion correction (shared/dispersion.js:76-82). Same bits every run.
//
// Barostat: the reference's attemptVolumeChange (webgpu/simulation.js:995-1070) does two
// host round trips per move. Here the proposal (the same uniformAt draws on seed^0x5a17),
// the molecule-centroid scaling (barostat.js:25-108), the Metropolis test
// (barostat.js:158-162) in FP64 and the restore on rejection are all kernels, so a move
// sits inside a CUDA graph with no host synchronisation.
#include <cmath>

#include "common.cuh"
#include "kernels.h"

namespace rmd {

__global__ void k_segment_sum(const Segment *__restrict__ segs, double *__restrict__ out) {
  const Segment sg = segs[blockIdx.x];
  double acc = 0.0;
  for (long long k = sg.start + threadIdx.x; k < sg.end; k += blockDim.x) {
    acc += sg.data[k];
    if (sg.data2) acc += sg.data2[k];
  }
  __shared__ double red[32];
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    out[blockIdx.x] = t;
  }
}

__global__ void k_energy_finalize(const Segment *__restrict__ segs, int n_segments,
                                  const double *__restrict__ seg_out, double *__restrict__ energies,
                                  const DevSysD *__restrict__ sysd, int n_systems) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_systems) return;
  double e[N_ENERGY];
  for (int k = 0; k < N_ENERGY; ++k) e[k] = 0.0;
  for (int k = 0; k < n_segments; ++k)
    if (segs[k].sys == s) e[segs[k].term] += seg_out[k];
  const DevSysD d = sysd[s];
  const double sqrt_pi = 1.7724538509055160273;
  if (d.alpha > 0) {
    e[E_SELF] = -ONE_4PI_EPS0 * d.alpha * d.q2_sum / sqrt_pi;
    e[E_NET] = -ONE_4PI_EPS0 * M_PI * d.q_sum * d.q_sum / (2.0 * d.alpha * d.alpha * d.volume);
  }
  if (d.dispersion_on && d.volume > 0 && d.cutoff > 0) {
    const double c3 = d.cutoff * d.cutoff * d.cutoff, c9 = c3 * c3 * c3;
    e[E_DISPERSION] = (2.0 * M_PI / d.volume) * (d.disp_a / (9.0 * c9) - d.disp_b / (3.0 * c3));
  }
  e[E_POTENTIAL] = e[E_BOND] + e[E_ANGLE] + e[E_TORSION] + e[E_LJ] + e[E_COUL_DIRECT] +
                   e[E_RECIP] + e[E_SELF] + e[E_NET] + e[E_DISPERSION] + e[E_RESTRAINT];
  // dU/dlnV with every coordinate scaled with the box: -(1/3) sum F.r for the pair,
  // exception and bonded terms (F.r about any atom of a term); for the reciprocal sum
  // E = sum_k f(m^2) |S(m)|^2 / V with m^2 ~ V^(-2/3), -E + (2/3) sum_k E_k (1 + pi^2 m^2 /
  // alpha^2); the 1/V terms (dispersion, net charge) give -E each. Scaling molecules rigidly
  // about their centres instead moves atom i by (lambda - 1) R_mol(i) rather than
  // (lambda - 1) r_i, which adds (1/3) sum_i F_i.(r_i - R_mol(i)).
  e[E_DUDLNV] = (-e[E_VIR_SR] + e[E_VIR_MOL]) / 3.0 - e[E_RECIP] + (2.0 / 3.0) * e[E_VIR_REC] -
                e[E_DISPERSION] - e[E_NET];
  for (int k = 0; k < N_ENERGY; ++k) energies[s * N_ENERGY + k] = e[k];
}

void launch_energy_reduce(const Segment *segments, int n_segments, double *seg_out,
                          double *energies, const DevSysD *sysd, int n_systems, cudaStream_t stream) {
  if (n_segments > 0) k_segment_sum<<<n_segments, 256, 0, stream>>>(segments, seg_out);
  k_energy_finalize<<<(n_systems + 63) / 64, 64, 0, stream>>>(segments, n_segments, seg_out,
                                                              energies, sysd, n_systems);
}

// ------------------------------------------------------------------------ box helpers
__device__ void set_box(DevSys &s, DevSysD &d, const double *b) {
  for (int k = 0; k < 9; ++k) d.box[k] = b[k];
  const double ax = b[0], bx = b[3], by = b[4], cx = b[6], cy = b[7], cz = b[8];
  double r[9] = {1.0 / ax, 0, 0, -bx / (ax * by), 1.0 / by, 0,
                 (bx * cy - by * cx) / (ax * by * cz), -cy / (by * cz), 1.0 / cz};
  for (int k = 0; k < 9; ++k) {
    s.box[k] = (float)b[k];
    s.recip[k] = (float)r[k];
  }
  for (int code = 0; code < 27; ++code) {
    const int ka = code / 9 - 1, kb = (code / 3) % 3 - 1, kc = code % 3 - 1;
    s.shift[code] = make_float4((float)(ka * b[0] + kb * b[3] + kc * b[6]), (float)(ka * b[1] + kb * b[4] + kc * b[7]),
                                (float)(ka * b[2] + kb * b[5] + kc * b[8]), 0.f);
  }
  s.inv_diag[0] = (float)(1.0 / ax);
  s.inv_diag[1] = (float)(1.0 / by);
  s.inv_diag[2] = (float)(1.0 / cz);
  d.volume = fabs(ax * by * cz);
  // Cells at least the list cutoff wide (cells.js:101-171), never more than allocated.
  const double w[3] = {fabs(ax), fabs(by), fabs(cz)};
  for (int k = 0; k < 3; ++k) {
    int c = (int)floor(w[k] / d.list_cutoff);
    c = c < 1 ? 1 : c;
    s.cell_counts[k] = c < d.max_counts[k] ? c : d.max_counts[k];
  }
}

__global__ void k_update_box(DevSys *sys, DevSysD *sysd, int n) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  double b[9];
  for (int k = 0; k < 9; ++k) b[k] = sysd[s].box[k];
  set_box(sys[s], sysd[s], b);
}

void launch_update_box(DevSys *sys, DevSysD *sysd, int n_systems, cudaStream_t stream) {
  k_update_box<<<(n_systems + 63) / 64, 64, 0, stream>>>(sys, sysd, n_systems);
}

__global__ void k_advance_steps(long long *step_base, int n, int count) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) step_base[s] += count;
}

void launch_advance_steps(long long *step_base, int n_systems, int count, cudaStream_t stream) {
  k_advance_steps<<<(n_systems + 63) / 64, 64, 0, stream>>>(step_base, n_systems, count);
}

// ------------------------------------------------------------------------ barostat
__device__ __forceinline__ double uniform_d(uint32_t seed, uint32_t a, uint32_t b, uint32_t c) {
  return rng_uniform_d(seed, a, b, c);
}

// One thread per system: draw the volume change, refuse it if the cutoff would not fit,
// save the old box and energies, and install the proposed box.
__global__ void k_baro_propose(BaroArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n_systems) return;
  double *b = a.baro + (long long)s * N_BARO;
  const bool learned = b[B_LEARNED] != 0.0;
  if (!learned) {
    b[B_ACCEPT] = 1.0;
    b[B_REFUSED] = 0.0;
    b[B_LSCALE] = 1.0;
  }
  if (b[B_ACTIVE] == 0.0) return;
  if (a.keep_lists) {
    a.rebuilt[s] = 0;
    a.saved_allow[s] = a.allow[s];
  }
  DevSysD &d = a.sysd[s];
  const double volume = d.volume;
  for (int k = 0; k < N_ENERGY; ++k) a.saved_energies[s * N_ENERGY + k] = a.energies[s * N_ENERGY + k];
  b[B_OLD_E] = a.energies[s * N_ENERGY + E_POTENTIAL];
  b[B_OLD_VOL] = volume;
  double ls;
  if (learned) {
    // the move was drawn (and refused or screened) by the surrogate's stage 1
    b[B_ACCEPT] = 1.0;
    if (b[B_REFUSED] != 0.0 || b[B_SCREENED] != 0.0) return;
    ls = b[B_LSCALE];
  } else {
    if (b[B_SCALE] == 0.0) b[B_SCALE] = 0.01 * volume;
    b[B_ATTEMPTS] += 1.0;
    b[B_WINDOW_ATT] += 1.0;
    const uint32_t seed = ((uint32_t)b[B_SEED]) ^ 0x5a17u;
    const uint32_t attempt = (uint32_t)b[B_ATTEMPTS];
    const double u = uniform_d(seed, attempt, 0, 0);
    const double dv = b[B_SCALE] * 2.0 * (u - 0.5);
    const double nv = volume + dv;
    b[B_DV] = dv;
    if (!(nv > 0)) {
      b[B_REFUSED] = 1.0;
      b[B_REFUSALS] += 1.0;
      return;
    }
    ls = cbrt(nv / volume);
    const double smallest = ls * fmin(fabs(d.box[0]), fmin(fabs(d.box[4]), fabs(d.box[8])));
    if (d.cutoff > 0.5 * smallest) {  // simulation.js:1016-1035
      b[B_REFUSED] = 1.0;
      b[B_REFUSALS] += 1.0;
      return;
    }
    b[B_LSCALE] = ls;
  }
  for (int k = 0; k < 9; ++k) d.saved_box[k] = d.box[k];
  d.saved_volume = volume;
  for (int k = 0; k < 3; ++k) d.saved_counts[k] = a.sys[s].cell_counts[k];
  double nb[9];
  for (int k = 0; k < 9; ++k) nb[k] = d.box[k] * ls;
  set_box(a.sys[s], d, nb);
}

// One warp per molecule: mass-weighted centroid (FP64 accumulation), then shift every
// atom of the molecule by (s - 1) * centroid; the old positions and forces are saved.
__global__ void k_baro_centroid_scale(BaroArgs a, int n_molecules, const double *__restrict__ fixed_scales) {
  const int m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (m >= n_molecules) return;
  const int begin = a.mol_start[m], end = a.mol_start[m + 1];
  const int s = a.sys_of_atom[a.mol_atoms[begin]];
  const double ls = fixed_scales ? fixed_scales[s] : a.baro[(long long)s * N_BARO + B_LSCALE];
  // Save positions and forces of this molecule's atoms (restored if the move is rejected), and
  // for a move on the current lists their wrap shifts and displacement origins.
  const bool keep = a.keep_lists && !fixed_scales;
  for (int k = begin + lane; k < end; k += 32) {
    const int i = a.mol_atoms[k];
    a.saved_posq[i] = a.posq[i];
    a.saved_force[i] = a.force[i];
    a.saved_force[a.n_atoms + i] = a.force[a.n_atoms + i];
    a.saved_force[2 * (long long)a.n_atoms + i] = a.force[2 * (long long)a.n_atoms + i];
    if (keep) {
      a.saved_wrap[i] = a.wrap[i];
      a.saved_origin[i] = a.origin[i];
    }
  }
  if (ls == 1.0) return;
  double cx = 0, cy = 0, cz = 0, mt = 0;
  for (int k = begin + lane; k < end; k += 32) {
    const int i = a.mol_atoms[k];
    const float4 p = a.posq[i];
    const double mm = a.masses[i];
    cx += mm * p.x;
    cy += mm * p.y;
    cz += mm * p.z;
    mt += mm;
  }
  cx = warp_sum(cx);
  cy = warp_sum(cy);
  cz = warp_sum(cz);
  mt = warp_sum(mt);
  if (!(mt > 0)) {  // massless molecule: plain mean (barostat.js:47-58)
    cx = cy = cz = 0;
    for (int k = begin + lane; k < end; k += 32) {
      const float4 p = a.posq[a.mol_atoms[k]];
      cx += p.x;
      cy += p.y;
      cz += p.z;
    }
    cx = warp_sum(cx);
    cy = warp_sum(cy);
    cz = warp_sum(cz);
    mt = (double)(end - begin);
  }
  cx /= mt;
  cy /= mt;
  cz /= mt;
  const double f = ls - 1.0;
  float spread = 0.f;  // the molecule's largest atom-centroid distance
  for (int k = begin + lane; k < end; k += 32) {
    const int i = a.mol_atoms[k];
    float4 p = a.posq[i];
    if (keep) {
      const double ex = (double)p.x - cx, ey = (double)p.y - cy, ez = (double)p.z - cz;
      spread = fmaxf(spread, (float)sqrt(ex * ex + ey * ey + ez * ez));
    }
    p.x = (float)((double)p.x + f * cx);
    p.y = (float)((double)p.y + f * cy);
    p.z = (float)((double)p.z + f * cz);
    a.posq[i] = p;
    if (keep) {
      // The lists keep describing the scaled state: the wrap shift is the same whole number of
      // box vectors in the scaled box, the displacement origin moves with the atom (so the
      // check keeps measuring the motion since the build; what the scaling does to a pair
      // distance is counted in `allow`), and the cell-ordered copy follows.
      const float4 w = a.wrap[i], o = a.origin[i];
      const float4 ws = make_float4((float)((double)w.x * ls), (float)((double)w.y * ls), (float)((double)w.z * ls), 0.f);
      a.wrap[i] = ws;
      a.origin[i] = make_float4((float)((double)o.x + f * cx), (float)((double)o.y + f * cy),
                                (float)((double)o.z + f * cz), o.w);
      a.spos[a.rank[i]] = make_float4(p.x - ws.x, p.y - ws.y, p.z - ws.z, p.w);
    }
  }
  if (keep) {
    spread = warp_max(spread);
    if (lane == 0) atomic_max_nonneg(&a.spread_bits[s], spread);
  }
}

// One thread per system moving on its current lists: the move changes a pair's vector by
// (s - 1)(d + c_i - x_i - c_j + x_j) (d the vector before the move, c the molecules'
// centroids), at most |s - 1| (r_list + 2 spread) for a pair within the list cutoff: half of
// that per atom is added to the rebuild decision's allowance.
__global__ void k_baro_allow(BaroArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n_systems) return;
  const double *b = a.baro + (long long)s * N_BARO;
  const float spread = __uint_as_float(a.spread_bits[s]);
  a.spread_bits[s] = 0u;
  if (b[B_ACTIVE] == 0.0 || b[B_REFUSED] != 0.0 || b[B_SCREENED] != 0.0) return;
  const double ls = b[B_LSCALE];
  if (ls == 1.0) return;
  const double reach = fabs(ls - 1.0) * ((double)a.sys[s].list_cutoff + 2.0 * (double)spread);
  a.allow[s] += (float)(0.5 * reach * 1.001);
}

// One thread per system: the Metropolis test in FP64 (metropolisWeight, barostat.js:158-162)
// with the second uniformAt draw, the acceptance window, and on rejection the old box and
// energies (positions and forces are restored per atom by k_baro_restore).
__global__ void k_baro_decide(BaroArgs a) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= a.n_systems) return;
  double *b = a.baro + (long long)s * N_BARO;
  if (b[B_ACTIVE] == 0.0 || b[B_REFUSED] != 0.0 || b[B_SCREENED] != 0.0) {
    b[B_ACCEPT] = 1.0;  // nothing moved; nothing to restore
    if (b[B_ACTIVE] != 0.0) {
      b[B_ACCEPT] = 0.0;
      b[B_NEW_E] = b[B_OLD_E];
      b[B_WEIGHT] = b[B_SCREENED] != 0.0 ? b[B_PRED] : 0.0;
    }
    return;
  }
  const bool learned = b[B_LEARNED] != 0.0;
  DevSysD &d = a.sysd[s];
  const double kT = b[B_KT];
  const double new_e = a.energies[s * N_ENERGY + E_POTENTIAL];
  b[B_NEW_E] = new_e;
  const double ratio = d.volume / b[B_OLD_VOL];
  const double w = (new_e - b[B_OLD_E]) + b[B_PRESSURE] * b[B_DV] - b[B_NMOL] * kT * log(ratio);
  b[B_WEIGHT] = w;
  const uint32_t seed = ((uint32_t)b[B_SEED]) ^ 0x5a17u;
  const uint32_t attempt = (uint32_t)b[B_ATTEMPTS];
  bool accept;
  if (learned && b[B_SCREENING] != 0.0) {
    // stage 2 of delayed acceptance: min(1, exp(-w/kT) a1(reverse) / a1(forward))
    const double log_a2 = -w / kT + fmin(0.0, -b[B_PRED_REV] / kT) - fmin(0.0, -b[B_PRED] / kT);
    accept = log_a2 >= 0.0 || uniform_d(seed, attempt, 1, 0) < exp(log_a2);
  } else {
    accept = w <= 0.0 || uniform_d(seed, attempt, 1, 0) < exp(-w / kT);
  }
  b[B_EXACT_EVALS] += 1.0;
  if (learned) {  // the exact sample, appended to the surrogate's replay by its training kernel
    b[B_FEATURE0 + 8] = new_e - b[B_OLD_E];
    b[B_FEATURE0 + 9] = 1.0;
  }
  b[B_ACCEPT] = accept ? 1.0 : 0.0;
  if (accept) {
    b[B_ACCEPTED] += 1.0;
    b[B_WINDOW_ACC] += 1.0;
  } else {
    for (int k = 0; k < 9; ++k) d.box[k] = d.saved_box[k];
    double ob[9];
    for (int k = 0; k < 9; ++k) ob[k] = d.saved_box[k];
    set_box(a.sys[s], d, ob);
    for (int k = 0; k < 3; ++k) a.sys[s].cell_counts[k] = d.saved_counts[k];
    for (int k = 0; k < N_ENERGY; ++k) a.energies[s * N_ENERGY + k] = a.saved_energies[s * N_ENERGY + k];
    if (!a.keep_lists || a.rebuilt[s]) {
      // The lists of the trial evaluation were built in the trial box, with wrap shifts that
      // are multiples of its vectors: they do not describe the restored positions in the
      // restored box. Mark them stale (the largest finite displacement), so that the next
      // rebuild decision rebuilds this system before its next force evaluation.
      a.disp[s] = 0x7f7fffffu;
    } else {
      a.allow[s] = a.saved_allow[s];  // the lists from before the move describe the restored state
    }
  }
  if (!learned && b[B_WINDOW_ATT] >= 10.0) {  // simulation.js:1058-1063 (stage 1 does it when learned)
    const double rate = b[B_WINDOW_ACC] / b[B_WINDOW_ATT];
    if (rate < 0.25) b[B_SCALE] /= 1.1;
    else if (rate > 0.75) b[B_SCALE] = fmin(b[B_SCALE] * 1.1, 0.3 * d.volume);
    b[B_WINDOW_ATT] = 0.0;
    b[B_WINDOW_ACC] = 0.0;
  }
}

__global__ void k_baro_restore(BaroArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n_atoms) return;
  const int s = a.sys_of_atom[i];
  if (a.baro[(long long)s * N_BARO + B_ACCEPT] != 0.0) return;
  const float4 p = a.saved_posq[i];
  a.posq[i] = p;
  a.force[i] = a.saved_force[i];
  a.force[a.n_atoms + i] = a.saved_force[a.n_atoms + i];
  a.force[2 * (long long)a.n_atoms + i] = a.saved_force[2 * (long long)a.n_atoms + i];
  if (a.keep_lists && !a.rebuilt[s]) {  // the lists stand: their wraps, origins and copy as before
    const float4 w = a.saved_wrap[i];
    a.wrap[i] = w;
    a.origin[i] = a.saved_origin[i];
    a.spos[a.rank[i]] = make_float4(p.x - w.x, p.y - w.y, p.z - w.z, p.w);
  }
}

void launch_baro_propose(const BaroArgs &a, cudaStream_t stream) {
  k_baro_propose<<<(a.n_systems + 63) / 64, 64, 0, stream>>>(a);
}
void launch_baro_scale(const BaroArgs &a, cudaStream_t stream) {
  const int tb = 128;
  k_baro_centroid_scale<<<(a.n_molecules * 32 + tb - 1) / tb, tb, 0, stream>>>(a, a.n_molecules, nullptr);
}
void launch_scale_fixed(const BaroArgs &a, const double *scales, cudaStream_t stream) {
  const int tb = 128;
  k_baro_centroid_scale<<<(a.n_molecules * 32 + tb - 1) / tb, tb, 0, stream>>>(a, a.n_molecules, scales);
}
void launch_baro_allow(const BaroArgs &a, cudaStream_t stream) {
  k_baro_allow<<<(a.n_systems + 63) / 64, 64, 0, stream>>>(a);
}
void launch_baro_decide(const BaroArgs &a, cudaStream_t stream) {
  k_baro_decide<<<(a.n_systems + 63) / 64, 64, 0, stream>>>(a);
}
void launch_baro_restore(const BaroArgs &a, cudaStream_t stream) {
  k_baro_restore<<<(a.n_atoms + 127) / 128, 128, 0, stream>>>(a);
}

}  // namespace rmd
