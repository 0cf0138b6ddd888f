// Cell list and Verlet neighbour list for a batch of systems.
//
// Follows RainMD's cell-list.js:43-176 and neighbours.js:46-151 in what it produces —
// cells in (x, y, z) row-major order, each cell's atoms ascending by index, and per
// atom a full (both-direction) list of every non-excluded partner within cutoff+skin in
// the order of the deduplicated 27-cell stencil — so the lists are bit-identical to the
// reference's on the same f32 positions. How it is produced is B200-shaped:
//   - the histogram and the scatter use integer atomics, and a per-cell block rank-sort
//     (shared memory) restores the deterministic index order;
//   - the scan is one block per system;
//   - the neighbour search is one WARP per atom: lanes test 32 candidates of a cell at
//     once and a ballot/popc prefix compacts the survivors in order, so the list order
//     equals the sequential one without any per-atom serial loop.
#include "common.cuh"
#include "kernels.h"

namespace rmd {

struct LaunchCtxView {
  const float4 *posq;
  const int *atom_type;
  float4 *spos;
  float4 *wrap;
  int *sorted_orig, *sorted_type, *rank;
};

__global__ void k_cells_assign(const float4 *__restrict__ posq, const int *__restrict__ sys_of_atom,
                               const DevSys *__restrict__ sys, int *__restrict__ cell_of_atom,
                               int *__restrict__ cell_count, int n_atoms) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_atoms) return;
  const DevSys &s = sys[sys_of_atom[i]];
  float4 p = posq[i];
  int3 c = cell_coord(make_float3(p.x, p.y, p.z), s);
  int cell = (c.x * s.cell_counts[1] + c.y) * s.cell_counts[2] + c.z;
  cell_of_atom[i] = cell;
  atomicAdd(&cell_count[s.cell_base + cell], 1);
}

// One block per system: exclusive scan of the counts into cell_start, count -> 0.
__global__ void k_cells_scan(const DevSys *__restrict__ sys, int *__restrict__ cell_count,
                             int *__restrict__ cell_start) {
  const DevSys &s = sys[blockIdx.x];
  const int cells = s.cell_counts[0] * s.cell_counts[1] * s.cell_counts[2];
  __shared__ int warp_totals[32];
  __shared__ int running;
  if (threadIdx.x == 0) running = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  for (int chunk = 0; chunk < cells; chunk += blockDim.x) {
    int c = chunk + threadIdx.x;
    int v = c < cells ? cell_count[s.cell_base + c] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_totals[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int t = lane < warps ? warp_totals[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += y;
      }
      warp_totals[lane] = t;  // inclusive over warps
    }
    __syncthreads();
    int before = (warp > 0 ? warp_totals[warp - 1] : 0) + x - v;
    if (c < cells) {
      cell_start[s.cell_start_base + c] = running + before;
      cell_count[s.cell_base + c] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) running += warp_totals[warps - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) cell_start[s.cell_start_base + cells] = running;
}

__global__ void k_cells_scatter(const int *__restrict__ sys_of_atom, const DevSys *__restrict__ sys,
                                const int *__restrict__ cell_of_atom, const int *__restrict__ cell_start,
                                int *__restrict__ cell_cursor, int *__restrict__ cell_atoms,
                                int n_atoms) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_atoms) return;
  const DevSys &s = sys[sys_of_atom[i]];
  int cell = cell_of_atom[i];
  int slot = cell_start[s.cell_start_base + cell] + atomicAdd(&cell_cursor[s.cell_base + cell], 1);
  cell_atoms[s.atom_start + slot] = i;
}

// Write slot g's cell-ordered record for atom j: its position shifted into the box by
// whole box vectors (the shift is kept per atom so the integrator can apply it every step).
__device__ __forceinline__ void place_sorted(const LaunchCtxView &v, const DevSys &s, int g, int j) {
  const float4 p = v.posq[j];
  // floor of the same exact-rounding fractional coordinate the cell assignment used, so the
  // wrapped copy lies in (the closure of) the cell the atom was counted in
  float fl[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) fl[d] = floorf(frac_exact(make_float3(p.x, p.y, p.z), s, d));
  const float wx = fl[0] * s.box[0] + fl[1] * s.box[3] + fl[2] * s.box[6];
  const float wy = fl[0] * s.box[1] + fl[1] * s.box[4] + fl[2] * s.box[7];
  const float wz = fl[0] * s.box[2] + fl[1] * s.box[5] + fl[2] * s.box[8];
  v.spos[g] = make_float4(p.x - wx, p.y - wy, p.z - wz, p.w);
  v.wrap[j] = make_float4(wx, wy, wz, 0.f);
  v.sorted_orig[g] = j;
  v.sorted_type[g] = v.atom_type[j];
  v.rank[j] = g;
}

// One block per allocated cell: rank-sort the cell's slice ascending, zero the cursor, and
// write the cell-ordered records of its atoms.
__global__ void k_cells_sort(const int *__restrict__ cell_sys, const DevSys *__restrict__ sys,
                             const int *__restrict__ cell_start, int *__restrict__ cell_cursor,
                             int *__restrict__ cell_atoms, LaunchCtxView v) {
  const int g = blockIdx.x;
  const DevSys &s = sys[cell_sys[g]];
  const int c = g - s.cell_base;
  const int cells = s.cell_counts[0] * s.cell_counts[1] * s.cell_counts[2];
  if (c >= cells) return;
  if (threadIdx.x == 0) cell_cursor[g] = 0;
  const int begin = cell_start[s.cell_start_base + c], end = cell_start[s.cell_start_base + c + 1];
  const int n = end - begin;
  if (n <= 0) return;
  int *slice = cell_atoms + s.atom_start + begin;
  const int gbase = s.atom_start + begin;
  constexpr int SMEM = 2048;
  __shared__ int keys[SMEM];
  if (n <= SMEM) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) keys[k] = slice[k];
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      int key = keys[k], rank = 0;
      for (int m = 0; m < n; ++m) rank += keys[m] < key;
      slice[rank] = key;
      place_sorted(v, s, gbase + rank, key);
    }
  } else {
    // Oversized cell (only in pathological inputs): serial insertion sort by one thread.
    if (threadIdx.x == 0) {
      for (int a = 1; a < n; ++a) {
        int key = slice[a], b = a;
        while (b > 0 && slice[b - 1] > key) {
          slice[b] = slice[b - 1];
          --b;
        }
        slice[b] = key;
      }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) place_sorted(v, s, gbase + k, slice[k]);
  }
}

__device__ __forceinline__ bool is_excluded(const int *__restrict__ start, const int *__restrict__ partners,
                                            int atom, int partner) {
  int lo = start[atom], hi = start[atom + 1];
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    int v = partners[mid];
    if (v == partner) return true;
    if (v < partner) lo = mid + 1; else hi = mid;
  }
  return false;
}

// One warp per atom, atoms visited in cell order: the full neighbour row within the list
// cutoff, in the reference's stencil order. Candidates of a cell are read as one coalesced
// run of the cell-ordered records. With at least three cells per axis every stencil cell
// is reached through one known lattice shift (no per-candidate minimum image) and, in a
// rectangular box, cells entirely beyond the list cutoff are skipped. Membership near the
// cutoff is decided by the exact-rounding test of the reference's WGSL on the original
// coordinates, so rows are bit-identical to the reference's. An entry is the partner's
// cell-ordered slot with the code of the lattice shift to its nearest image.
__global__ void k_neighbours(const float4 *__restrict__ posq, const int *__restrict__ sys_of_atom,
                             const DevSys *__restrict__ sys, const int *__restrict__ cell_start,
                             const int *__restrict__ excl_start, const int *__restrict__ excl_partners,
                             const float4 *__restrict__ spos, const int *__restrict__ sorted_orig,
                             int *__restrict__ nbr, int *__restrict__ nbr_count, int *__restrict__ required,
                             float4 *__restrict__ origin, int n_atoms) {
  const int si = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (si >= n_atoms) return;
  const int i = sorted_orig[si];
  const int sidx = sys_of_atom[i];
  const DevSys &s = sys[sidx];
  const float4 po = posq[i];
  const float4 pw = spos[si];
  if (lane == 0) origin[i] = po;  // displacement origin for the skin check
  const int3 c = cell_coord(make_float3(po.x, po.y, po.z), s);
  const int counts[3] = {s.cell_counts[0], s.cell_counts[1], s.cell_counts[2]};
  int base[3], count[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    base[d] = counts[d] >= 3 ? -1 : 0;
    count[d] = counts[d] >= 3 ? 3 : (counts[d] == 2 ? 2 : 1);
  }
  const bool stencil_shift = counts[0] >= 3 && counts[1] >= 3 && counts[2] >= 3;
  const bool rectangular = s.box[3] == 0.f && s.box[6] == 0.f && s.box[7] == 0.f;
  const float wcell[3] = {s.box[0] / counts[0], s.box[4] / counts[1], s.box[8] / counts[2]};
  const int cc[3] = {c.x, c.y, c.z};
  const float lc2 = s.list_cutoff2;
  const float band_hi = lc2 * 1.00001f, band_lo = lc2 * 0.99999f;
  const int cap = s.nbr_capacity;
  int *row = nbr + s.nbr_base + (long long)(si - s.atom_start) * cap;
  int stored = 0, found = 0;
  const unsigned lt = (1u << lane) - 1u;
  for (int ox = 0; ox < count[0]; ++ox) {
    const int rx = cc[0] + base[0] + ox;
    const int wx = rx < 0 ? -1 : (rx >= counts[0] ? 1 : 0);
    const int cx = rx - wx * counts[0];
    for (int oy = 0; oy < count[1]; ++oy) {
      const int ry = cc[1] + base[1] + oy;
      const int wy = ry < 0 ? -1 : (ry >= counts[1] ? 1 : 0);
      const int cy = ry - wy * counts[1];
      for (int oz = 0; oz < count[2]; ++oz) {
        const int rz = cc[2] + base[2] + oz;
        const int wz = rz < 0 ? -1 : (rz >= counts[2] ? 1 : 0);
        const int cz = rz - wz * counts[2];
        const int cell = (cx * counts[1] + cy) * counts[2] + cz;
        int code = 13;
        float4 S = make_float4(0.f, 0.f, 0.f, 0.f);
        if (stencil_shift) {
          code = shift_code(wx, wy, wz);
          S = s.shift[code];
          if (rectangular) {  // skip a cell whose nearest point is beyond the list cutoff
            const float lo[3] = {rx * wcell[0], ry * wcell[1], rz * wcell[2]};
            const float p[3] = {pw.x, pw.y, pw.z};
            float d2 = 0.f;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              const float e = fmaxf(fmaxf(lo[d] - p[d], p[d] - (lo[d] + wcell[d])), 0.f);
              d2 = fmaf(e, e, d2);
            }
            if (d2 > band_hi * 1.0001f) continue;
          }
        }
        const int begin = s.atom_start + cell_start[s.cell_start_base + cell];
        const int end = s.atom_start + cell_start[s.cell_start_base + cell + 1];
        for (int b = begin; b < end; b += 32) {
          const int g = b + lane;
          bool ok = g < end;
          int j = -1, jcode = code;
          if (ok) {
            j = sorted_orig[g];
            ok = j != i;
          }
          if (ok) {
            const float4 pj = spos[g];
            float3 d = make_float3(pw.x - pj.x - S.x, pw.y - pj.y - S.y, pw.z - pj.z - S.z);
            if (!stencil_shift) {
              const float kc = rintf(d.z * s.inv_diag[2]);
              d.x = fmaf(-kc, s.box[6], d.x); d.y = fmaf(-kc, s.box[7], d.y); d.z = fmaf(-kc, s.box[8], d.z);
              const float kb = rintf(d.y * s.inv_diag[1]);
              d.x = fmaf(-kb, s.box[3], d.x); d.y = fmaf(-kb, s.box[4], d.y);
              const float ka = rintf(d.x * s.inv_diag[0]);
              d.x = fmaf(-ka, s.box[0], d.x);
              jcode = shift_code(max(-1, min(1, (int)ka)), max(-1, min(1, (int)kb)), max(-1, min(1, (int)kc)));
            }
            const float r2 = fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z));
            if (r2 > band_hi) ok = false;
            else if (r2 < band_lo) ok = true;
            else {
              const float4 qj = posq[j];
              const float3 d0 = make_float3(__fsub_rn(po.x, qj.x), __fsub_rn(po.y, qj.y), __fsub_rn(po.z, qj.z));
              ok = !(dot_exact(min_image_exact(d0, s)) > lc2);
            }
          }
          if (ok) ok = !is_excluded(excl_start, excl_partners, i, j);
          const unsigned mask = __ballot_sync(0xffffffffu, ok);
          const int rank = __popc(mask & lt);
          if (ok && stored + rank < cap)
            row[stored + rank] = (int)((unsigned)g | ((unsigned)jcode << NBR_SLOT_BITS));
          const int total = __popc(mask);
          found += total;
          stored = min(cap, stored + total);
        }
      }
    }
  }
  if (lane == 0) {
    nbr_count[si] = stored;
    atomicMax(&required[sidx], found);
  }
}

void launch_rebuild(const LaunchCtx &ctx, cudaStream_t stream) {
  const int n = ctx.n_atoms;
  const int tb = 128;
  k_cells_assign<<<(n + tb - 1) / tb, tb, 0, stream>>>(ctx.posq, ctx.sys_of_atom, ctx.sys,
                                                        ctx.cell_of_atom, ctx.cell_count, n);
  k_cells_scan<<<ctx.n_systems, 1024, 0, stream>>>(ctx.sys, ctx.cell_count, ctx.cell_start);
  k_cells_scatter<<<(n + tb - 1) / tb, tb, 0, stream>>>(ctx.sys_of_atom, ctx.sys, ctx.cell_of_atom,
                                                         ctx.cell_start, ctx.cell_count,
                                                         ctx.cell_atoms, n);
  LaunchCtxView v{ctx.posq, ctx.atom_type, ctx.spos, ctx.wrap, ctx.sorted_orig, ctx.sorted_type, ctx.rank};
  k_cells_sort<<<ctx.n_cells_total, 128, 0, stream>>>(ctx.cell_sys, ctx.sys, ctx.cell_start,
                                                      ctx.cell_count, ctx.cell_atoms, v);
  const int warps_per_block = 4;
  k_neighbours<<<(n + warps_per_block - 1) / warps_per_block, 32 * warps_per_block, 0, stream>>>(
      ctx.posq, ctx.sys_of_atom, ctx.sys, ctx.cell_start, ctx.excl_start, ctx.excl_partners, ctx.spos,
      ctx.sorted_orig, ctx.nbr, ctx.nbr_count, ctx.required, ctx.origin, n);
}

}  // namespace rmd
