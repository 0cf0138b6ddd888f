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
//   - the neighbour search is one WARP per group of 4, 8, 16 or 32 spatially close atoms of a
//     cell: the group's bounding box culls stencil cells and candidates once for all its
//     atoms, the survivors are staged in shared memory, and each atom's lanes append its
//     hits in candidate order, so every row's order equals the sequential one.
#include <climits>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace rmd {

struct LaunchCtxView {
  const float4 *posq;
  const int *atom_type;
  float4 *spos;
  float4 *wrap;
  int *sorted_orig, *sorted_type, *rank;
  int *group_order;
  int2 *slot_info;  // per slot: LJ type, original index (the group-pair kernel's partner record)
  int *order_pos;   // per slot: its position in group_order
  // group-pair rows only (else null): per 4-atom group slot its bounding box (lo, hi) of wrapped
  // positions, and the cell scan's first group per cell
  float4 *group_box;
  const int *cell_gstart;
};

__global__ void k_cells_assign(const float4 *__restrict__ posq, const int *__restrict__ sys_of_atom,
                               const DevSys *__restrict__ sys, int *__restrict__ cell_of_atom,
                               int *__restrict__ cell_count, int n_atoms, const int *__restrict__ only) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_atoms) return;
  if (only && !only[sys_of_atom[i]]) return;
  const DevSys &s = sys[sys_of_atom[i]];
  float4 p = posq[i];
  int3 c = cell_coord(make_float3(p.x, p.y, p.z), s);
  int cell = (c.x * s.cell_counts[1] + c.y) * s.cell_counts[2] + c.z;
  cell_of_atom[i] = cell;
  atomicAdd(&cell_count[s.cell_base + cell], 1);
}

// Block-wide exclusive scan step over one chunk of blockDim.x values; returns the value's
// exclusive prefix within the chunk and leaves the chunk total in *total.
__device__ __forceinline__ int block_exclusive_scan(int v, int *warp_totals, int *total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
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
  const int before = (warp > 0 ? warp_totals[warp - 1] : 0) + x - v;
  *total = warp_totals[warps - 1];
  __syncthreads();
  return before;
}

// One block per system: exclusive scans of the counts into cell_start and of the number
// of neighbour-search groups per cell (ceil(count / group_atoms)) into cell_gstart;
// count -> 0.
__global__ void k_cells_scan(const DevSys *__restrict__ sys, int *__restrict__ cell_count,
                             int *__restrict__ cell_start, int *__restrict__ cell_gstart, int group_atoms,
                             const int *__restrict__ only) {
  if (only && !only[blockIdx.x]) return;
  const DevSys &s = sys[blockIdx.x];
  const int cells = s.cell_counts[0] * s.cell_counts[1] * s.cell_counts[2];
  __shared__ int warp_totals[2][32];
  int running = 0, running_groups = 0;
  for (int chunk = 0; chunk < cells; chunk += blockDim.x) {
    const int c = chunk + threadIdx.x;
    const int v = c < cells ? cell_count[s.cell_base + c] : 0;
    int total, total_groups;
    const int before = block_exclusive_scan(v, warp_totals[0], &total);
    const int before_groups = block_exclusive_scan((v + group_atoms - 1) / group_atoms, warp_totals[1], &total_groups);
    if (c < cells) {
      cell_start[s.cell_start_base + c] = running + before;
      cell_gstart[s.cell_start_base + c] = running_groups + before_groups;
      cell_count[s.cell_base + c] = 0;
    }
    running += total;
    running_groups += total_groups;
  }
  if (threadIdx.x == 0) {
    cell_start[s.cell_start_base + cells] = running;
    cell_gstart[s.cell_start_base + cells] = running_groups;
  }
}

__global__ void k_cells_scatter(const int *__restrict__ sys_of_atom, const DevSys *__restrict__ sys,
                                const int *__restrict__ cell_of_atom, const int *__restrict__ cell_start,
                                int *__restrict__ cell_cursor, int *__restrict__ cell_atoms,
                                int n_atoms, const int *__restrict__ only) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_atoms) return;
  if (only && !only[sys_of_atom[i]]) return;
  const DevSys &s = sys[sys_of_atom[i]];
  int cell = cell_of_atom[i];
  int slot = cell_start[s.cell_start_base + cell] + atomicAdd(&cell_cursor[s.cell_base + cell], 1);
  cell_atoms[s.atom_start + slot] = i;
}

// Index of sub-cell (x, y, z) of a 4x4x4 grid along a 3D Hilbert curve (J. Skilling, "Programming
// the Hilbert curve", AIP Conf. Proc. 707, 381 (2004): axes to transposed index, then the bits
// interleaved): consecutive indices are face-adjacent sub-cells, so consecutive atoms in this
// order stay close (a Z-order curve jumps across the cell between its octants, which made some
// 4-atom search groups a cell wide).
__device__ __forceinline__ int hilbert_key(int x, int y, int z) {
  constexpr int BITS = 2;
  int X[3] = {x, y, z};
#pragma unroll
  for (int q = 1 << (BITS - 1); q > 1; q >>= 1) {
    const int p = q - 1;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (X[i] & q) {
        X[0] ^= p;
      } else {
        const int t = (X[0] ^ X[i]) & p;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  X[1] ^= X[0];
  X[2] ^= X[1];
  int t = 0;
#pragma unroll
  for (int q = 1 << (BITS - 1); q > 1; q >>= 1)
    if (X[2] & q) t ^= q - 1;
  int h = 0;
#pragma unroll
  for (int b = 0; b < BITS; ++b)
#pragma unroll
    for (int i = 0; i < 3; ++i) h |= (((X[i] ^ t) >> b) & 1) << (b * 3 + (2 - i));
  return h;
}

// Write slot g's cell-ordered record for atom j: its position shifted into the box by
// whole box vectors (the shift is kept per atom so the integrator can apply it every step).
// Returns the atom's sub-cell key: the Hilbert index of its position on a 4x4x4 grid inside
// its cell (the order in which the neighbour search groups a cell's atoms).
__device__ __forceinline__ int place_sorted(const LaunchCtxView &v, const DevSys &s, int g, int j,
                                            const int cc[3]) {
  const float4 p = v.posq[j];
  // floor of the same exact-rounding fractional coordinate the cell assignment used, so the
  // wrapped copy lies in (the closure of) the cell the atom was counted in
  float fl[3];
  int sub[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float f = frac_exact(make_float3(p.x, p.y, p.z), s, d);
    fl[d] = floorf(f);
    const float inside = (f - fl[d]) * (float)s.cell_counts[d] - (float)cc[d];
    sub[d] = min(3, max(0, (int)(inside * 4.f)));
  }
  const float wx = fl[0] * s.box[0] + fl[1] * s.box[3] + fl[2] * s.box[6];
  const float wy = fl[0] * s.box[1] + fl[1] * s.box[4] + fl[2] * s.box[7];
  const float wz = fl[0] * s.box[2] + fl[1] * s.box[5] + fl[2] * s.box[8];
  v.spos[g] = make_float4(p.x - wx, p.y - wy, p.z - wz, p.w);
  v.wrap[j] = make_float4(wx, wy, wz, 0.f);
  v.sorted_orig[g] = j;
  v.sorted_type[g] = v.atom_type[j];
  v.slot_info[g] = make_int2(v.atom_type[j], j);
  v.rank[j] = g;
  return hilbert_key(sub[0], sub[1], sub[2]);
}

// One block per allocated cell: rank-sort the cell's slice ascending, zero the cursor, write
// the cell-ordered records of its atoms, and order the cell's slots by sub-cell key (ties by
// slot) into group_order, so that 32 consecutive entries there are spatially compact.
__global__ void k_cells_sort(const int *__restrict__ cell_sys, const DevSys *__restrict__ sys,
                             const int *__restrict__ cell_start, int *__restrict__ cell_cursor,
                             int *__restrict__ cell_atoms, LaunchCtxView v, const int *__restrict__ only) {
  const int g = blockIdx.x;
  if (only && !only[cell_sys[g]]) return;
  const DevSys &s = sys[cell_sys[g]];
  const int c = g - s.cell_base;
  const int cells = s.cell_counts[0] * s.cell_counts[1] * s.cell_counts[2];
  if (c >= cells) return;
  if (threadIdx.x == 0) cell_cursor[g] = 0;
  const int begin = cell_start[s.cell_start_base + c], end = cell_start[s.cell_start_base + c + 1];
  const int n = end - begin;
  if (n <= 0) return;
  const int cc[3] = {c / (s.cell_counts[1] * s.cell_counts[2]), (c / s.cell_counts[2]) % s.cell_counts[1],
                     c % s.cell_counts[2]};
  int *slice = cell_atoms + s.atom_start + begin;
  const int gbase = s.atom_start + begin;
  constexpr int SMEM = 2048;
  __shared__ int keys[SMEM];
  __shared__ int sub_keys[SMEM];
  if (n <= SMEM) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) keys[k] = slice[k];
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      int key = keys[k], rank = 0;
      for (int m = 0; m < n; ++m) rank += keys[m] < key;
      slice[rank] = key;
      sub_keys[rank] = (place_sorted(v, s, gbase + rank, key, cc) << 11) | rank;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      int key = sub_keys[k], rank = 0;
      for (int m = 0; m < n; ++m) rank += sub_keys[m] < key;
      v.group_order[gbase + rank] = gbase + k;
      v.order_pos[gbase + k] = gbase + rank;
    }
  } else {
    // Oversized cell (only in pathological inputs): serial insertion sort by one thread;
    // the groups then follow slot order.
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
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      place_sorted(v, s, gbase + k, slice[k], cc);
      v.group_order[gbase + k] = gbase + k;
      v.order_pos[gbase + k] = gbase + k;
    }
  }
  if (v.group_box) {  // the bounding box of each 4-atom group of this cell, for the search's cull
    __syncthreads();
    const int first_group = s.group_base + v.cell_gstart[s.cell_start_base + c];
    for (int k = threadIdx.x; 4 * k < n; k += blockDim.x) {
      float4 lo = make_float4(INFINITY, INFINITY, INFINITY, 0.f), hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
      for (int a = 4 * k; a < min(n, 4 * k + 4); ++a) {
        const float4 p = v.spos[v.group_order[gbase + a]];
        lo = make_float4(fminf(lo.x, p.x), fminf(lo.y, p.y), fminf(lo.z, p.z), 0.f);
        hi = make_float4(fmaxf(hi.x, p.x), fmaxf(hi.y, p.y), fmaxf(hi.z, p.z), 0.f);
      }
      v.group_box[2 * (first_group + k)] = lo;
      v.group_box[2 * (first_group + k) + 1] = hi;
    }
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

constexpr int NBR_WARPS = 4;        // groups per block when one warp searches for a group
constexpr int NBR_SPLIT = 3;        // warps per group in the split search (one stencil x-slab each)
constexpr int NBR_SPLIT_STAGE = 2048;  // hits a split warp stages in shared memory (G atoms together)
// Launches with fewer groups than this take the split search (4-atom groups): half of what one
// wave holds at 24 resident warps per SM on 148 SMs. Measured on one B200: a 2,854-atom box
// (~800 groups) rebuilds in 0.117 ms split; a 23,558-atom box (~6,000 groups) took 0.315 ms
// split against 0.221 ms with a warp a group.
constexpr int NBR_SPLIT_GROUPS_MAX = 148 * 24 / 2;

// One WARP per search group of G atoms of one cell, taken in sub-cell order so the group is
// spatially compact; lane l works for the group's atom l / J on candidate sub-lane l % J
// (J = 32 / G). The group walks the reference's stencil once for all its atoms: per stencil
// cell (skipped when the cell's box is beyond the list cutoff from the group's bounding
// box), 32 candidates at a time are read as one coalesced run of the cell-ordered records,
// those beyond the list cutoff from the bounding box are dropped, and the survivors are
// staged in shared memory; then each atom's J lanes test J survivors at a time and append
// the hits with a prefix count over those J lanes, so every row keeps the reference's
// order: stencil cell by stencil cell, partners ascending by index within a cell. With at
// least three cells per axis every stencil cell is reached through one known lattice shift
// (no per-candidate minimum image). Membership near the cutoff is decided by the
// exact-rounding test of the reference's WGSL on the original coordinates, so rows are
// bit-identical to the reference's. An entry is the partner's cell-ordered slot with the
// code of the lattice shift to its nearest image.
//
// SPLIT = 3 (4-atom groups in small launches): a block of three warps per group, warp w walking the
// stencil's x-slab w (nine cells) and staging its hits per atom in shared memory; after a
// block barrier each warp copies its hits to the rows behind those of the slabs before it,
// so the rows are the same as one warp's. A group is then three short serial chains instead
// of one long one, which fills the SMs when there are few groups. If a warp's hits overflow its
// staging (512 per atom: a very dense neighbourhood) the first warp walks the whole stencil
// again and writes the rows directly.
template <int G, int SPLIT>
__global__ void __launch_bounds__(SPLIT == 1 ? 32 * NBR_WARPS : 32 * SPLIT)
    k_neighbours(const float4 *__restrict__ posq, const int *__restrict__ group_sys,
                 const DevSys *__restrict__ sys, const int *__restrict__ cell_start,
                 const int *__restrict__ cell_gstart, const int *__restrict__ group_order,
                 const int *__restrict__ excl_start, const int *__restrict__ excl_partners,
                 const float4 *__restrict__ spos, const int *__restrict__ sorted_orig,
                 int *__restrict__ nbr, int *__restrict__ nbr_count, int *__restrict__ required,
                 float4 *__restrict__ origin, int n_groups, const int *__restrict__ only) {
  constexpr int J = 32 / G;
  constexpr int WARPS = SPLIT == 1 ? NBR_WARPS : SPLIT;
  constexpr int HITS = NBR_SPLIT_STAGE / G;  // staged hits per atom per split warp
  __shared__ float4 stage_pos[WARPS][32];
  __shared__ int stage_orig[WARPS][32];
  __shared__ int split_hits[SPLIT == 1 ? 1 : SPLIT * NBR_SPLIT_STAGE];
  __shared__ int split_found[SPLIT][G];
  const int wib = threadIdx.x >> 5;
  const int warp = SPLIT == 1 ? blockIdx.x * NBR_WARPS + wib : blockIdx.x;  // the group
  const int lane = threadIdx.x & 31;
  const int a = lane / J, sub = lane % J;
  // (every exit before the split search's barrier depends on the group alone, so the three
  // warps of a split block leave together)
  if (warp >= n_groups) return;
  const int sidx = group_sys[warp];
  if (only && !only[sidx]) return;  // this system's lists are still valid
  const DevSys &s = sys[sidx];
  const int q = warp - s.group_base;
  const int counts[3] = {s.cell_counts[0], s.cell_counts[1], s.cell_counts[2]};
  const int cells = counts[0] * counts[1] * counts[2];
  const int *gstart = cell_gstart + s.cell_start_base;
  if (q >= gstart[cells]) return;
  // the cell holding group q: gstart[c] <= q < gstart[c + 1]
  int lo = 0, hi = cells;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (gstart[mid] <= q) lo = mid; else hi = mid;
  }
  const int cell0 = lo;
  const int cbegin = s.atom_start + cell_start[s.cell_start_base + cell0];
  const int cend = s.atom_start + cell_start[s.cell_start_base + cell0 + 1];
  const int k = cbegin + (q - gstart[cell0]) * G + a;
  const bool valid = k < cend;
  const int si = valid ? group_order[k] : -1;
  const int i = valid ? sorted_orig[si] : 0;
  const float4 pw = valid ? spos[si] : make_float4(0.f, 0.f, 0.f, 0.f);
  if (valid && sub == 0 && (SPLIT == 1 || wib == 0)) origin[i] = posq[i];  // skin check origin
  // exclusions of this lane's atom: sorted partners; the range check skips the search
  const int e_lo = valid ? excl_start[i] : 0, e_hi = valid ? excl_start[i + 1] : 0;
  const int p_min = e_lo < e_hi ? excl_partners[e_lo] : INT_MAX;
  const int p_max = e_lo < e_hi ? excl_partners[e_hi - 1] : INT_MIN;
  // the group's bounding box (wrapped coordinates)
  float blo[3], bhi[3];
  {
    const float c[3] = {pw.x, pw.y, pw.z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      float lo_d = valid ? c[d] : INFINITY, hi_d = valid ? c[d] : -INFINITY;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        lo_d = fminf(lo_d, __shfl_xor_sync(0xffffffffu, lo_d, o));
        hi_d = fmaxf(hi_d, __shfl_xor_sync(0xffffffffu, hi_d, o));
      }
      blo[d] = lo_d;
      bhi[d] = hi_d;
    }
  }
  const int cc[3] = {cell0 / (counts[1] * counts[2]), (cell0 / counts[2]) % counts[1], cell0 % counts[2]};
  int base[3], count[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    base[d] = counts[d] >= 3 ? -1 : 0;
    count[d] = counts[d] >= 3 ? 3 : (counts[d] == 2 ? 2 : 1);
  }
  const bool stencil_shift = counts[0] >= 3 && counts[1] >= 3 && counts[2] >= 3;
  const bool rectangular = s.box[3] == 0.f && s.box[6] == 0.f && s.box[7] == 0.f;
  const float wcell[3] = {s.box[0] / counts[0], s.box[4] / counts[1], s.box[8] / counts[2]};
  const float lc2 = s.list_cutoff2;
  // the fast test below is within a few 1e-6 of lc2 relative: the band around it goes to the
  // exact test; culling keeps a further margin
  const float band_hi = lc2 * 1.00004f, band_lo = lc2 * 0.99996f, cull2 = band_hi * 1.0001f;
  const int cap = s.nbr_capacity;
  int *row = nbr + s.nbr_base + (long long)(valid ? si - s.atom_start : 0) * cap;
  const unsigned seg_mask = J == 32 ? 0xffffffffu : ((1u << J) - 1u);
  const unsigned below = (1u << sub) - 1u;
  float4 *st_pos = stage_pos[wib];
  int *st_orig = stage_orig[wib];
  // Walk the stencil's x-slabs [ox_begin, ox_end), appending this lane's atom's hits to
  // dst[0 .. dst_cap); returns the atom's hit count (which may exceed dst_cap).
  auto walk = [&](int ox_begin, int ox_end, int *dst, int dst_cap) -> int {
    int found = 0;
    for (int ox = ox_begin; ox < ox_end; ++ox) {
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
            if (rectangular) {  // skip a cell whose box is beyond the list cutoff from the group's
              const float r[3] = {(float)rx, (float)ry, (float)rz};
              float d2 = 0.f;
  #pragma unroll
              for (int d = 0; d < 3; ++d) {
                const float clo = r[d] * wcell[d], chi = clo + wcell[d];
                const float e = fmaxf(fmaxf(clo - bhi[d], blo[d] - chi), 0.f);
                d2 = fmaf(e, e, d2);
              }
              if (d2 > cull2) continue;
            }
          }
          // the bounding box seen from the unshifted copies of this cell's atoms
          const float slo[3] = {blo[0] - S.x, blo[1] - S.y, blo[2] - S.z};
          const float shi[3] = {bhi[0] - S.x, bhi[1] - S.y, bhi[2] - S.z};
          const int begin = s.atom_start + cell_start[s.cell_start_base + cell];
          const int end = s.atom_start + cell_start[s.cell_start_base + cell + 1];
          for (int b = begin; b < end; b += 32) {
            const int g = b + lane;
            bool keep = g < end;
            float4 pj = make_float4(0.f, 0.f, 0.f, 0.f);
            if (keep) {
              pj = spos[g];
              if (stencil_shift) {  // drop candidates beyond the list cutoff from the bounding box
                const float c[3] = {pj.x, pj.y, pj.z};
                float d2 = 0.f;
  #pragma unroll
                for (int d = 0; d < 3; ++d) {
                  const float e = fmaxf(fmaxf(slo[d] - c[d], c[d] - shi[d]), 0.f);
                  d2 = fmaf(e, e, d2);
                }
                keep = d2 <= cull2;
              } else if (rectangular) {
                // fewer than three cells on an axis: every cell is visited and the image is
                // chosen per pair, so the cull measures from the nearest image on each axis
                // (for a rectangular lattice that is the nearest image of the whole box)
                const float c[3] = {pj.x, pj.y, pj.z};
                float d2 = 0.f;
  #pragma unroll
                for (int d = 0; d < 3; ++d) {
                  float x = c[d] - 0.5f * (blo[d] + bhi[d]);
                  x = fmaf(-rintf(x * s.inv_diag[d]), s.box[4 * d], x);
                  const float e = fmaxf(fabsf(x) - 0.5f * (bhi[d] - blo[d]), 0.f);
                  d2 = fmaf(e, e, d2);
                }
                keep = d2 <= cull2;
              }
            }
            const unsigned mask = __ballot_sync(0xffffffffu, keep);
            if (keep) {
              const int at = __popc(mask & ((1u << lane) - 1u));
              st_pos[at] = make_float4(pj.x + S.x, pj.y + S.y, pj.z + S.z, __int_as_float(g));
              st_orig[at] = sorted_orig[g];
            }
            __syncwarp();
            const int survivors = __popc(mask);
            for (int t = 0; t < survivors; t += J) {
              const int tt = t + sub;
              bool in = valid && tt < survivors;
              int entry = 0;
              if (in) {
                const float4 c = st_pos[tt];
                const int j = st_orig[tt];
                const int gj = __float_as_int(c.w);
                float3 d = make_float3(pw.x - c.x, pw.y - c.y, pw.z - c.z);
                int jcode = code;
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
                in = r2 <= band_hi && gj != si;
                if (in && r2 >= band_lo) {  // rare: reload both original positions
                  const float4 po = posq[i], qj = posq[j];
                  const float3 d0 = make_float3(__fsub_rn(po.x, qj.x), __fsub_rn(po.y, qj.y), __fsub_rn(po.z, qj.z));
                  in = !(dot_exact(min_image_exact(d0, s)) > lc2);
                }
                if (in && j >= p_min && j <= p_max) in = !is_excluded(excl_start, excl_partners, i, j);
                entry = (int)((unsigned)gj | ((unsigned)jcode << NBR_SLOT_BITS));
              }
              const unsigned hits = (__ballot_sync(0xffffffffu, in) >> (a * J)) & seg_mask;
              if (in) {
                const int pos = found + __popc(hits & below);
                if (pos < dst_cap) dst[pos] = entry;
              }
              found += __popc(hits);
            }
            __syncwarp();
          }
        }
      }
    }
    return found;
  };
  // One call site of the walk (a loop rather than two calls, so that it is inlined): the
  // one-warp search walks every slab into the rows; a split warp walks its slab into shared
  // memory and, only if some warp's staging overflowed, warp 0 walks again into the rows.
  int *staged = split_hits + (SPLIT == 1 ? 0 : wib * NBR_SPLIT_STAGE);
  int ox_begin = SPLIT == 1 ? 0 : min(wib, count[0]);
  int ox_end = SPLIT == 1 ? count[0] : min(wib + 1, count[0]);
  int *dst = SPLIT == 1 ? row : staged + a * HITS;
  int dst_cap = SPLIT == 1 ? cap : HITS;
  int found = 0;
  for (int pass = 0;; ++pass) {
    found = walk(ox_begin, ox_end, dst, dst_cap);
    if (SPLIT == 1 || pass > 0) break;
    if (sub == 0) split_found[wib][a] = valid ? found : 0;
    __syncthreads();
    bool spill = false;
    found = 0;
#pragma unroll
    for (int w = 0; w < SPLIT; ++w) {
      found += split_found[w][a];
#pragma unroll
      for (int b = 0; b < G; ++b) spill |= split_found[w][b] > HITS;
    }
    if (!spill) {
      // this warp's staged hits of each atom, behind the earlier slabs' hits of that atom
      for (int b = 0; b < G; ++b) {
        const int n = split_found[wib][b];
        const int sb = __shfl_sync(0xffffffffu, si, b * J);
        if (n == 0) continue;  // (also every atom past the end of the cell)
        int off = 0;
        for (int w = 0; w < wib; ++w) off += split_found[w][b];
        int *rb = nbr + s.nbr_base + (long long)(sb - s.atom_start) * cap;
        const int *src = staged + b * HITS;
        for (int k = lane; k < n; k += 32)
          if (off + k < cap) rb[off + k] = src[k];
      }
      break;
    }
    if (wib != 0) break;
    ox_begin = 0;
    ox_end = count[0];
    dst = row;
    dst_cap = cap;
  }
  if (SPLIT > 1 && wib != 0) return;
  if (valid && sub == 0) nbr_count[si] = min(found, cap);
  int most = valid ? found : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) most = max(most, __shfl_xor_sync(0xffffffffu, most, o));
  if (lane == 0) atomicMax(&required[sidx], most);
}

// ---------------------------------------------------------------- group-pair rows
// One WARP per search group of GROUP_ATOMS atoms (the groups of k_neighbours<4, 1>): the
// group's row lists every partner atom that lies within the list cutoff of the group's
// bounding box through some lattice image, once per such image, and only if the pair belongs
// to this group: the partner comes later in search order (order_pos beyond the group), or it
// is one of the group's own atoms, when the entry's mask keeps only the pairs seen from the
// group's earlier atoms. Mask bits also mark the excluded pairs (cells.js:191-227) and the
// atoms past the end of a short group. Every pair within the list cutoff of its two atoms is
// therefore listed exactly once over all rows (the bounding box contains the atom), and an
// atom is never paired with its own image.
//
// With at least three cells on every axis the stencil reaches each cell through one lattice
// shift, as in k_neighbours; otherwise every visited cell is searched through each of the
// lattice images -1, 0, +1 of the axes with fewer than three cells, so that every image of a
// partner within the list cutoff is found.
//
// A block of GROUP_ROW_WARPS warps builds one group's row: the stencil's cells are dealt out to
// the warps in turn, and each warp appends its survivors behind a shared-memory counter, so the
// row is several short serial walks instead of one long one. The order of a row's entries then
// depends on the warps' timing; its contents do not, and neither does any force (every pair's
// fixed-point force is added whatever the order).
constexpr int GROUP_ROW_WARPS = 4;
__global__ void __launch_bounds__(32 * GROUP_ROW_WARPS)
    k_group_rows(const float4 *__restrict__ posq, const int *__restrict__ group_sys,
                 const DevSys *__restrict__ sys, const int *__restrict__ cell_start,
                 const int *__restrict__ cell_gstart, const int *__restrict__ group_order,
                 const int *__restrict__ excl_start, const int *__restrict__ excl_partners,
                 const float4 *__restrict__ spos, const int2 *__restrict__ slot_info,
                 const float4 *__restrict__ group_box, int *__restrict__ gnbr, int *__restrict__ gnbr_count,
                 int *__restrict__ gfirst, int *__restrict__ gsize, int *__restrict__ required,
                 float4 *__restrict__ origin, int n_groups, const int *__restrict__ only) {
  constexpr int G = GROUP_ATOMS;
  __shared__ int row_count;
  __shared__ int survivors[GROUP_ROW_WARPS][32];
  const int warp = blockIdx.x;  // the group slot (every exit before the barriers is the block's)
  const int wib = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n_groups) return;
  const int sidx = group_sys[warp];
  if (only && !only[sidx]) return;  // this system's lists are still valid
  const DevSys &s = sys[sidx];
  const int q = warp - s.group_base;
  const int counts[3] = {s.cell_counts[0], s.cell_counts[1], s.cell_counts[2]};
  const int cells = counts[0] * counts[1] * counts[2];
  const int *gstart = cell_gstart + s.cell_start_base;
  if (q >= gstart[cells]) {  // an unused slot (the cells hold fewer groups than allocated)
    if (threadIdx.x == 0) {
      gsize[warp] = 0;
      gnbr_count[warp] = 0;
    }
    return;
  }
  if (threadIdx.x == 0) row_count = 0;
  __syncthreads();
  int lo = 0, hi = cells;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (gstart[mid] <= q) lo = mid; else hi = mid;
  }
  const int cell0 = lo;
  const int cbegin = s.atom_start + cell_start[s.cell_start_base + cell0];
  const int cend = s.atom_start + cell_start[s.cell_start_base + cell0 + 1];
  const int o0 = cbegin + (q - gstart[cell0]) * G;
  const int size = min(G, cend - o0);
  // every lane holds atom lane % G of the group
  const int a = lane % G;
  const bool valid = a < size;
  const int si = valid ? group_order[o0 + a] : group_order[o0];
  const int i = slot_info[si].y;
  const float4 pw = spos[si];
  if (valid && threadIdx.x < G) origin[i] = posq[i];  // skin check origin
  const int e_lo = valid ? excl_start[i] : 0, e_hi = valid ? excl_start[i + 1] : 0;
  const int p_min = e_lo < e_hi ? excl_partners[e_lo] : INT_MAX;
  const int p_max = e_lo < e_hi ? excl_partners[e_hi - 1] : INT_MIN;
  int atom_i[G], atom_lo[G], atom_hi[G];
#pragma unroll
  for (int b = 0; b < G; ++b) {
    atom_i[b] = __shfl_sync(0xffffffffu, i, b);
    atom_lo[b] = __shfl_sync(0xffffffffu, p_min, b);
    atom_hi[b] = __shfl_sync(0xffffffffu, p_max, b);
  }
  const unsigned absent = 0xFu & ~((1u << size) - 1u);  // atoms past the end of a short group
  // the group's bounding box (wrapped coordinates)
  float blo[3], bhi[3];
  {
    const float c[3] = {pw.x, pw.y, pw.z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      float lo_d = valid ? c[d] : INFINITY, hi_d = valid ? c[d] : -INFINITY;
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) {
        lo_d = fminf(lo_d, __shfl_xor_sync(0xffffffffu, lo_d, o));
        hi_d = fmaxf(hi_d, __shfl_xor_sync(0xffffffffu, hi_d, o));
      }
      blo[d] = lo_d;
      bhi[d] = hi_d;
    }
  }
  const int cc[3] = {cell0 / (counts[1] * counts[2]), (cell0 / counts[2]) % counts[1], cell0 % counts[2]};
  int base[3], count[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    base[d] = counts[d] >= 3 ? -1 : 0;
    count[d] = counts[d] >= 3 ? 3 : (counts[d] == 2 ? 2 : 1);
  }
  const bool stencil_shift = counts[0] >= 3 && counts[1] >= 3 && counts[2] >= 3;
  const bool rectangular = s.box[3] == 0.f && s.box[6] == 0.f && s.box[7] == 0.f;
  const float wcell[3] = {s.box[0] / counts[0], s.box[4] / counts[1], s.box[8] / counts[2]};
  const float cull2 = s.list_cutoff2 * 1.00004f * 1.0001f;  // the margin k_neighbours culls with
  const int cap = s.nbr_capacity;
  int *row = gnbr + s.gnbr_base + (long long)q * cap;
  const int stencil_cells = count[0] * count[1] * count[2];
  // the stencil's cells that need a search are dealt to the warps in turn (a cell before the
  // group's own holds only atoms earlier in search order, whose groups list those pairs; in the
  // shifted stencil of a rectangular box a cell beyond the list cutoff of the group's box is
  // skipped), so the warps of a block get even shares: lane sc decides for stencil cell sc
  // (at most 27), and the needed cells' ranks deal them out
  bool need = false;
  if (lane < stencil_cells) {
    const int ox = lane / (count[1] * count[2]), oy = (lane / count[2]) % count[1], oz = lane % count[2];
    const int rx = cc[0] + base[0] + ox, ry = cc[1] + base[1] + oy, rz = cc[2] + base[2] + oz;
    const int cx = rx - (rx < 0 ? -1 : (rx >= counts[0] ? 1 : 0)) * counts[0];
    const int cy = ry - (ry < 0 ? -1 : (ry >= counts[1] ? 1 : 0)) * counts[1];
    const int cz = rz - (rz < 0 ? -1 : (rz >= counts[2] ? 1 : 0)) * counts[2];
    need = (cx * counts[1] + cy) * counts[2] + cz >= cell0;
    if (need && stencil_shift && rectangular) {
      const float r[3] = {(float)rx, (float)ry, (float)rz};
      float d2 = 0.f;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float clo = r[d] * wcell[d], chi = clo + wcell[d];
        const float e = fmaxf(fmaxf(clo - bhi[d], blo[d] - chi), 0.f);
        d2 = fmaf(e, e, d2);
      }
      need = d2 <= cull2;
    }
  }
  const unsigned need_mask = __ballot_sync(0xffffffffu, need);
  const int rank = __popc(need_mask & ((1u << lane) - 1u));
  for (unsigned mine = __ballot_sync(0xffffffffu, need && rank % GROUP_ROW_WARPS == wib); mine; mine &= mine - 1u) {
    const int sc = __ffs(mine) - 1;
    const int ox = sc / (count[1] * count[2]), oy = (sc / count[2]) % count[1], oz = sc % count[2];
    {
      const int rx = cc[0] + base[0] + ox;
      const int wx = rx < 0 ? -1 : (rx >= counts[0] ? 1 : 0);
      const int cx = rx - wx * counts[0];
      const int ry = cc[1] + base[1] + oy;
      const int wy = ry < 0 ? -1 : (ry >= counts[1] ? 1 : 0);
      const int cy = ry - wy * counts[1];
      {
        const int rz = cc[2] + base[2] + oz;
        const int wz = rz < 0 ? -1 : (rz >= counts[2] ? 1 : 0);
        const int cz = rz - wz * counts[2];
        const int cell = (cx * counts[1] + cy) * counts[2] + cz;
        const int begin = s.atom_start + cell_start[s.cell_start_base + cell];
        const int end = s.atom_start + cell_start[s.cell_start_base + cell + 1];
        // the lattice images to search this cell through: the stencil's own wrap on an axis
        // with three cells or more, each of -1, 0, +1 on the others
        const int na = counts[0] >= 3 ? 1 : 3, nb = counts[1] >= 3 ? 1 : 3, nc = counts[2] >= 3 ? 1 : 3;
        for (int image = 0; image < na * nb * nc; ++image) {
          const int ka = counts[0] >= 3 ? wx : image / (nb * nc) - 1;
          const int kb = counts[1] >= 3 ? wy : (image / nc) % nb - 1;
          const int kc = counts[2] >= 3 ? wz : image % nc - 1;
          const int code = shift_code(ka, kb, kc);
          const float4 S = s.shift[code];
          const float slo[3] = {blo[0] - S.x, blo[1] - S.y, blo[2] - S.z};
          const float shi[3] = {bhi[0] - S.x, bhi[1] - S.y, bhi[2] - S.z};
          // the cell's groups, 32 at a time: a group before this one (its pairs with this group
          // are in its own row) or whose box is beyond the list cutoff of this group's box is
          // dropped whole; the atoms of the others are tested one by one, 8 groups at a time
          const int gs0 = s.group_base + gstart[cell], gs1 = s.group_base + gstart[cell + 1];
          for (int gb = max(gs0, warp); gb < gs1; gb += 32) {
            const int gq = gb + lane;
            bool near = gq < gs1;
            if (near) {
              const float4 lo2 = group_box[2 * gq], hi2 = group_box[2 * gq + 1];
              const float l2[3] = {lo2.x, lo2.y, lo2.z}, h2[3] = {hi2.x, hi2.y, hi2.z};
              float d2 = 0.f;
#pragma unroll
              for (int d = 0; d < 3; ++d) {
                const float e = fmaxf(fmaxf(slo[d] - h2[d], l2[d] - shi[d]), 0.f);
                d2 = fmaf(e, e, d2);
              }
              near = d2 <= cull2;
            }
            const unsigned near_mask = __ballot_sync(0xffffffffu, near);
            if (near) survivors[wib][__popc(near_mask & ((1u << lane) - 1u))] = gq;
            __syncwarp();
            const int n_near = __popc(near_mask);
            for (int t0 = 0; t0 < n_near; t0 += 8) {
              const int t = t0 + (lane >> 2);
              bool keep = t < n_near;
              unsigned mask = 0;
              int g = 0;
              if (keep) {
                const int opos = begin + (survivors[wib][t] - gs0) * G + (lane & 3);
                keep = opos < end;
                if (keep) {
                  g = group_order[opos];
                  const float4 pj = spos[g];
                  const float c[3] = {pj.x, pj.y, pj.z};
                  float d2 = 0.f;
#pragma unroll
                  for (int d = 0; d < 3; ++d) {
                    const float e = fmaxf(fmaxf(slo[d] - c[d], c[d] - shi[d]), 0.f);
                    d2 = fmaf(e, e, d2);
                  }
                  keep = d2 <= cull2;
                }
                if (keep) {
                  // a later group's atom, or one of this group's own: earlier atoms only
                  if (opos < o0 + G) mask = 0xFu & ~((1u << (opos - o0)) - 1u);
                  const int j = slot_info[g].y;
#pragma unroll
                  for (int u = 0; u < G; ++u)
                    if (j >= atom_lo[u] && j <= atom_hi[u] && is_excluded(excl_start, excl_partners, atom_i[u], j))
                      mask |= 1u << u;
                  mask |= absent;
                  keep = mask != 0xFu;
                }
              }
              const unsigned hits = __ballot_sync(0xffffffffu, keep);
              if (hits) {
                int at = 0;
                if (lane == 0) at = atomicAdd(&row_count, __popc(hits));
                at = __shfl_sync(0xffffffffu, at, 0) + __popc(hits & ((1u << lane) - 1u));
                if (keep && at < cap)
                  row[at] = (int)((unsigned)g | ((unsigned)code << GROUP_CODE_SHIFT) | (mask << GROUP_MASK_SHIFT));
              }
            }
            __syncwarp();
          }
        }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int found = row_count;
    gnbr_count[warp] = min(found, cap);
    gfirst[warp] = o0;
    gsize[warp] = size;
    atomicMax(&required[sidx], found);
  }
}

// ---------------------------------------------------------------- rebuild on demand
// A list built with cutoff rc + skin holds every pair that is within rc while no atom has
// moved more than skin / 2 from where it was at the build (two atoms close by at most the sum
// of their displacements). A volume move evaluated on the current lists (reduce.cu) shifts the
// origins with the atoms and adds to `allow` the most it can change a pair distance by, per
// atom, so the test stays a bound. The integrator leaves each system's largest squared displacement
// since the build in disp[s]; this kernel sets the graph's IF condition so that the rebuild
// runs exactly when some system of the batch has passed that bound (with a 0.1% margin on the
// squared distance for the f32 skin), and counts the rebuilds. A non-finite displacement does
// not trigger one: the host's block check reports it.
__global__ void k_rebuild_decide(cudaGraphConditionalHandle handle, const unsigned *__restrict__ disp,
                                 const float *__restrict__ allow, const DevSys *__restrict__ sys, int S,
                                 int *__restrict__ stale, unsigned long long *__restrict__ rebuilds,
                                 ulonglong2 *__restrict__ clear, long long clear_pairs) {
  // the force array the group-pair kernel accumulates into, cleared by the whole grid (the
  // decision itself is block 0's), which saves the step graph a memset node
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < clear_pairs;
       k += (long long)gridDim.x * blockDim.x)
    clear[k] = make_ulonglong2(0ull, 0ull);
  if (blockIdx.x != 0) return;
  int need = 0;
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    const float skin = sys[s].list_cutoff - sys[s].cutoff;
    const float limit2 = 0.25f * skin * skin * 0.999f;
    // the largest displacement since the build, plus what volume moves kept on these lists
    // may have changed a pair distance by (counted per atom)
    const float reach = sqrtf(__uint_as_float(disp[s])) + allow[s];
    const int mine = !(reach * reach <= limit2);
    stale[s] = mine;
    need |= mine;
  }
  need = __syncthreads_or(need);
  if (threadIdx.x == 0) {
    cudaGraphSetConditional(handle, need ? 1u : 0u);
    if (need) *rebuilds += 1;
  }
}

// Start of every rebuild: fold the previous build's requirement (entries of the longest per-atom
// row in required[s], of the longest group-pair row in required[S + s]) into the running
// maximum the host reads after each block (so an overflow at a rebuild inside a block is seen
// too), then clear the requirement and the displacement since the build, and count the build.
__global__ void k_rebuild_reset(int *__restrict__ required, int *__restrict__ required_max,
                                unsigned *__restrict__ disp, float *__restrict__ allow, int *__restrict__ rebuilt,
                                int S, unsigned long long *__restrict__ builds, const int *__restrict__ only) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *builds += 1;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
    if (only && !only[s]) continue;
    required_max[s] = max(required_max[s], max(required[s], required[S + s]));
    required[s] = 0;
    required[S + s] = 0;
    disp[s] = 0u;
    allow[s] = 0.f;
    rebuilt[s] = 1;  // (a volume move clears it, to learn whether its trial rebuilt the lists)
  }
}

void launch_rebuild_decide(cudaGraphConditionalHandle handle, const unsigned *disp, const float *allow,
                           const DevSys *sys, int S, int *stale, unsigned long long *rebuilds,
                           unsigned long long *clear_force, int n_atoms, cudaStream_t stream) {
  // 3 N words of fixed-point force, two a thread (the array is 16-byte aligned and 3 N is
  // rounded up to even in its allocation)
  const long long pairs = clear_force ? (3LL * n_atoms + 1) / 2 : 0;
  const int blocks = (int)std::max(1LL, std::min(1184LL, (pairs + 255) / 256));
  k_rebuild_decide<<<blocks, 256, 0, stream>>>(handle, disp, allow, sys, S, stale, rebuilds,
                                                reinterpret_cast<ulonglong2 *>(clear_force), pairs);
}

void launch_rebuild_reset(int *required, int *required_max, unsigned *disp, float *allow, int *rebuilt, int S,
                          unsigned long long *builds, const int *only, cudaStream_t stream) {
  k_rebuild_reset<<<(S + 255) / 256, 256, 0, stream>>>(required, required_max, disp, allow, rebuilt, S, builds, only);
}

int neighbour_group_slots(int atoms, int cells, int group_atoms) {
  return (atoms + group_atoms - 1) / group_atoms + cells;
}

int rebuild_launches(const LaunchCtx &ctx) { return ctx.pair_list == 2 ? 6 : 5; }

void launch_rebuild(const LaunchCtx &ctx, cudaStream_t stream) {
  const int n = ctx.n_atoms;
  const int tb = 128;
  const int G = ctx.group_atoms;
  const int *only = ctx.rebuild_only;
  k_cells_assign<<<(n + tb - 1) / tb, tb, 0, stream>>>(ctx.posq, ctx.sys_of_atom, ctx.sys,
                                                        ctx.cell_of_atom, ctx.cell_count, n, only);
  k_cells_scan<<<ctx.n_systems, 1024, 0, stream>>>(ctx.sys, ctx.cell_count, ctx.cell_start, ctx.cell_gstart, G,
                                                   only);
  k_cells_scatter<<<(n + tb - 1) / tb, tb, 0, stream>>>(ctx.sys_of_atom, ctx.sys, ctx.cell_of_atom,
                                                         ctx.cell_start, ctx.cell_count,
                                                         ctx.cell_atoms, n, only);
  LaunchCtxView v{ctx.posq,      ctx.atom_type, ctx.spos,      ctx.wrap,      ctx.sorted_orig,
                  ctx.sorted_type, ctx.rank,   ctx.group_order, ctx.slot_info, ctx.order_pos,
                  ctx.pair_list != 1 ? ctx.group_box : nullptr, ctx.cell_gstart};
  k_cells_sort<<<ctx.n_cells_total, 256, 0, stream>>>(ctx.cell_sys, ctx.sys, ctx.cell_start,
                                                      ctx.cell_count, ctx.cell_atoms, v, only);
  const int blocks = (ctx.n_groups_total + NBR_WARPS - 1) / NBR_WARPS;
  if (ctx.pair_list != 1) {  // group-pair rows (the cell scan counted 4-atom groups)
    k_group_rows<<<ctx.n_groups_total, 32 * GROUP_ROW_WARPS, 0, stream>>>(
        ctx.posq, ctx.group_sys, ctx.sys, ctx.cell_start, ctx.cell_gstart, ctx.group_order, ctx.excl_start,
        ctx.excl_partners, ctx.spos, ctx.slot_info, ctx.group_box, ctx.gnbr, ctx.gnbr_count, ctx.gfirst, ctx.gsize,
        ctx.required + ctx.n_systems, ctx.origin, ctx.n_groups_total, only);
    if (ctx.pair_list != 2) return;
  }
#define RMD_NBR_ARGS                                                                                      \
  ctx.posq, ctx.group_sys, ctx.sys, ctx.cell_start, ctx.cell_gstart, ctx.group_order, ctx.excl_start,  \
      ctx.excl_partners, ctx.spos, ctx.sorted_orig, ctx.nbr, ctx.nbr_count, ctx.required, ctx.origin, \
      ctx.n_groups_total, only
  // 4-atom groups too few to fill the GPU with one warp each (a box of a few thousand atoms)
  // search three warps a group; otherwise one warp a group keeps more groups resident
  if (G == 4 && ctx.n_groups_total < NBR_SPLIT_GROUPS_MAX)
    k_neighbours<4, NBR_SPLIT><<<ctx.n_groups_total, 32 * NBR_SPLIT, 0, stream>>>(RMD_NBR_ARGS);
  else if (G == 4)
    k_neighbours<4, 1><<<blocks, 32 * NBR_WARPS, 0, stream>>>(RMD_NBR_ARGS);
  else if (G == 8)
    k_neighbours<8, 1><<<blocks, 32 * NBR_WARPS, 0, stream>>>(RMD_NBR_ARGS);
  else if (G == 16)
    k_neighbours<16, 1><<<blocks, 32 * NBR_WARPS, 0, stream>>>(RMD_NBR_ARGS);
  else
    k_neighbours<32, 1><<<blocks, 32 * NBR_WARPS, 0, stream>>>(RMD_NBR_ARGS);
#undef RMD_NBR_ARGS
}

}  // namespace rmd
