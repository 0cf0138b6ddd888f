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

// One block per allocated cell: rank-sort the cell's slice ascending, zero the cursor.
__global__ void k_cells_sort(const int *__restrict__ cell_sys, const DevSys *__restrict__ sys,
                             const int *__restrict__ cell_start, int *__restrict__ cell_cursor,
                             int *__restrict__ cell_atoms) {
  const int g = blockIdx.x;
  const DevSys &s = sys[cell_sys[g]];
  const int c = g - s.cell_base;
  const int cells = s.cell_counts[0] * s.cell_counts[1] * s.cell_counts[2];
  if (c >= cells) return;
  if (threadIdx.x == 0) cell_cursor[g] = 0;
  const int begin = cell_start[s.cell_start_base + c], end = cell_start[s.cell_start_base + c + 1];
  const int n = end - begin;
  if (n <= 1) return;
  int *slice = cell_atoms + s.atom_start + begin;
  constexpr int SMEM = 2048;
  __shared__ int keys[SMEM];
  if (n <= SMEM) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) keys[k] = slice[k];
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      int key = keys[k], rank = 0;
      for (int m = 0; m < n; ++m) rank += keys[m] < key;
      slice[rank] = key;
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

// One warp per atom: the full neighbour row within the list cutoff, in stencil order.
__global__ void k_neighbours(const float4 *__restrict__ posq, const int *__restrict__ sys_of_atom,
                             const DevSys *__restrict__ sys, const int *__restrict__ cell_start,
                             const int *__restrict__ cell_atoms, const int *__restrict__ excl_start,
                             const int *__restrict__ excl_partners, int *__restrict__ nbr,
                             int *__restrict__ nbr_count, int *__restrict__ required,
                             float4 *__restrict__ origin, int n_atoms) {
  const int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp_global >= n_atoms) return;
  const int i = warp_global;
  const int sidx = sys_of_atom[i];
  const DevSys &s = sys[sidx];
  const float4 pi4 = posq[i];
  const float3 pi = make_float3(pi4.x, pi4.y, pi4.z);
  if (lane == 0) origin[i] = pi4;  // displacement origin for the skin check
  const int3 c = cell_coord(pi, s);
  int base[3], count[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int n = s.cell_counts[d];
    base[d] = n >= 3 ? -1 : 0;
    count[d] = n >= 3 ? 3 : (n == 2 ? 2 : 1);
  }
  const int cc[3] = {c.x, c.y, c.z};
  const float lc2 = s.list_cutoff2;
  const int cap = s.nbr_capacity;
  int *row = nbr + s.nbr_base + (long long)(i - s.atom_start) * cap;
  int stored = 0, found = 0;
  const unsigned lt = (1u << lane) - 1u;
  for (int ox = 0; ox < count[0]; ++ox) {
    const int cx = wrap_index(cc[0] + base[0] + ox, s.cell_counts[0]);
    for (int oy = 0; oy < count[1]; ++oy) {
      const int cy = wrap_index(cc[1] + base[1] + oy, s.cell_counts[1]);
      for (int oz = 0; oz < count[2]; ++oz) {
        const int cz = wrap_index(cc[2] + base[2] + oz, s.cell_counts[2]);
        const int cell = (cx * s.cell_counts[1] + cy) * s.cell_counts[2] + cz;
        const int begin = cell_start[s.cell_start_base + cell];
        const int end = cell_start[s.cell_start_base + cell + 1];
        for (int b = begin; b < end; b += 32) {
          const int slot = b + lane;
          bool ok = slot < end;
          int j = ok ? cell_atoms[s.atom_start + slot] : -1;
          ok = ok && j != i;
          if (ok) {
            const float4 pj = posq[j];
            const float3 d0 = make_float3(__fsub_rn(pi.x, pj.x), __fsub_rn(pi.y, pj.y), __fsub_rn(pi.z, pj.z));
            // Cull with the cheap form (reciprocal multiply, rint, FMA); it agrees with the
            // exact-rounding form to a few ulp, so only candidates within a 1e-5 relative band
            // of the list cutoff need the exact test that decides membership.
            const float3 df = min_image(d0, s);
            const float r2f = fmaf(df.x, df.x, fmaf(df.y, df.y, df.z * df.z));
            if (r2f > lc2 * 1.00001f) ok = false;
            else if (r2f < lc2 * 0.99999f) ok = true;
            else ok = !(dot_exact(min_image_exact(d0, s)) > lc2);
          }
          if (ok) ok = !is_excluded(excl_start, excl_partners, i, j);
          const unsigned mask = __ballot_sync(0xffffffffu, ok);
          const int rank = __popc(mask & lt);
          if (ok && stored + rank < cap) row[stored + rank] = j;
          const int total = __popc(mask);
          found += total;
          stored = min(cap, stored + total);
        }
      }
    }
  }
  if (lane == 0) {
    nbr_count[i] = stored;
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
  k_cells_sort<<<ctx.n_cells_total, 128, 0, stream>>>(ctx.cell_sys, ctx.sys, ctx.cell_start,
                                                      ctx.cell_count, ctx.cell_atoms);
  const int warps_per_block = 4;
  k_neighbours<<<(n + warps_per_block - 1) / warps_per_block, 32 * warps_per_block, 0, stream>>>(
      ctx.posq, ctx.sys_of_atom, ctx.sys, ctx.cell_start, ctx.cell_atoms, ctx.excl_start,
      ctx.excl_partners, ctx.nbr, ctx.nbr_count, ctx.required, ctx.origin, n);
}

}  // namespace rmd
