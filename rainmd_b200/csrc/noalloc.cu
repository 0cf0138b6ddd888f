// An allocation-free charge-spreading entry point.
//
// Some callers cannot call cudaMalloc: code that records work into its own CUDA graph
// while the stream is being captured (cudaMalloc is an illegal call under global capture
// mode), hosts that own all device memory through their own arena and forbid runtime
// allocations behind their back, and latency-bound callers for whom cudaMalloc/cudaFree's
// implicit device synchronisation is unacceptable. rmd_spread_charges_noalloc serves them:
// it is the engine's PME charge-spreading kernel (the B-spline spread into a 64-bit
// fixed-point grid, then the conversion to the caller's f64 grid) with its fixed-point
// accumulation grid held in a file-scope device array instead of engine-allocated memory.
// The caller passes device pointers for the input positions and the output grid.
//
// Limits and sharing rules:
//   - the scratch holds at most SCRATCH_POINTS = 64^3 grid points (2 MiB, 256-byte
//     aligned); larger grids are refused with RMD_ERR_INVALID. Every GPU that loads the
//     library holds this array until the process exits;
//   - every call shares the one array and it keeps the last call's contents, so each call
//     clears the part it uses before spreading. Calls that overlap on the GPU (different
//     streams, or different host threads, without ordering between them) race on it;
//   - the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current), loads every kernel this entry point
//     launches (both spline orders and the conversion), and caches the address; that first
//     call should come before any stream capture begins, so that a later call, captured or
//     not, neither resolves a symbol nor loads a module. The cached address belongs to the
//     device's primary context: after cudaDeviceReset on that device it is stale, and the
//     library must not be called on that device again in this process;
//   - an error already pending on the calling thread (an earlier launch that failed) is
//     returned as RMD_ERR_CUDA before anything is launched, so a failure reported by a call
//     is that call's own.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/rmd.h"
#include "common.cuh"

namespace rmd {

constexpr long long SCRATCH_POINTS = 64LL * 64LL * 64LL;
static __device__ __align__(256) unsigned long long g_spread_scratch[SCRATCH_POINTS];

// Same arithmetic, order and fixed-point format as the engine's k_spread (pme.cu):
// fractional coordinates from the rows of the inverse box, wrap with floor, B-spline
// weights of ORDER, grid index (floor(u) + k - ORDER + 1) mod K, one z-row per thread.
template <int ORDER>
__global__ void k_spread_noalloc(const float4 *__restrict__ posq, int n_atoms, DevSys s,
                                 unsigned long long *__restrict__ grid) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(t / (ORDER * ORDER));
  if (i >= n_atoms) return;
  const int kx = (int)(t % (ORDER * ORDER)) / ORDER, ky = (int)(t % ORDER);
  const float4 p = posq[i];
  if (p.w == 0.f) return;
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
  unsigned long long *rowp = grid + ((long long)ix * ny + iy) * nz;
#pragma unroll
  for (int kz = 0; kz < ORDER; ++kz) {
    const int iz = wrap_index(base[2] + kz - ORDER + 1, nz);
    atomicAdd(rowp + iz, to_fixed(wxy * w[2][kz]));
  }
}

__global__ void k_fixed_to_f64(const unsigned long long *__restrict__ grid, double *__restrict__ out,
                               long long points) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < points) out[k] = (double)(long long)grid[k] / FORCE_SCALE;
}

namespace {
constexpr int MAX_DEVICES = 64;
std::mutex g_mutex;
unsigned long long *g_scratch_address[MAX_DEVICES] = {nullptr};
}  // namespace

}  // namespace rmd

extern "C" rmd_status rmd_spread_charges_noalloc(const void *posq, int32_t atom_count,
                                                 const double box_vectors[9], const int32_t grid[3],
                                                 int32_t order, double *grid_out, void *stream) {
  using namespace rmd;
  if (!posq || !grid_out || !box_vectors || !grid || atom_count < 0 || (order != 4 && order != 5))
    return RMD_ERR_INVALID;
  // Bound each size before multiplying, so that no product of the three can overflow and
  // wrap to a small value that would pass the scratch limit (64^3 points).
  long long points = 1;
  for (int d = 0; d < 3; ++d) {
    if (grid[d] < order || grid[d] > SCRATCH_POINTS) return RMD_ERR_INVALID;
    if (points > SCRATCH_POINTS / grid[d]) return RMD_ERR_INVALID;
    points *= grid[d];
  }
  const double ax = box_vectors[0], bx = box_vectors[3], by = box_vectors[4];
  const double cx = box_vectors[6], cy = box_vectors[7], cz = box_vectors[8];
  if (box_vectors[1] != 0.0 || box_vectors[2] != 0.0 || box_vectors[5] != 0.0 || !(ax > 0) || !(by > 0) || !(cz > 0))
    return RMD_ERR_INVALID;  // reduced upper-triangular boxes only, as the engine
  if (cudaPeekAtLastError() != cudaSuccess) return RMD_ERR_CUDA;  // an earlier failure, still pending
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= MAX_DEVICES) return RMD_ERR_CUDA;
  unsigned long long *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_address[device]) {
      void *address = nullptr;
      if (cudaGetSymbolAddress(&address, g_spread_scratch) != cudaSuccess || address == nullptr)
        return RMD_ERR_CUDA;
      // load the three kernels now (lazy module loading would otherwise load each at its
      // first launch, possibly inside a capture)
      cudaFuncAttributes attributes;
      if (cudaFuncGetAttributes(&attributes, k_spread_noalloc<4>) != cudaSuccess ||
          cudaFuncGetAttributes(&attributes, k_spread_noalloc<5>) != cudaSuccess ||
          cudaFuncGetAttributes(&attributes, k_fixed_to_f64) != cudaSuccess)
        return RMD_ERR_CUDA;
      g_scratch_address[device] = static_cast<unsigned long long *>(address);
    }
    scratch = g_scratch_address[device];
  }
  // the box and its inverse rows exactly as the engine forms them (reduce.cu set_box)
  DevSys s;
  memset(&s, 0, sizeof s);
  const double r[9] = {1.0 / ax, 0, 0, -bx / (ax * by), 1.0 / by, 0,
                       (bx * cy - by * cx) / (ax * by * cz), -cy / (by * cz), 1.0 / cz};
  for (int k = 0; k < 9; ++k) {
    s.box[k] = (float)box_vectors[k];
    s.recip[k] = (float)r[k];
  }
  for (int d = 0; d < 3; ++d) s.grid[d] = grid[d];
  s.order = order;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(scratch, 0, sizeof(unsigned long long) * points, st) != cudaSuccess) return RMD_ERR_CUDA;
  const int tb = 128;
  const float4 *p = static_cast<const float4 *>(posq);
  if (atom_count > 0) {
    if (order == 4)
      k_spread_noalloc<4><<<(int)(((long long)atom_count * 16 + tb - 1) / tb), tb, 0, st>>>(p, atom_count, s, scratch);
    else
      k_spread_noalloc<5><<<(int)(((long long)atom_count * 25 + tb - 1) / tb), tb, 0, st>>>(p, atom_count, s, scratch);
  }
  k_fixed_to_f64<<<(int)((points + 255) / 256), 256, 0, st>>>(scratch, grid_out, points);
  return cudaGetLastError() == cudaSuccess ? RMD_OK : RMD_ERR_CUDA;
}
