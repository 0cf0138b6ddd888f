// Minimiser helpers: the largest per-atom force magnitude of each system and the capped
// displacement along the force (integrate.js:589-666). The maximum, not the norm: one
// clashing pair is what decides whether a structure is safe to start dynamics from.
#include "common.cuh"
#include "kernels.h"

namespace rmd {

__global__ void k_max_force(const unsigned long long *__restrict__ force, const int *__restrict__ sys_of_atom,
                            int n, unsigned *__restrict__ out_bits) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float fx = from_fixed(force[i]), fy = from_fixed(force[n + i]), fz = from_fixed(force[2 * (long long)n + i]);
  atomicMax(out_bits + sys_of_atom[i], __float_as_uint(sqrtf(fx * fx + fy * fy + fz * fz)));
}

__global__ void k_displace(float4 *__restrict__ posq, const unsigned long long *__restrict__ force,
                           const int *__restrict__ sys_of_atom, int n, const float *__restrict__ scale,
                           float max_disp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float s = scale[sys_of_atom[i]];
  if (s == 0.f) return;
  float dx = s * from_fixed(force[i]), dy = s * from_fixed(force[n + i]), dz = s * from_fixed(force[2 * (long long)n + i]);
  const float d = sqrtf(dx * dx + dy * dy + dz * dz);
  if (d > max_disp) {
    const float k = max_disp / d;
    dx *= k;
    dy *= k;
    dz *= k;
  }
  float4 p = posq[i];
  p.x += dx;
  p.y += dy;
  p.z += dz;
  posq[i] = p;
}

void launch_max_force(const unsigned long long *force, const int *sys_of_atom, int n, unsigned *out_bits,
                      cudaStream_t stream) {
  k_max_force<<<(n + 127) / 128, 128, 0, stream>>>(force, sys_of_atom, n, out_bits);
}

void launch_displace(float4 *posq, const unsigned long long *force, const int *sys_of_atom, int n,
                     const float *scale, float max_disp, cudaStream_t stream) {
  k_displace<<<(n + 127) / 128, 128, 0, stream>>>(posq, force, sys_of_atom, n, scale, max_disp);
}

}  // namespace rmd
