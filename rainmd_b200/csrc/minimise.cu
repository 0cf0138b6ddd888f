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

// ---------------------------------------------------------------- device line search
// The line search of minimise() (simulation.js:880-979) run as one captured graph per trial:
// max force -> min_begin -> min_save -> displace -> constrain -> forces and energies ->
// min_decide -> min_restore. The host launches the graph in batches and reads the states
// back between batches only to see whether every system has finished.

// One thread per system: open an iteration at the accepted structure (the force test, and
// the copy of the structure for the rollback and for the constraint projection), then set the
// trial's scale so that the largest force moves `step` nm.
__global__ void k_min_begin(MinState *__restrict__ st, const unsigned *__restrict__ worst_bits,
                            float *__restrict__ scale, int S, int max_iterations, float tol) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  MinState m = st[s];
  m.trial = 0;
  m.save = 0;
  m.reject_now = 0;
  float sc = 0.f;
  if (!m.done && !m.overflow) {
    if (!m.open) {
      m.save = 1;  // also when the system stops here: the copy is what later trials restore
      if (m.iterations >= max_iterations) {
        m.done = 1;
      } else {
        m.iterations++;
        m.worst = __uint_as_float(worst_bits[s]);
        if (m.worst <= tol) {
          m.done = 1;
        } else {
          m.open = 1;
          m.attempt = 0;
        }
      }
    }
    if (!m.done) {
      sc = (float)(m.step / fmax((double)m.worst, 1e-6));
      m.trial = 1;
    }
  }
  scale[s] = sc;
  st[s] = m;
}

__global__ void k_min_save(const MinState *__restrict__ st, const float4 *__restrict__ posq,
                           const unsigned long long *__restrict__ force, float4 *__restrict__ saved_posq,
                           unsigned long long *__restrict__ saved_force, const int *__restrict__ sys_of_atom,
                           int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !st[sys_of_atom[i]].save) return;
  saved_posq[i] = posq[i];
  for (int c = 0; c < 3; ++c) saved_force[(long long)c * n + i] = force[(long long)c * n + i];
}

// One thread per system: accept the trial if it lowered the potential (the step grows by
// 1.3), else count a rejection and halve the step; 14 rejections in one iteration, or a step
// below 1e-9, stall the search. A trial whose neighbour list overflowed dropped pairs, so
// its energy decides nothing: it is undone and the system waits for the host to grow the list.
__global__ void k_min_decide(MinState *__restrict__ st, const double *__restrict__ energies,
                             const int *__restrict__ required, const DevSys *__restrict__ sys, int S) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  MinState m = st[s];
  if (!m.trial) return;
  const int req = max(required[s], required[S + s]);  // per-atom rows, group-pair rows
  if (req > sys[s].nbr_capacity) {
    m.overflow = 1;
    m.need = max(m.need, req);
    m.reject_now = 1;
  } else {
    const double trial = energies[(size_t)s * N_ENERGY + E_POTENTIAL];
    if (trial < m.potential) {  // false for a non-finite trial
      m.potential = trial;
      m.step *= 1.3;
      m.open = 0;
    } else {
      m.rejected++;
      m.step *= 0.5;
      m.reject_now = 1;
      m.attempt++;
      if (m.step < 1e-9 || m.attempt >= MIN_ATTEMPTS) {
        m.stalled = 1;
        m.done = 1;
      }
    }
  }
  st[s] = m;
}

// Every system except one whose trial was accepted gets its accepted structure and forces
// back: a rejected trial is undone, and a finished or paused system undoes the constraint
// pass that ran over it.
__global__ void k_min_restore(const MinState *__restrict__ st, float4 *__restrict__ posq,
                              unsigned long long *__restrict__ force, const float4 *__restrict__ saved_posq,
                              const unsigned long long *__restrict__ saved_force,
                              const int *__restrict__ sys_of_atom, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const MinState &m = st[sys_of_atom[i]];
  if (m.trial && !m.reject_now) return;
  posq[i] = saved_posq[i];
  for (int c = 0; c < 3; ++c) force[(long long)c * n + i] = saved_force[(long long)c * n + i];
}

void launch_min_begin(MinState *st, const unsigned *worst_bits, float *scale, int S, int max_iterations,
                      float force_tolerance, cudaStream_t stream) {
  k_min_begin<<<(S + 127) / 128, 128, 0, stream>>>(st, worst_bits, scale, S, max_iterations, force_tolerance);
}

void launch_min_save(const MinState *st, const float4 *posq, const unsigned long long *force, float4 *saved_posq,
                     unsigned long long *saved_force, const int *sys_of_atom, int n, cudaStream_t stream) {
  k_min_save<<<(n + 255) / 256, 256, 0, stream>>>(st, posq, force, saved_posq, saved_force, sys_of_atom, n);
}

void launch_min_decide(MinState *st, const double *energies, const int *required, const DevSys *sys, int S,
                       cudaStream_t stream) {
  k_min_decide<<<(S + 127) / 128, 128, 0, stream>>>(st, energies, required, sys, S);
}

void launch_min_restore(const MinState *st, float4 *posq, unsigned long long *force, const float4 *saved_posq,
                        const unsigned long long *saved_force, const int *sys_of_atom, int n,
                        cudaStream_t stream) {
  k_min_restore<<<(n + 255) / 256, 256, 0, stream>>>(st, posq, force, saved_posq, saved_force, sys_of_atom, n);
}

}  // namespace rmd
