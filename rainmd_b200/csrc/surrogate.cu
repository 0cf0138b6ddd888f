// Learned barostat: an MLP surrogate of a volume move's energy change screens moves as the
// first stage of a two-stage delayed-acceptance Metropolis test, so most moves that the
// exact test would reject never pay for an exact trial-energy evaluation.
//
// The exact move is the reference's Monte Carlo barostat (webgpu/simulation.js:995-1070,
// webgpu/kernels/barostat.js:25-162): a volume change dV drawn uniformly from the adaptive
// window, molecule centroids scaled, and acceptance on
//   w = dU + P dV - N_mol kT ln(V'/V).
// Delayed acceptance (Christen and Fox, J. Comput. Graph. Stat. 14:795, 2005): with a
// surrogate weight w*(x -> y), stage 1 passes the move with probability
//   a1(x -> y) = min(1, exp(-w*(x -> y) / kT))
// and only a passed move gets the exact evaluation; stage 2 accepts it with probability
//   a2 = min(1, exp(-w / kT) a1(y -> x) / a1(x -> y)),
// where a1(y -> x) is the stage-1 probability of the reverse move (from V' back to V) as the
// chain would compute it at y. For any surrogate this satisfies detailed balance with respect
// to the exact NPT distribution, so the surrogate's errors cost acceptance, never correctness.
//
// The surrogate is an approximate target density pi*_x(V') ~ exp(-(F_x(V') + P V')/kT) V'^N_mol
// built around the current state x (Christen and Fox's state-dependent approximation):
//   F_x(V') - F_x(V) = dUdlnV(x) ln(V'/V) + kT sqrt(N_mol) g ln(V'/V)-gated MLP(inputs(x)),
// the first-order term from the virial of the current state (reduce.cu: every term's atomic
// virial, the reciprocal-space sum and the molecular correction) plus a learned correction
// that vanishes at V' = V (the network's output is multiplied by input 0). Inputs (8):
// 100 ln(V'/V), 10 ln(V/V_ref), the kinetic energy over its equipartition value minus 1,
// dU/dlnV over N_mol kT, and the last four exact energy changes over kT sqrt(N_mol); all but
// the first are fixed by the current state and history. Because the approximation depends on
// the state it is built around, a1(y -> x) is not minus the forward weight: it is evaluated
// around the trial state y after the exact evaluation there (k_surrogate_reverse: the
// volume and dU/dlnV of y; the kinetic energy, which a volume move does not change, the
// history and the weights, which only change after the decision, as for the forward move).
// Two tanh layers of 64, one linear
// output. BF16 weights (FP32 biases) with FP32 accumulation in every forward pass; FP32 master
// weights trained by Adam on minibatches of 64 drawn from a per-system replay buffer of
// (inputs, target) pairs that every exact evaluation appends to. Moves before `warm-up` exact
// samples are plain exact moves (they train the network); screening starts after.
//
// Kernels: one block of 256 threads per system. The three 64x64x64 products of a training
// step are shared-memory FMA loops (a step is ~0.8 MFLOP per system, run once per volume
// move, every 25 MD steps).
#include <cuda_bf16.h>

#include <cstdio>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace rmd {

namespace {

constexpr int TPB = 256;
constexpr float ADAM_B1 = 0.9f, ADAM_B2 = 0.999f, ADAM_EPS = 1e-8f;

__device__ __forceinline__ float bf16_bits_to_float(unsigned short b) {
  return __uint_as_float((unsigned)b << 16);
}
__device__ __forceinline__ unsigned short float_to_bf16_bits(float v) {
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  return *reinterpret_cast<const unsigned short *>(&h);
}

// Shared-memory workspace of one block (dynamic shared memory, floats).
struct Work {
  float *x;    // [MLP_BATCH][MLP_IN]
  float *t;    // [MLP_BATCH]
  float *h1;   // [MLP_BATCH][MLP_H]
  float *h2;   // [MLP_BATCH][MLP_H]
  float *d2;   // [MLP_BATCH][MLP_H]
  float *d1;   // [MLP_BATCH][MLP_H]
  float *w1;   // [MLP_H][MLP_IN]   (BF16 values)
  float *w2;   // [MLP_H][MLP_H]    (BF16 values)
  float *w3;   // [MLP_H]           (BF16 values)
  float *bias; // b1[MLP_H], b2[MLP_H], b3
  float *y;    // [MLP_BATCH]
  float *red;  // [TPB / 32]
};
constexpr int WORK_FLOATS = MLP_BATCH * MLP_IN + MLP_BATCH + 4 * MLP_BATCH * MLP_H + MLP_H * MLP_IN +
                            MLP_H * MLP_H + MLP_H + 2 * MLP_H + 1 + MLP_BATCH + TPB / 32 + 7;
constexpr size_t WORK_BYTES = sizeof(float) * WORK_FLOATS;

__device__ Work carve(float *base) {
  Work w;
  float *p = base;
  w.x = p; p += MLP_BATCH * MLP_IN;
  w.t = p; p += MLP_BATCH;
  w.h1 = p; p += MLP_BATCH * MLP_H;
  w.h2 = p; p += MLP_BATCH * MLP_H;
  w.d2 = p; p += MLP_BATCH * MLP_H;
  w.d1 = p; p += MLP_BATCH * MLP_H;
  w.w1 = p; p += MLP_H * MLP_IN;
  w.w2 = p; p += MLP_H * MLP_H;
  w.w3 = p; p += MLP_H;
  w.bias = p; p += 2 * MLP_H + 1;
  w.y = p; p += MLP_BATCH;
  w.red = p;
  return w;
}

// Stage the network in shared memory: weights through BF16 (from `wbf`, or rounded from
// `master` when no BF16 copy is given), biases in FP32.
__device__ void load_network(const Work &w, const float *master, const unsigned short *wbf) {
  for (int k = threadIdx.x; k < MLP_H * MLP_IN; k += blockDim.x)
    w.w1[k] = wbf ? bf16_bits_to_float(wbf[MLP_W1 + k]) : bf16_bits_to_float(float_to_bf16_bits(master[MLP_W1 + k]));
  for (int k = threadIdx.x; k < MLP_H * MLP_H; k += blockDim.x)
    w.w2[k] = wbf ? bf16_bits_to_float(wbf[MLP_W2 + k]) : bf16_bits_to_float(float_to_bf16_bits(master[MLP_W2 + k]));
  for (int k = threadIdx.x; k < MLP_H; k += blockDim.x) {
    w.w3[k] = wbf ? bf16_bits_to_float(wbf[MLP_W3 + k]) : bf16_bits_to_float(float_to_bf16_bits(master[MLP_W3 + k]));
    w.bias[k] = master[MLP_B1 + k];
    w.bias[MLP_H + k] = master[MLP_B2 + k];
  }
  if (threadIdx.x == 0) w.bias[2 * MLP_H] = master[MLP_B3];
}

// Forward pass of `count` (<= MLP_BATCH) samples in w.x: h1, h2 and the outputs y.
__device__ void forward(const Work &w, int count) {
  __syncthreads();
  for (int idx = threadIdx.x; idx < count * MLP_H; idx += blockDim.x) {
    const int b = idx / MLP_H, h = idx % MLP_H;
    float acc = w.bias[h];
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) acc = fmaf(w.w1[h * MLP_IN + k], w.x[b * MLP_IN + k], acc);
    w.h1[idx] = tanhf(acc);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < count * MLP_H; idx += blockDim.x) {
    const int b = idx / MLP_H, h = idx % MLP_H;
    float acc = w.bias[MLP_H + h];
    const float *wr = w.w2 + h * MLP_H, *hr = w.h1 + b * MLP_H;
#pragma unroll 16
    for (int k = 0; k < MLP_H; ++k) acc = fmaf(wr[k], hr[k], acc);
    w.h2[idx] = tanhf(acc);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < count; b += blockDim.x) {
    float acc = w.bias[2 * MLP_H];
    const float *hr = w.h2 + b * MLP_H;
#pragma unroll 16
    for (int h = 0; h < MLP_H; ++h) acc = fmaf(w.w3[h], hr[h], acc);
    w.y[b] = w.x[b * MLP_IN] * acc;  // gated by input 0: zero for a zero volume step
  }
  __syncthreads();
}

// Mean squared error of the forward outputs against w.t, and its gradient with respect to
// every parameter (through the BF16 weights used in the forward pass). Each parameter's
// gradient is produced by one thread and handed to `use(param_index, gradient)`. Returns the
// loss (valid in thread 0).
template <typename Use>
__device__ float backward(const Work &w, int count, Use use) {
  const float inv = 1.0f / (float)count;
  // dL/dy and the loss
  float part = 0.f;
  for (int b = threadIdx.x; b < count; b += blockDim.x) {
    const float e = w.y[b] - w.t[b];
    part += e * e;
  }
  part = warp_sum(part);
  if ((threadIdx.x & 31) == 0) w.red[threadIdx.x >> 5] = part;
  __syncthreads();
  float loss = 0.f;
  if (threadIdx.x == 0) {
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) loss += w.red[k];
    loss *= inv;
  }
  // d2 = dz * w3 * (1 - h2^2), with dz = dL/d(ungated output) = 2 (y - t) x0 / count
  for (int idx = threadIdx.x; idx < count * MLP_H; idx += blockDim.x) {
    const int b = idx / MLP_H, h = idx % MLP_H;
    const float dz = 2.f * (w.y[b] - w.t[b]) * inv * w.x[b * MLP_IN];
    const float a = w.h2[idx];
    w.d2[idx] = dz * w.w3[h] * (1.f - a * a);
  }
  __syncthreads();
  // output layer
  for (int h = threadIdx.x; h <= MLP_H; h += blockDim.x) {
    float g = 0.f;
    for (int b = 0; b < count; ++b) {
      const float dz = 2.f * (w.y[b] - w.t[b]) * inv * w.x[b * MLP_IN];
      g = fmaf(dz, h < MLP_H ? w.h2[b * MLP_H + h] : 1.f, g);
    }
    use(h < MLP_H ? MLP_W3 + h : MLP_B3, g);
  }
  // second layer: gW2[h][k] = sum_b d2[b][h] h1[b][k]; gb2[h] = sum_b d2[b][h]
  for (int idx = threadIdx.x; idx < MLP_H * MLP_H; idx += blockDim.x) {
    const int h = idx / MLP_H, k = idx % MLP_H;
    float g = 0.f;
    for (int b = 0; b < count; ++b) g = fmaf(w.d2[b * MLP_H + h], w.h1[b * MLP_H + k], g);
    use(MLP_W2 + idx, g);
  }
  for (int h = threadIdx.x; h < MLP_H; h += blockDim.x) {
    float g = 0.f;
    for (int b = 0; b < count; ++b) g += w.d2[b * MLP_H + h];
    use(MLP_B2 + h, g);
  }
  // d1[b][k] = (sum_h w2[h][k] d2[b][h]) (1 - h1[b][k]^2)
  for (int idx = threadIdx.x; idx < count * MLP_H; idx += blockDim.x) {
    const int b = idx / MLP_H, k = idx % MLP_H;
    float acc = 0.f;
    const float *dr = w.d2 + b * MLP_H;
#pragma unroll 16
    for (int h = 0; h < MLP_H; ++h) acc = fmaf(w.w2[h * MLP_H + k], dr[h], acc);
    const float a = w.h1[idx];
    w.d1[idx] = acc * (1.f - a * a);
  }
  __syncthreads();
  // first layer
  for (int idx = threadIdx.x; idx < MLP_H * MLP_IN; idx += blockDim.x) {
    const int h = idx / MLP_IN, k = idx % MLP_IN;
    float g = 0.f;
    for (int b = 0; b < count; ++b) g = fmaf(w.d1[b * MLP_H + h], w.x[b * MLP_IN + k], g);
    use(MLP_W1 + idx, g);
  }
  for (int h = threadIdx.x; h < MLP_H; h += blockDim.x) {
    float g = 0.f;
    for (int b = 0; b < count; ++b) g += w.d1[b * MLP_H + h];
    use(MLP_B1 + h, g);
  }
  __syncthreads();
  return loss;
}

// ---------------------------------------------------------------------------- stage 1
// One block per system. Draws the move (the window adapted first, as the exact barostat
// does after every ten attempts), refuses what the exact barostat refuses, evaluates the
// surrogate for the forward and the reverse move and, once screening is on, decides stage 1.
__global__ void __launch_bounds__(TPB) k_surrogate_stage1(BaroArgs a, SurrogateArgs m) {
  extern __shared__ float smem[];
  const int s = blockIdx.x;
  double *b = a.baro + (long long)s * N_BARO;
  if (b[B_ACTIVE] == 0.0 || b[B_LEARNED] == 0.0) return;
  const Work w = carve(smem);
  __shared__ int go;
  __shared__ double dv_s, dlnv_s, nv_s;
  if (threadIdx.x == 0) {
    const DevSysD &d = a.sysd[s];
    const double volume = d.volume;
    b[B_SCREENED] = 0.0;
    b[B_REFUSED] = 0.0;
    b[B_LSCALE] = 1.0;
    if (b[B_SCALE] == 0.0) b[B_SCALE] = 0.01 * volume;
    if (b[B_WINDOW_ATT] >= 10.0) {  // simulation.js:1058-1063
      const double rate = b[B_WINDOW_ACC] / b[B_WINDOW_ATT];
      if (rate < 0.25) b[B_SCALE] /= 1.1;
      else if (rate > 0.75) b[B_SCALE] = fmin(b[B_SCALE] * 1.1, 0.3 * volume);
      b[B_WINDOW_ATT] = 0.0;
      b[B_WINDOW_ACC] = 0.0;
    }
    b[B_ATTEMPTS] += 1.0;
    const bool screening_now = b[B_REPLAY_N] >= b[B_WARMUP];
    if (!screening_now) b[B_WINDOW_ATT] += 1.0;  // while screening, counted when stage 1 passes
    const uint32_t seed = ((uint32_t)b[B_SEED]) ^ 0x5a17u;
    const uint32_t attempt = (uint32_t)b[B_ATTEMPTS];
    const double dv = b[B_SCALE] * 2.0 * (rng_uniform_d(seed, attempt, 0, 0) - 0.5);
    const double nv = volume + dv;
    b[B_DV] = dv;
    go = 1;
    double ls = 1.0;
    if (!(nv > 0)) {
      go = 0;
    } else {
      ls = cbrt(nv / volume);
      const double smallest = ls * fmin(fabs(d.box[0]), fmin(fabs(d.box[4]), fabs(d.box[8])));
      if (d.cutoff > 0.5 * smallest) go = 0;  // simulation.js:1016-1035
    }
    if (!go) {
      b[B_REFUSED] = 1.0;
      b[B_REFUSALS] += 1.0;
    } else {
      b[B_LSCALE] = ls;
      const double kT = b[B_KT], nmol = fmax(b[B_NMOL], 1.0), root = sqrt(nmol);
      const double dlnv = log(nv / volume);
      const double ke = a.energies[s * N_ENERGY + E_KINETIC];
      const double equip = 0.5 * fmax(b[B_DOF], 1.0) * kT;
      const double dudlnv = a.energies[s * N_ENERGY + E_DUDLNV];
      b[B_DUDLNV] = dudlnv;
      // F(V') - F(V) with F anchored at the current state: only input 0 depends on V'
      float *x = w.x;
      x[0] = (float)(100.0 * dlnv);
      x[1] = (float)(10.0 * log(volume / b[B_VOL_REF]));
      x[2] = (float)(ke / equip - 1.0);
      x[3] = (float)(dudlnv / (nmol * kT));
      for (int h = 0; h < 4; ++h) x[4 + h] = (float)(b[B_HIST0 + h] / (kT * root));
      for (int k = 0; k < MLP_IN; ++k) b[B_FEATURE0 + k] = w.x[k];
      b[B_FEATURE0 + 10] = dlnv;
      dv_s = dv;
      dlnv_s = dlnv;
      nv_s = nv;
    }
  }
  __syncthreads();
  if (!go) return;
  load_network(w, m.master + (long long)s * MLP_STRIDE, m.wbf + (long long)s * MLP_STRIDE);
  forward(w, 1);
  if (threadIdx.x == 0) {
    const DevSysD &d = a.sysd[s];
    const double kT = b[B_KT], nmol = fmax(b[B_NMOL], 1.0), root = sqrt(nmol);
    const double volume = d.volume, nv = nv_s, dv = dv_s, dlnv = dlnv_s;
    const double dudlnv = b[B_DUDLNV];
    const double du = dudlnv * dlnv + kT * root * (double)w.y[0];
    const double wf = du + b[B_PRESSURE] * dv - b[B_NMOL] * kT * log(nv / volume);
    b[B_PRED] = wf;
    b[B_PRED_REV] = -wf;  // replaced by k_surrogate_reverse once the trial state has been evaluated
    const bool screening = b[B_REPLAY_N] >= b[B_WARMUP];
    b[B_SCREENING] = screening ? 1.0 : 0.0;
    if (screening) {
      const uint32_t seed = ((uint32_t)b[B_SEED]) ^ 0x5a17u;
      const uint32_t attempt = (uint32_t)b[B_ATTEMPTS];
      const bool pass = wf <= 0.0 || rng_uniform_d(seed, attempt, 2, 0) < exp(-wf / kT);
      if (!pass) {
        b[B_SCREENED] = 1.0;
        b[B_SCREENED_TOTAL] += 1.0;
        b[B_LSCALE] = 1.0;
      } else {
        b[B_WINDOW_ATT] += 1.0;
      }
    }
  }
}

// --------------------------------------------------------------------- reverse move
// One block per system whose move passed stage 1 while screening: the surrogate's weight of
// the reverse move V' -> V around the trial state y, whose energies (dU/dlnV at V') the trial
// evaluation has just reduced; the move's box has not been restored yet (the decision follows).
__global__ void __launch_bounds__(TPB) k_surrogate_reverse(BaroArgs a, SurrogateArgs m) {
  extern __shared__ float smem[];
  const int s = blockIdx.x;
  double *b = a.baro + (long long)s * N_BARO;
  if (b[B_ACTIVE] == 0.0 || b[B_LEARNED] == 0.0 || b[B_SCREENING] == 0.0 || b[B_REFUSED] != 0.0 ||
      b[B_SCREENED] != 0.0)
    return;
  const Work w = carve(smem);
  if (threadIdx.x == 0) {
    const double kT = b[B_KT], nmol = fmax(b[B_NMOL], 1.0);
    const double dlnv = b[B_FEATURE0 + 10];  // ln(V'/V) of the forward move
    const double v_trial = a.sysd[s].volume;
    const double dudlnv = a.energies[s * N_ENERGY + E_DUDLNV];
    float *x = w.x;
    x[0] = (float)(-100.0 * dlnv);
    x[1] = (float)(10.0 * log(v_trial / b[B_VOL_REF]));
    x[2] = (float)b[B_FEATURE0 + 2];
    x[3] = (float)(dudlnv / (nmol * kT));
    for (int h = 0; h < 4; ++h) x[4 + h] = (float)b[B_FEATURE0 + 4 + h];
  }
  __syncthreads();
  load_network(w, m.master + (long long)s * MLP_STRIDE, m.wbf + (long long)s * MLP_STRIDE);
  forward(w, 1);
  if (threadIdx.x == 0) {
    const double kT = b[B_KT], nmol = fmax(b[B_NMOL], 1.0), root = sqrt(nmol);
    const double dlnv = b[B_FEATURE0 + 10];
    const double dudlnv = a.energies[s * N_ENERGY + E_DUDLNV];
    const double du = dudlnv * (-dlnv) + kT * root * (double)w.y[0];
    b[B_PRED_REV] = du - b[B_PRESSURE] * b[B_DV] + b[B_NMOL] * kT * dlnv;
  }
}

// ---------------------------------------------------------------------------- training
// One block per system: append the pending exact sample (if any) to the replay buffer and
// the energy-change history, then take `steps` Adam steps on minibatches from the buffer.
__global__ void __launch_bounds__(TPB) k_surrogate_train(SurrogateArgs m) {
  extern __shared__ float smem[];
  const int s = blockIdx.x;
  double *b = m.baro + (long long)s * N_BARO;
  if (b[B_ACTIVE] == 0.0 || b[B_LEARNED] == 0.0) return;
  const Work w = carve(smem);
  float *master = m.master + (long long)s * MLP_STRIDE;
  float *am = m.adam_m + (long long)s * MLP_STRIDE, *av = m.adam_v + (long long)s * MLP_STRIDE;
  unsigned short *wbf = m.wbf + (long long)s * MLP_STRIDE;
  float *replay = m.replay + (long long)s * MLP_REPLAY * (MLP_IN + 1);
  __shared__ int n_samples;
  __shared__ unsigned step0;
  if (threadIdx.x == 0) {
    const int pending = (int)b[B_FEATURE0 + 9];
    if (pending) {
      const double kT = b[B_KT], root = sqrt(fmax(b[B_NMOL], 1.0));
      const double du = b[B_FEATURE0 + 8];
      const double dlnv = b[B_FEATURE0 + 10];
      const long long n = (long long)b[B_REPLAY_N];
      float *row = replay + (n % MLP_REPLAY) * (MLP_IN + 1);
      for (int k = 0; k < MLP_IN; ++k) row[k] = (float)b[B_FEATURE0 + k];
      row[MLP_IN] = (float)((du - b[B_DUDLNV] * dlnv) / (kT * root));
      b[B_REPLAY_N] = (double)(n + 1);
      // prediction error of the forward weight, in kT (running mean over ~50 moves)
      const double exact_w = b[B_WEIGHT];
      const double err = fabs(b[B_PRED] - exact_w) / kT;
      b[B_PRED_ERR] = b[B_PRED_ERR] == 0.0 ? err : 0.98 * b[B_PRED_ERR] + 0.02 * err;
      for (int h = 3; h > 0; --h) b[B_HIST0 + h] = b[B_HIST0 + h - 1];
      b[B_HIST0] = du;
      b[B_FEATURE0 + 9] = 0.0;
    }
    n_samples = (int)fmin(b[B_REPLAY_N], (double)MLP_REPLAY);
    step0 = (unsigned)b[B_TRAIN_STEPS];
  }
  __syncthreads();
  const int n = n_samples;
  if (n < 8) return;  // too few samples for a minibatch
  const uint32_t seed = ((uint32_t)b[B_SEED]) ^ 0x3c6ef372u;
  float loss_sum = 0.f;
  for (int it = 0; it < m.steps; ++it) {
    const unsigned t = step0 + it + 1;
    for (int idx = threadIdx.x; idx < MLP_BATCH; idx += blockDim.x) {
      int pick = (int)(rng_uniform(seed, t, idx, 0) * (float)n);
      pick = min(pick, n - 1);
      const float *row = replay + (long long)pick * (MLP_IN + 1);
      for (int k = 0; k < MLP_IN; ++k) w.x[idx * MLP_IN + k] = row[k];
      w.t[idx] = row[MLP_IN];
    }
    load_network(w, master, wbf);
    forward(w, MLP_BATCH);
    const float c1 = 1.f - powf(ADAM_B1, (float)t), c2 = 1.f - powf(ADAM_B2, (float)t);
    const float lr = m.lr;
    const float loss = backward(w, MLP_BATCH, [&](int p, float g) {
      const float mm = ADAM_B1 * am[p] + (1.f - ADAM_B1) * g;
      const float vv = ADAM_B2 * av[p] + (1.f - ADAM_B2) * g * g;
      am[p] = mm;
      av[p] = vv;
      const float v = master[p] - lr * (mm / c1) / (sqrtf(vv / c2) + ADAM_EPS);
      master[p] = v;
      wbf[p] = float_to_bf16_bits(v);
    });
    loss_sum += loss;
    __syncthreads();  // the updated weights are read by every thread of the next step
  }
  if (threadIdx.x == 0) {
    b[B_TRAIN_STEPS] += (double)m.steps;
    const double l = loss_sum / m.steps;
    b[B_LOSS] = b[B_LOSS] == 0.0 ? l : 0.95 * b[B_LOSS] + 0.05 * l;
  }
}

// ------------------------------------------------------------------- standalone checks
__global__ void __launch_bounds__(TPB) k_surrogate_eval(const float *params, const float *x, const float *target,
                                                      int count, float *out, float *grads, float *loss) {
  extern __shared__ float smem[];
  const Work w = carve(smem);
  for (int k = threadIdx.x; k < count * MLP_IN; k += blockDim.x) w.x[k] = x[k];
  for (int k = threadIdx.x; k < count; k += blockDim.x) w.t[k] = target ? target[k] : 0.f;
  load_network(w, params, nullptr);
  forward(w, count);
  if (out)
    for (int k = threadIdx.x; k < count; k += blockDim.x) out[k] = w.y[k];
  if (grads) {
    const float l = backward(w, count, [&](int p, float g) { grads[p] = g; });
    if (threadIdx.x == 0) *loss = l;
  }
}

bool g_attr_set[64] = {false};
void set_smem_attr() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !g_attr_set[dev]) {
    cudaFuncSetAttribute(k_surrogate_stage1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WORK_BYTES);
    cudaFuncSetAttribute(k_surrogate_reverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WORK_BYTES);
    cudaFuncSetAttribute(k_surrogate_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WORK_BYTES);
    cudaFuncSetAttribute(k_surrogate_eval, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WORK_BYTES);
    g_attr_set[dev] = true;
  }
}

}  // namespace

void launch_surrogate_stage1(const BaroArgs &a, const SurrogateArgs &m, cudaStream_t stream) {
  set_smem_attr();
  k_surrogate_stage1<<<a.n_systems, TPB, WORK_BYTES, stream>>>(a, m);
}

void launch_surrogate_reverse(const BaroArgs &a, const SurrogateArgs &m, cudaStream_t stream) {
  set_smem_attr();
  k_surrogate_reverse<<<a.n_systems, TPB, WORK_BYTES, stream>>>(a, m);
}

void launch_surrogate_train(const SurrogateArgs &m, cudaStream_t stream) {
  set_smem_attr();
  k_surrogate_train<<<m.n_systems, TPB, WORK_BYTES, stream>>>(m);
}

void surrogate_predict(const float *params, const float *x, int count, float *out, cudaStream_t stream) {
  set_smem_attr();
  k_surrogate_eval<<<1, TPB, WORK_BYTES, stream>>>(params, x, nullptr, count, out, nullptr, nullptr);
}

void surrogate_gradients(const float *params, const float *x, const float *target, int count, float *grads,
                         float *loss, cudaStream_t stream) {
  set_smem_attr();
  k_surrogate_eval<<<1, TPB, WORK_BYTES, stream>>>(params, x, target, count, nullptr, grads, loss);
}

}  // namespace rmd
