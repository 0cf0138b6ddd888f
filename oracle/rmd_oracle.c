/*
 * CPU oracle for the RainMD per-step MD path — TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker, never the product: only tests/, the smoke check and the
 * bench's CPU-baseline leg load it. It restates RainMD's FP64 host reference, which the
 * reference itself treats as its oracle (cpu/forces/nonbonded.js:1-9, cpu/forces/pme.js:1-15):
 *
 *   erfc (Cody rational Chebyshev)      shared/erf.js:17-107
 *   counter RNG, Box-Muller             shared/random.js:24-87
 *   minimum image, reciprocal box       cpu/forces/geometry.js:27-59
 *   direct space, exceptions            cpu/forces/nonbonded.js:24-162
 *   PME: spread, naive DFT, convolve,
 *        gather, self/net-charge        cpu/forces/pme.js:28-286
 *   B-splines, moduli, alpha, grid      shared/pme/parameters.js:43-252
 *   bonded terms                        cpu/forces/bonded.js:22-207
 *   positional restraint                shared/topology/restraints.js:93-126
 *   dispersion correction               shared/dispersion.js:37-82
 *   SHAKE / RATTLE                      cpu/integrate/constraints.js:93-222
 *   BAOAB Langevin + run loop           cpu/integrate/langevin.js:30-230, cpu/simulation.js:114-156
 *   barostat Metropolis weight          webgpu/kernels/barostat.js:158-162
 *
 * and, for bit-exact comparison of the device's index structures, an f32 restatement of
 * the WGSL cell assignment and neighbour search with the same operation order
 * (webgpu/kernels/wgsl-common.js:81-123, cell-list.js:43-176, neighbours.js:46-151).
 * That part must be compiled without floating-point contraction (-ffp-contract=off).
 *
 * The O(N^2) direct space and the naive per-axis DFT are deliberate: the oracle shares no
 * neighbour list and no FFT with the thing it checks. OpenMP parallelises the pair loop
 * and the DFT lines; per-thread force buffers are reduced in thread order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ONE_4PI_EPS0 138.935456
#define BOLTZMANN 0.008314462618
#define SQRT_PI_INVERSE 5.6418958354775628695e-1

typedef struct {
  int n;
  const double *charges, *masses;
  const int *types;
  int ntypes;
  const double *lj_a, *lj_b;
  int nbonds;
  const int *bond_a, *bond_b;
  const double *bond_k, *bond_r0;
  int nangles;
  const int *angle_a, *angle_b, *angle_c;
  const double *angle_k, *angle_theta0;
  int ntorsions;
  const int *tor_a, *tor_b, *tor_c, *tor_d;
  const double *tor_k, *tor_n, *tor_phase;
  int nexceptions;
  const int *exc_a, *exc_b;
  const double *exc_q, *exc_lja, *exc_ljb;
  int nconstraints;
  const int *con_a, *con_b;
  const double *con_d;
  int nmolecules;
  const int *mol_start, *mol_atoms;
  const double *box; /* 9 doubles, reduced, row-major; NULL when not periodic */
  double cutoff;
  int degrees_of_freedom;
} orc_system;

/* ---------------------------------------------------------------- erfc (shared/erf.js) */
static const double CA[5] = {3.16112374387056560e+00, 1.13864154151050156e+02,
                             3.77485237685302021e+02, 3.20937758913846947e+03,
                             1.85777706184603153e-01};
static const double CB[4] = {2.36012909523441209e+01, 2.44024637934444173e+02,
                             1.28261652607737228e+03, 2.84423683343917062e+03};
static const double CC[9] = {5.64188496988670089e-01, 8.88314979438837594e+00,
                             6.61191906371416295e+01, 2.98635138197400131e+02,
                             8.81952221241769090e+02, 1.71204761263407058e+03,
                             2.05107837782607147e+03, 1.23033935479799725e+03,
                             2.15311535474403846e-08};
static const double CD[8] = {1.57449261107098347e+01, 1.17693950891312499e+02,
                             5.37181101862009858e+02, 1.62138957456669019e+03,
                             3.29079923573345963e+03, 4.36261909014324716e+03,
                             3.43936767414372164e+03, 1.23033935480374942e+03};
static const double CP[6] = {3.05326634961232344e-01, 3.60344899949804439e-01,
                             1.25781726111229246e-01, 1.60837851487422766e-02,
                             6.58749161529837803e-04, 1.63153871373020978e-02};
static const double CQ[5] = {2.56852019228982242e+00, 1.87295284992346047e+00,
                             5.27905102951428412e-01, 6.05183413124413191e-02,
                             2.33520497626869185e-03};

static double scaled_exponential(double y) {
  double z = trunc(y * 16.0) / 16.0;
  double del = (y - z) * (y + z);
  return exp(-z * z) * exp(-del);
}

double orc_erfc(double x) {
  double y = fabs(x), result;
  if (y <= 0.46875) {
    double z = y > 1e-20 ? y * y : 0.0;
    double num = CA[4] * z, den = z;
    for (int i = 0; i < 3; ++i) {
      num = (num + CA[i]) * z;
      den = (den + CB[i]) * z;
    }
    return 1.0 - (x * (num + CA[3])) / (den + CB[3]);
  }
  if (y <= 4.0) {
    double num = CC[8] * y, den = y;
    for (int i = 0; i < 7; ++i) {
      num = (num + CC[i]) * y;
      den = (den + CD[i]) * y;
    }
    result = ((num + CC[7]) / (den + CD[7])) * scaled_exponential(y);
  } else if (y >= 26.543) {
    result = 0.0;
  } else {
    double z = 1.0 / (y * y);
    double num = CP[5] * z, den = z;
    for (int i = 0; i < 4; ++i) {
      num = (num + CP[i]) * z;
      den = (den + CQ[i]) * z;
    }
    result = (z * (num + CP[4])) / (den + CQ[4]);
    result = ((SQRT_PI_INVERSE - result) / y) * scaled_exponential(y);
  }
  return x < 0 ? 2.0 - result : result;
}

double orc_erf(double x) { return 1.0 - orc_erfc(x); }

/* ------------------------------------------------------------ RNG (shared/random.js) */
static uint32_t mix32(uint32_t s) {
  s ^= s >> 16;
  s *= 0x7feb352du;
  s ^= s >> 15;
  s *= 0x846ca68bu;
  s ^= s >> 16;
  return s;
}

double orc_uniform_at(uint32_t seed, uint32_t a, uint32_t b, uint32_t c) {
  uint32_t s = mix32(seed ^ (a * 0x9e3779b1u));
  s = mix32(s ^ (b * 0x85ebca6bu));
  s = mix32(s ^ (c * 0xc2b2ae35u));
  return ((double)(s >> 9) + 0.5) * (1.0 / 8388608.0);
}

void orc_gaussian_triple(double *out, uint32_t seed, uint32_t atom, uint32_t step) {
  double u1 = orc_uniform_at(seed, atom, step, 0), u2 = orc_uniform_at(seed, atom, step, 1);
  double u3 = orc_uniform_at(seed, atom, step, 2), u4 = orc_uniform_at(seed, atom, step, 3);
  double r1 = sqrt(-2.0 * log(u1)), r2 = sqrt(-2.0 * log(u3));
  out[0] = r1 * cos(2.0 * M_PI * u2);
  out[1] = r1 * sin(2.0 * M_PI * u2);
  out[2] = r2 * cos(2.0 * M_PI * u4);
}

/* ------------------------------------------------- geometry (cpu/forces/geometry.js) */
static double js_round(double x) { return floor(x + 0.5); }

static void minimum_image(double *d, const double *box) {
  if (box == NULL) return;
  double s2 = js_round(d[2] / box[8]);
  d[0] -= s2 * box[6];
  d[1] -= s2 * box[7];
  d[2] -= s2 * box[8];
  double s1 = js_round(d[1] / box[4]);
  d[0] -= s1 * box[3];
  d[1] -= s1 * box[4];
  double s0 = js_round(d[0] / box[0]);
  d[0] -= s0 * box[0];
}

void orc_reciprocal_box(const double *b, double *r) {
  double ax = b[0], bx = b[3], by = b[4], cx = b[6], cy = b[7], cz = b[8];
  r[0] = 1.0 / ax; r[1] = 0; r[2] = 0;
  r[3] = -bx / (ax * by); r[4] = 1.0 / by; r[5] = 0;
  r[6] = (bx * cy - by * cx) / (ax * by * cz); r[7] = -cy / (by * cz); r[8] = 1.0 / cz;
}

static int nthreads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_threads(int count) {
#ifdef _OPENMP
  if (count > 0) omp_set_num_threads(count);
#else
  (void)count;
#endif
}

int orc_get_threads(void) { return nthreads(); }

/* ----------------------------------------- exclusions as sorted per-atom partner lists */
typedef struct {
  int *start, *partners;
} excl_csr;

static int cmp_int(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

static excl_csr build_exclusions(const orc_system *s) {
  excl_csr e;
  e.start = (int *)calloc((size_t)s->n + 1, sizeof(int));
  e.partners = (int *)malloc(sizeof(int) * (size_t)(2 * s->nexceptions + 1));
  for (int k = 0; k < s->nexceptions; ++k) {
    e.start[s->exc_a[k] + 1]++;
    e.start[s->exc_b[k] + 1]++;
  }
  for (int i = 0; i < s->n; ++i) e.start[i + 1] += e.start[i];
  int *cursor = (int *)malloc(sizeof(int) * (size_t)(s->n + 1));
  memcpy(cursor, e.start, sizeof(int) * (size_t)(s->n + 1));
  for (int k = 0; k < s->nexceptions; ++k) {
    e.partners[cursor[s->exc_a[k]]++] = s->exc_b[k];
    e.partners[cursor[s->exc_b[k]]++] = s->exc_a[k];
  }
  for (int i = 0; i < s->n; ++i)
    qsort(e.partners + e.start[i], (size_t)(e.start[i + 1] - e.start[i]), sizeof(int), cmp_int);
  free(cursor);
  return e;
}

static int is_excluded(const excl_csr *e, int i, int j) {
  int lo = e->start[i], hi = e->start[i + 1];
  while (lo < hi) {
    int mid = lo + (hi - lo) / 2, v = e->partners[mid];
    if (v == j) return 1;
    if (v < j) lo = mid + 1; else hi = mid;
  }
  return 0;
}

/* ---------------------------------------------------- direct space (nonbonded.js:24) */
/* alpha <= 0 means plain Coulomb; cutoff <= 0 means no cutoff. */
void orc_direct_space(const orc_system *s, const double *pos, double alpha, double cutoff,
                      double *forces, double *lj_out, double *coulomb_out) {
  excl_csr e = build_exclusions(s);
  int threads = nthreads();
  double *fbuf = (double *)calloc((size_t)threads * 3 * s->n, sizeof(double));
  double *ebuf = (double *)calloc((size_t)threads * 2, sizeof(double));
  double cut2 = cutoff > 0 ? cutoff * cutoff : INFINITY;
  const double *box = s->box;
  double two_alpha_over_sqrt_pi = 2.0 * alpha / sqrt(M_PI);
#pragma omp parallel
  {
#ifdef _OPENMP
    int t = omp_get_thread_num();
#else
    int t = 0;
#endif
    double *f = fbuf + (size_t)t * 3 * s->n;
    double lj = 0, coul = 0;
#pragma omp for schedule(dynamic, 16)
    for (int i = 0; i < s->n; ++i) {
      double qi = s->charges[i];
      int row = s->ntypes * s->types[i];
      for (int j = i + 1; j < s->n; ++j) {
        double d[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1],
                       pos[3 * i + 2] - pos[3 * j + 2]};
        minimum_image(d, box);
        double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        if (r2 > cut2) continue;
        if (is_excluded(&e, i, j)) continue;
        double r = sqrt(r2), ir = 1.0 / r, ir2 = ir * ir, ir6 = ir2 * ir2 * ir2;
        int tp = row + s->types[j];
        double a = s->lj_a[tp], b = s->lj_b[tp];
        lj += a * ir6 * ir6 - b * ir6;
        double scalar = (12.0 * a * ir6 * ir6 - 6.0 * b * ir6) * ir2;
        double qq = ONE_4PI_EPS0 * qi * s->charges[j];
        if (alpha <= 0) {
          coul += qq * ir;
          scalar += qq * ir * ir2;
        } else {
          double ar = alpha * r, screened = orc_erfc(ar);
          coul += qq * screened * ir;
          double gaussian = two_alpha_over_sqrt_pi * exp(-ar * ar);
          scalar += qq * (screened * ir + gaussian) * ir2;
        }
        for (int c = 0; c < 3; ++c) {
          f[3 * i + c] += scalar * d[c];
          f[3 * j + c] -= scalar * d[c];
        }
      }
    }
    ebuf[2 * t] = lj;
    ebuf[2 * t + 1] = coul;
  }
  double lj = 0, coul = 0;
  for (int t = 0; t < threads; ++t) {
    lj += ebuf[2 * t];
    coul += ebuf[2 * t + 1];
    for (int k = 0; k < 3 * s->n; ++k) forces[k] += fbuf[(size_t)t * 3 * s->n + k];
  }
  *lj_out = lj;
  *coulomb_out = coul;
  free(fbuf);
  free(ebuf);
  free(e.start);
  free(e.partners);
}

/* ------------------------------------------------------ exceptions (nonbonded.js:106) */
void orc_exceptions(const orc_system *s, const double *pos, double alpha, double *forces,
                    double *lj_out, double *coulomb_out) {
  double lj = 0, coul = 0;
  for (int k = 0; k < s->nexceptions; ++k) {
    int i = s->exc_a[k], j = s->exc_b[k];
    double d[3] = {pos[3 * i] - pos[3 * j], pos[3 * i + 1] - pos[3 * j + 1],
                   pos[3 * i + 2] - pos[3 * j + 2]};
    minimum_image(d, s->box);
    double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    double r = sqrt(r2), ir = 1.0 / r, ir2 = ir * ir, ir6 = ir2 * ir2 * ir2;
    double scalar = 0;
    double a = s->exc_lja[k], b = s->exc_ljb[k];
    if (a != 0 || b != 0) {
      lj += a * ir6 * ir6 - b * ir6;
      scalar += (12.0 * a * ir6 * ir6 - 6.0 * b * ir6) * ir2;
    }
    double sp = s->exc_q[k];
    if (sp != 0) {
      double qq = ONE_4PI_EPS0 * sp;
      coul += qq * ir;
      scalar += qq * ir * ir2;
    }
    if (alpha > 0) {
      double qf = ONE_4PI_EPS0 * s->charges[i] * s->charges[j];
      if (qf != 0) {
        double ar = alpha * r, un = orc_erf(ar);
        coul -= qf * un * ir;
        double gaussian = 2.0 * alpha * exp(-ar * ar) / sqrt(M_PI);
        scalar -= qf * (un * ir - gaussian) * ir2;
      }
    }
    for (int c = 0; c < 3; ++c) {
      forces[3 * i + c] += scalar * d[c];
      forces[3 * j + c] -= scalar * d[c];
    }
  }
  *lj_out = lj;
  *coulomb_out = coul;
}

/* -------------------------------------------- PME parameters (shared/pme/parameters.js) */
double orc_alpha_from_tolerance(double cutoff, double tolerance) {
  return sqrt(-log(2.0 * tolerance)) / cutoff;
}

static int transformable(int v) {
  int r = v;
  while (r % 2 == 0) r /= 2;
  while (r % 3 == 0) r /= 3;
  while (r % 5 == 0) r /= 5;
  return r == 1;
}

void orc_grid_size_for(const double *box, double alpha, double tolerance, int *grid) {
  double denom = 3.0 * pow(tolerance, 0.2);
  for (int d = 0; d < 3; ++d) {
    double len = sqrt(box[3 * d] * box[3 * d] + box[3 * d + 1] * box[3 * d + 1] +
                      box[3 * d + 2] * box[3 * d + 2]);
    int c = (int)ceil(2.0 * alpha * len / denom);
    if (c < 2) c = 2;
    while (!transformable(c)) ++c;
    grid[d] = c;
  }
}

/* de Boor recursion; the derivative is read at order-1 (parameters.js:121-149). */
void orc_bspline(double offset, int order, double *w, double *dw) {
  for (int k = 0; k < order; ++k) w[k] = 0;
  w[0] = 1.0 - offset;
  w[1] = offset;
  for (int k = 3; k < order; ++k) {
    double div = 1.0 / (k - 1);
    w[k - 1] = div * offset * w[k - 2];
    for (int j = 1; j < k - 1; ++j)
      w[k - j - 1] = div * ((offset + j) * w[k - j - 2] + (k - j - offset) * w[k - j - 1]);
    w[0] = div * (1.0 - offset) * w[0];
  }
  dw[0] = -w[0];
  for (int j = 1; j < order; ++j) dw[j] = w[j - 1] - w[j];
  double div = 1.0 / (order - 1);
  w[order - 1] = div * offset * w[order - 2];
  for (int j = 1; j < order - 1; ++j)
    w[order - j - 1] =
        div * ((offset + j) * w[order - j - 2] + (order - j - offset) * w[order - j - 1]);
  w[0] = div * (1.0 - offset) * w[0];
}

/* |b(m)|^2 as the explicit DFT of integer-point spline values, patched where < 1e-7. */
int orc_bspline_moduli(int size, int order, double *out) {
  double w[16], dw[16];
  orc_bspline(0.0, order, w, dw);
  double *raw = (double *)malloc(sizeof(double) * (size_t)size);
  for (int m = 0; m < size; ++m) {
    double re = 0, im = 0;
    for (int k = 0; k < order; ++k) {
      double ang = 2.0 * M_PI * m * k / size;
      re += w[k] * cos(ang);
      im += w[k] * sin(ang);
    }
    raw[m] = re * re + im * im;
  }
  int ok = 1;
  for (int m = 0; m < size; ++m) {
    out[m] = raw[m] < 1e-7 ? 0.5 * (raw[(m - 1 + size) % size] + raw[(m + 1) % size]) : raw[m];
    if (!(out[m] > 0)) ok = 0;
  }
  free(raw);
  return ok;
}

/* ------------------------------------------------------------------ naive DFT (pme.js:28) */
void orc_dft_axis(double *data, const int *grid, int axis, int sign) {
  int nx = grid[0], ny = grid[1], nz = grid[2];
  int n = grid[axis];
  int strides[3] = {ny * nz, nz, 1};
  int stride = strides[axis];
  double *ct = (double *)malloc(sizeof(double) * (size_t)n);
  double *st = (double *)malloc(sizeof(double) * (size_t)n);
  for (int k = 0; k < n; ++k) {
    double ang = sign * 2.0 * M_PI * k / n;
    ct[k] = cos(ang);
    st[k] = sin(ang);
  }
  int outer[3] = {nx, ny, nz};
  outer[axis] = 1;
  int lines = outer[0] * outer[1] * outer[2];
#pragma omp parallel
  {
    double *line = (double *)malloc(sizeof(double) * 2 * (size_t)n);
#pragma omp for schedule(static)
    for (int l = 0; l < lines; ++l) {
      int x = l / (outer[1] * outer[2]), y = (l / outer[2]) % outer[1], z = l % outer[2];
      int base = x * strides[0] + y * strides[1] + z * strides[2];
      for (int k = 0; k < n; ++k) {
        line[2 * k] = data[2 * (base + k * stride)];
        line[2 * k + 1] = data[2 * (base + k * stride) + 1];
      }
      for (int m = 0; m < n; ++m) {
        double re = 0, im = 0;
        for (int k = 0; k < n; ++k) {
          int t = (int)(((long)m * k) % n);
          re += line[2 * k] * ct[t] - line[2 * k + 1] * st[t];
          im += line[2 * k] * st[t] + line[2 * k + 1] * ct[t];
        }
        data[2 * (base + m * stride)] = re;
        data[2 * (base + m * stride) + 1] = im;
      }
    }
    free(line);
  }
  free(ct);
  free(st);
}

static int wrapi(int v, int n) {
  int r = v % n;
  return r < 0 ? r + n : r;
}

/* Reciprocal energy and forces (pme.js:76-259). `charge_grid_out`, when not NULL,
 * receives the real spread grid (nx*ny*nz, z fastest) before the transform. */
double orc_reciprocal(const orc_system *s, const double *pos, double alpha, const int *grid,
                      int order, double *forces, double *charge_grid_out) {
  int nx = grid[0], ny = grid[1], nz = grid[2];
  size_t points = (size_t)nx * ny * nz;
  double recip[9];
  orc_reciprocal_box(s->box, recip);
  double volume = s->box[0] * s->box[4] * s->box[8];
  double *q = (double *)calloc(2 * points, sizeof(double));
  int *base = (int *)malloc(sizeof(int) * 3 * (size_t)s->n);
  double *w = (double *)malloc(sizeof(double) * 3 * (size_t)order * s->n);
  double *dw = (double *)malloc(sizeof(double) * 3 * (size_t)order * s->n);
  for (int a = 0; a < s->n; ++a) {
    double r[3] = {pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]};
    for (int d = 0; d < 3; ++d) {
      double f = r[0] * recip[d] + r[1] * recip[3 + d] + r[2] * recip[6 + d];
      double wrapped = f - floor(f);
      double scaled = wrapped * grid[d];
      double integral = floor(scaled);
      base[3 * a + d] = (int)integral;
      orc_bspline(scaled - integral, order, w + (3 * a + d) * order, dw + (3 * a + d) * order);
    }
    double qa = s->charges[a];
    for (int kx = 0; kx < order; ++kx) {
      int ix = wrapi(base[3 * a] + kx - order + 1, nx);
      double wx = w[(3 * a) * order + kx];
      for (int ky = 0; ky < order; ++ky) {
        int iy = wrapi(base[3 * a + 1] + ky - order + 1, ny);
        double wxy = wx * w[(3 * a + 1) * order + ky];
        for (int kz = 0; kz < order; ++kz) {
          int iz = wrapi(base[3 * a + 2] + kz - order + 1, nz);
          q[2 * (((size_t)ix * ny + iy) * nz + iz)] += qa * wxy * w[(3 * a + 2) * order + kz];
        }
      }
    }
  }
  if (charge_grid_out != NULL)
    for (size_t p = 0; p < points; ++p) charge_grid_out[p] = q[2 * p];
  orc_dft_axis(q, grid, 0, 1);
  orc_dft_axis(q, grid, 1, 1);
  orc_dft_axis(q, grid, 2, 1);
  double *mod[3];
  for (int d = 0; d < 3; ++d) {
    mod[d] = (double *)malloc(sizeof(double) * (size_t)grid[d]);
    orc_bspline_moduli(grid[d], order, mod[d]);
  }
  double factor = M_PI * M_PI / (alpha * alpha);
  double prefactor = ONE_4PI_EPS0 / (2.0 * M_PI * volume);
  double energy = 0;
  for (int mx = 0; mx < nx; ++mx) {
    int kx = mx <= nx / 2 ? mx : mx - nx;
    for (int my = 0; my < ny; ++my) {
      int ky = my <= ny / 2 ? my : my - ny;
      for (int mz = 0; mz < nz; ++mz) {
        int kz = mz <= nz / 2 ? mz : mz - nz;
        size_t idx = ((size_t)mx * ny + my) * nz + mz;
        if (kx == 0 && ky == 0 && kz == 0) {
          q[2 * idx] = q[2 * idx + 1] = 0;
          continue;
        }
        double mxc = kx * recip[0] + ky * recip[1] + kz * recip[2];
        double myc = kx * recip[3] + ky * recip[4] + kz * recip[5];
        double mzc = kx * recip[6] + ky * recip[7] + kz * recip[8];
        double m2 = mxc * mxc + myc * myc + mzc * mzc;
        double kernel = exp(-factor * m2) / (m2 * mod[0][mx] * mod[1][my] * mod[2][mz]);
        double re = q[2 * idx], im = q[2 * idx + 1];
        energy += prefactor * kernel * (re * re + im * im);
        q[2 * idx] = re * kernel * 2.0 * prefactor;
        q[2 * idx + 1] = im * kernel * 2.0 * prefactor;
      }
    }
  }
  orc_dft_axis(q, grid, 0, -1);
  orc_dft_axis(q, grid, 1, -1);
  orc_dft_axis(q, grid, 2, -1);
  for (int a = 0; a < s->n; ++a) {
    double qa = s->charges[a];
    if (qa == 0) continue;
    double gu = 0, gv = 0, gw = 0;
    for (int kx = 0; kx < order; ++kx) {
      int ix = wrapi(base[3 * a] + kx - order + 1, nx);
      double wx = w[(3 * a) * order + kx], dx = dw[(3 * a) * order + kx];
      for (int ky = 0; ky < order; ++ky) {
        int iy = wrapi(base[3 * a + 1] + ky - order + 1, ny);
        double wy = w[(3 * a + 1) * order + ky], dy = dw[(3 * a + 1) * order + ky];
        for (int kz = 0; kz < order; ++kz) {
          int iz = wrapi(base[3 * a + 2] + kz - order + 1, nz);
          double wz = w[(3 * a + 2) * order + kz], dz = dw[(3 * a + 2) * order + kz];
          double v = q[2 * (((size_t)ix * ny + iy) * nz + iz)];
          gu += dx * wy * wz * v;
          gv += wx * dy * wz * v;
          gw += wx * wy * dz * v;
        }
      }
    }
    gu *= grid[0] * qa;
    gv *= grid[1] * qa;
    gw *= grid[2] * qa;
    forces[3 * a] -= gu * recip[0] + gv * recip[1] + gw * recip[2];
    forces[3 * a + 1] -= gu * recip[3] + gv * recip[4] + gw * recip[5];
    forces[3 * a + 2] -= gu * recip[6] + gv * recip[7] + gw * recip[8];
  }
  for (int d = 0; d < 3; ++d) free(mod[d]);
  free(q);
  free(base);
  free(w);
  free(dw);
  return energy;
}

/* Self and net-charge terms (pme.js:270-286): out[0] = self, out[1] = net. */
void orc_ewald_self(const orc_system *s, double alpha, double *out) {
  double q2 = 0, qs = 0;
  for (int a = 0; a < s->n; ++a) {
    q2 += s->charges[a] * s->charges[a];
    qs += s->charges[a];
  }
  double volume = s->box[0] * s->box[4] * s->box[8];
  out[0] = -ONE_4PI_EPS0 * alpha * q2 / sqrt(M_PI);
  out[1] = -ONE_4PI_EPS0 * M_PI * qs * qs / (2.0 * alpha * alpha * volume);
}

/* --------------------------------------------------------- dispersion (dispersion.js) */
void orc_dispersion_coefficients(const orc_system *s, double *ab) {
  int T = s->ntypes;
  double *counts = (double *)calloc((size_t)T, sizeof(double));
  for (int a = 0; a < s->n; ++a) counts[s->types[a]] += 1;
  double oa = 0, ob = 0, da = 0, db = 0;
  for (int i = 0; i < T; ++i) {
    for (int j = 0; j < T; ++j) {
      oa += counts[i] * counts[j] * s->lj_a[T * i + j];
      ob += counts[i] * counts[j] * s->lj_b[T * i + j];
    }
    da += counts[i] * s->lj_a[T * i + i];
    db += counts[i] * s->lj_b[T * i + i];
  }
  double scale = (double)s->n / (s->n + 1);
  ab[0] = (oa + da) * scale;
  ab[1] = (ob + db) * scale;
  free(counts);
}

double orc_dispersion_energy(const double *ab, double volume, double cutoff) {
  if (!(volume > 0) || !(cutoff > 0)) return 0;
  double c3 = cutoff * cutoff * cutoff, c9 = c3 * c3 * c3;
  return (2.0 * M_PI / volume) * (ab[0] / (9.0 * c9) - ab[1] / (3.0 * c3));
}

/* ------------------------------------------------------------ bonded (bonded.js) */
static void cross3(const double *a, const double *b, double *o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

double orc_bonds(const orc_system *s, const double *p, double *f) {
  double e = 0;
  for (int k = 0; k < s->nbonds; ++k) {
    int a = 3 * s->bond_a[k], b = 3 * s->bond_b[k];
    double d[3] = {p[a] - p[b], p[a + 1] - p[b + 1], p[a + 2] - p[b + 2]};
    double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double st = r - s->bond_r0[k];
    e += 0.5 * s->bond_k[k] * st * st;
    double sc = r > 0 ? s->bond_k[k] * st / r : 0;
    for (int c = 0; c < 3; ++c) {
      f[a + c] -= sc * d[c];
      f[b + c] += sc * d[c];
    }
  }
  return e;
}

double orc_angles(const orc_system *s, const double *p, double *f) {
  double e = 0;
  for (int k = 0; k < s->nangles; ++k) {
    int a = 3 * s->angle_a[k], b = 3 * s->angle_b[k], c = 3 * s->angle_c[k];
    double v1[3] = {p[a] - p[b], p[a + 1] - p[b + 1], p[a + 2] - p[b + 2]};
    double v2[3] = {p[c] - p[b], p[c + 1] - p[b + 1], p[c + 2] - p[b + 2]};
    double n1 = v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2];
    double n2 = v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2];
    double nm[3];
    cross3(v1, v2, nm);
    double cm = sqrt(nm[0] * nm[0] + nm[1] * nm[1] + nm[2] * nm[2]);
    double dot = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
    double theta = atan2(cm, dot), dev = theta - s->angle_theta0[k];
    e += 0.5 * s->angle_k[k] * dev * dev;
    double dE = s->angle_k[k] * dev, safe = cm > 1e-12 ? cm : 1e-12;
    double s1 = -dE / (n1 * safe), s2 = dE / (n2 * safe);
    double fa[3], fc[3], t1[3], t2[3];
    cross3(v1, nm, t1);
    cross3(v2, nm, t2);
    for (int q = 0; q < 3; ++q) {
      fa[q] = s1 * t1[q];
      fc[q] = s2 * t2[q];
      f[a + q] += fa[q];
      f[c + q] += fc[q];
      f[b + q] -= fa[q] + fc[q];
    }
  }
  return e;
}

double orc_torsions(const orc_system *s, const double *p, double *f) {
  double e = 0;
  for (int k = 0; k < s->ntorsions; ++k) {
    int a = 3 * s->tor_a[k], b = 3 * s->tor_b[k], c = 3 * s->tor_c[k], d = 3 * s->tor_d[k];
    double b1[3], b2[3], b3[3], n1[3], n2[3];
    for (int q = 0; q < 3; ++q) {
      b1[q] = p[b + q] - p[a + q];
      b2[q] = p[c + q] - p[b + q];
      b3[q] = p[d + q] - p[c + q];
    }
    cross3(b1, b2, n1);
    cross3(b2, b3, n2);
    double n1s = n1[0] * n1[0] + n1[1] * n1[1] + n1[2] * n1[2];
    double n2s = n2[0] * n2[0] + n2[1] * n2[1] + n2[2] * n2[2];
    double b2l = sqrt(b2[0] * b2[0] + b2[1] * b2[1] + b2[2] * b2[2]);
    if (n1s < 1e-24 || n2s < 1e-24 || b2l < 1e-12) continue;
    double dn = n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2];
    double cn[3];
    cross3(n1, n2, cn);
    double cdb = cn[0] * b2[0] + cn[1] * b2[1] + cn[2] * b2[2];
    double phi = atan2(cdb / b2l, dn);
    double n = s->tor_n[k], arg = n * phi - s->tor_phase[k];
    e += s->tor_k[k] * (1.0 + cos(arg));
    double dEdphi = -s->tor_k[k] * n * sin(arg);
    double fA = dEdphi * b2l / n1s, fD = -dEdphi * b2l / n2s;
    double inv = 1.0 / (b2l * b2l);
    double t = (b1[0] * b2[0] + b1[1] * b2[1] + b1[2] * b2[2]) * inv;
    double u = (b3[0] * b2[0] + b3[1] * b2[1] + b3[2] * b2[2]) * inv;
    for (int q = 0; q < 3; ++q) {
      double fa = fA * n1[q], fd = fD * n2[q];
      f[a + q] += fa;
      f[d + q] += fd;
      f[b + q] += -(1.0 + t) * fa + u * fd;
      f[c + q] += t * fa - (1.0 + u) * fd;
    }
  }
  return e;
}

/* k*d^2 with the minimum image against an absolute reference (restraints.js:93-126). */
double orc_restraint(const orc_system *s, int count, const int *atoms, const double *reference,
                     double k, const double *p, double *f) {
  if (k <= 0 || count == 0) return 0;
  double total = 0;
  for (int slot = 0; slot < count; ++slot) {
    int a = atoms[slot];
    double d[3] = {p[3 * a] - reference[3 * slot], p[3 * a + 1] - reference[3 * slot + 1],
                   p[3 * a + 2] - reference[3 * slot + 2]};
    minimum_image(d, s->box);
    total += k * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    for (int c = 0; c < 3; ++c) f[3 * a + c] -= 2.0 * k * d[c];
  }
  return total;
}

/* ------------------------------------------------ whole potential (cpu/energy.js:25-91) */
/* terms: [0] bond [1] angle [2] torsion [3] lennardJones [4] coulombDirect
 *        [5] coulombReciprocal [6] coulombSelf [7] coulombNetCharge [8] restraint [9] total
 * method 0 = NoCutoff, 1 = PME (alpha, grid and order given). forces are overwritten. */
void orc_potential(const orc_system *s, const double *pos, int method, double alpha,
                   const int *grid, int order, int restraint_count, const int *restraint_atoms,
                   const double *restraint_reference, double restraint_k, double *forces,
                   double *terms) {
  memset(forces, 0, sizeof(double) * 3 * (size_t)s->n);
  memset(terms, 0, sizeof(double) * 10);
  terms[8] = orc_restraint(s, restraint_count, restraint_atoms, restraint_reference,
                           restraint_k, pos, forces);
  terms[0] = orc_bonds(s, pos, forces);
  terms[1] = orc_angles(s, pos, forces);
  terms[2] = orc_torsions(s, pos, forces);
  double a = method == 1 ? alpha : 0.0, cut = method == 1 ? s->cutoff : 0.0;
  double lj, coul, elj, ecoul;
  orc_direct_space(s, pos, a, cut, forces, &lj, &coul);
  orc_exceptions(s, pos, a, forces, &elj, &ecoul);
  terms[3] = lj + elj;
  terms[4] = coul + ecoul;
  if (method == 1) {
    terms[5] = orc_reciprocal(s, pos, alpha, grid, order, forces, NULL);
    double se[2];
    orc_ewald_self(s, alpha, se);
    terms[6] = se[0];
    terms[7] = se[1];
  }
  terms[9] = terms[0] + terms[1] + terms[2] + terms[3] + terms[4] + terms[5] + terms[6] +
             terms[7] + terms[8];
}

/* ----------------------------------------------- constraints (cpu/integrate/constraints) */
int orc_constrain_positions(const orc_system *s, double *pos, const double *ref, double tol,
                            int max_iter, double *corrections) {
  if (s->nconstraints == 0) return 0;
  for (int it = 0; it < max_iter; ++it) {
    double worst = 0;
    for (int k = 0; k < s->nconstraints; ++k) {
      int a = s->con_a[k], b = s->con_b[k];
      double t = s->con_d[k];
      double d[3] = {pos[3 * a] - pos[3 * b], pos[3 * a + 1] - pos[3 * b + 1],
                     pos[3 * a + 2] - pos[3 * b + 2]};
      double cur = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      double err = cur - t * t, rel = fabs(err) / (t * t);
      if (rel > worst) worst = rel;
      if (rel <= tol) continue;
      double r[3] = {ref[3 * a] - ref[3 * b], ref[3 * a + 1] - ref[3 * b + 1],
                     ref[3 * a + 2] - ref[3 * b + 2]};
      double proj = d[0] * r[0] + d[1] * r[1] + d[2] * r[2];
      double ia = s->masses[a] > 0 ? 1.0 / s->masses[a] : 0, ib = s->masses[b] > 0 ? 1.0 / s->masses[b] : 0;
      double den = 2.0 * (ia + ib) * proj;
      if (fabs(den) < 1e-20) continue;
      double lam = -err / den;
      for (int c = 0; c < 3; ++c) {
        double sa = lam * ia * r[c], sb = lam * ib * r[c];
        pos[3 * a + c] += sa;
        pos[3 * b + c] -= sb;
        if (corrections) {
          corrections[3 * a + c] += sa;
          corrections[3 * b + c] -= sb;
        }
      }
    }
    if (worst <= tol) return it + 1;
  }
  return -1;
}

int orc_constrain_velocities(const orc_system *s, const double *pos, double *vel, double tol,
                             int max_iter) {
  if (s->nconstraints == 0) return 0;
  for (int it = 0; it < max_iter; ++it) {
    double worst = 0;
    for (int k = 0; k < s->nconstraints; ++k) {
      int a = s->con_a[k], b = s->con_b[k];
      double r[3], v[3];
      for (int c = 0; c < 3; ++c) {
        r[c] = pos[3 * a + c] - pos[3 * b + c];
        v[c] = vel[3 * a + c] - vel[3 * b + c];
      }
      double proj = r[0] * v[0] + r[1] * v[1] + r[2] * v[2];
      double t = s->con_d[k], rel = fabs(proj) / (t * t);
      if (rel > worst) worst = rel;
      if (rel <= tol) continue;
      double ia = s->masses[a] > 0 ? 1.0 / s->masses[a] : 0, ib = s->masses[b] > 0 ? 1.0 / s->masses[b] : 0;
      double den = (ia + ib) * (r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      if (den < 1e-20) continue;
      double lam = -proj / den;
      for (int c = 0; c < 3; ++c) {
        vel[3 * a + c] += lam * ia * r[c];
        vel[3 * b + c] -= lam * ib * r[c];
      }
    }
    if (worst <= tol) return it + 1;
  }
  return -1;
}

/* ------------------------------------------------ BAOAB (cpu/integrate/langevin.js) */
typedef struct {
  double timestep, temperature, friction;
  uint32_t seed;
  double tolerance;
  int max_iterations;
} orc_integrator;

static int drift_with_constraints(const orc_system *s, double *pos, double *vel, double h,
                                  const orc_integrator *o, double *ref, double *corr,
                                  const unsigned char *touched) {
  memcpy(ref, pos, sizeof(double) * 3 * (size_t)s->n);
  for (int k = 0; k < 3 * s->n; ++k) pos[k] += h * vel[k];
  if (s->nconstraints == 0) return 0;
  memset(corr, 0, sizeof(double) * 3 * (size_t)s->n);
  int r = orc_constrain_positions(s, pos, ref, o->tolerance, o->max_iterations, corr);
  double inv = 1.0 / h;
  for (int a = 0; a < s->n; ++a)
    if (touched[a])
      for (int c = 0; c < 3; ++c) vel[3 * a + c] += corr[3 * a + c] * inv;
  return r;
}

/* One langevinStep: B R A(S) O R A(S); noise NULL means the counter RNG at `step`. */
int orc_langevin_step(const orc_system *s, double *pos, double *vel, const double *forces,
                      const orc_integrator *o, uint32_t step, const double *noise) {
  int n = s->n;
  double h = 0.5 * o->timestep, decay = exp(-o->friction * o->timestep);
  double ns = sqrt(1.0 - decay * decay), kT = BOLTZMANN * o->temperature;
  double *ref = (double *)malloc(sizeof(double) * 3 * (size_t)n);
  double *corr = (double *)malloc(sizeof(double) * 3 * (size_t)n);
  unsigned char *touched = (unsigned char *)calloc((size_t)n, 1);
  for (int k = 0; k < s->nconstraints; ++k) touched[s->con_a[k]] = touched[s->con_b[k]] = 1;
  int status = 0;
  for (int a = 0; a < n; ++a) {
    double m = s->masses[a];
    if (m <= 0) continue;
    for (int c = 0; c < 3; ++c) vel[3 * a + c] += (h / m) * forces[3 * a + c];
  }
  if (orc_constrain_velocities(s, pos, vel, o->tolerance, o->max_iterations) < 0) status |= 2;
  if (drift_with_constraints(s, pos, vel, h, o, ref, corr, touched) < 0) status |= 1;
  for (int a = 0; a < n; ++a) {
    double m = s->masses[a];
    if (m <= 0) continue;
    double g[3];
    if (noise) {
      g[0] = noise[3 * a];
      g[1] = noise[3 * a + 1];
      g[2] = noise[3 * a + 2];
    } else {
      orc_gaussian_triple(g, o->seed, (uint32_t)a, step);
    }
    double amp = ns * sqrt(kT / m);
    for (int c = 0; c < 3; ++c) vel[3 * a + c] = decay * vel[3 * a + c] + amp * g[c];
  }
  if (orc_constrain_velocities(s, pos, vel, o->tolerance, o->max_iterations) < 0) status |= 2;
  if (drift_with_constraints(s, pos, vel, h, o, ref, corr, touched) < 0) status |= 1;
  free(ref);
  free(corr);
  free(touched);
  return status;
}

int orc_finish_step(const orc_system *s, const double *pos, double *vel, const double *forces,
                    const orc_integrator *o) {
  double h = 0.5 * o->timestep;
  for (int a = 0; a < s->n; ++a) {
    double m = s->masses[a];
    if (m <= 0) continue;
    for (int c = 0; c < 3; ++c) vel[3 * a + c] += (h / m) * forces[3 * a + c];
  }
  return orc_constrain_velocities(s, pos, vel, o->tolerance, o->max_iterations) < 0 ? 2 : 0;
}

double orc_kinetic(const orc_system *s, const double *vel) {
  double k = 0;
  for (int a = 0; a < s->n; ++a) {
    double m = s->masses[a];
    if (m <= 0) continue;
    k += m * (vel[3 * a] * vel[3 * a] + vel[3 * a + 1] * vel[3 * a + 1] + vel[3 * a + 2] * vel[3 * a + 2]);
  }
  return 0.5 * k;
}

/* runDynamics (cpu/simulation.js:114-156): returns the last potential; `kinetic_out`
 * gets the sample taken before the closing half kick. */
double orc_run_dynamics(const orc_system *s, double *pos, double *vel, int steps,
                        uint32_t first_step, const orc_integrator *o, double alpha,
                        const int *grid, int order, double *kinetic_out) {
  double *f = (double *)malloc(sizeof(double) * 3 * (size_t)s->n);
  double terms[10];
  orc_potential(s, pos, 1, alpha, grid, order, 0, NULL, NULL, 0, f, terms);
  double kin = 0;
  for (int st = 0; st < steps; ++st) {
    orc_langevin_step(s, pos, vel, f, o, first_step + (uint32_t)st, NULL);
    orc_potential(s, pos, 1, alpha, grid, order, 0, NULL, NULL, 0, f, terms);
    kin = orc_kinetic(s, vel);
    orc_finish_step(s, pos, vel, f, o);
  }
  if (kinetic_out) *kinetic_out = kin;
  free(f);
  return terms[9];
}

/* --------------------------------------- barostat (webgpu/kernels/barostat.js:158-162) */
double orc_metropolis_weight(double delta_energy, double delta_volume, double volume_ratio,
                             double pressure, double kT, int molecules) {
  return delta_energy + pressure * delta_volume - molecules * kT * log(volume_ratio);
}

/* Molecule-centroid scaling in f64 (barostat.js:25-108 restated at full precision). */
void orc_scale_molecules(const orc_system *s, double *pos, double scale) {
  for (int m = 0; m < s->nmolecules; ++m) {
    double c[3] = {0, 0, 0}, total = 0;
    for (int k = s->mol_start[m]; k < s->mol_start[m + 1]; ++k) {
      int a = s->mol_atoms[k];
      for (int q = 0; q < 3; ++q) c[q] += s->masses[a] * pos[3 * a + q];
      total += s->masses[a];
    }
    if (total > 0) {
      for (int q = 0; q < 3; ++q) c[q] /= total;
    } else {
      int cnt = s->mol_start[m + 1] - s->mol_start[m];
      c[0] = c[1] = c[2] = 0;
      for (int k = s->mol_start[m]; k < s->mol_start[m + 1]; ++k)
        for (int q = 0; q < 3; ++q) c[q] += pos[3 * s->mol_atoms[k] + q];
      for (int q = 0; q < 3; ++q) c[q] /= (cnt > 0 ? cnt : 1);
    }
    for (int k = s->mol_start[m]; k < s->mol_start[m + 1]; ++k) {
      int a = s->mol_atoms[k];
      for (int q = 0; q < 3; ++q) pos[3 * a + q] += (scale - 1.0) * c[q];
    }
  }
}

/* --------------------------- f32 "as-device" cell list and neighbour list restatement
 * params: the 28-float uniform of wgsl-common.js:24-64 (box rows, recip rows, scalars).
 * Compiled with -ffp-contract=off: every operation below is one IEEE f32 rounding. */
static void f32_fractional(const float *p, const float *P, float *f) {
  /* dot(p, (recipA.x, recipB.x, recipC.x)) etc., summed left to right */
  for (int d = 0; d < 3; ++d) {
    float t0 = p[0] * P[12 + d];
    float t1 = p[1] * P[16 + d];
    float t2 = p[2] * P[20 + d];
    f[d] = (t0 + t1) + t2;
  }
}

static void f32_min_image(float *d, const float *P) {
  float s = floorf(d[2] / P[10] + 0.5f);
  d[0] = d[0] - s * P[8];
  d[1] = d[1] - s * P[9];
  d[2] = d[2] - s * P[10];
  s = floorf(d[1] / P[5] + 0.5f);
  d[0] = d[0] - s * P[4];
  d[1] = d[1] - s * P[5];
  d[2] = d[2] - s * P[6];
  s = floorf(d[0] / P[0] + 0.5f);
  d[0] = d[0] - s * P[0];
  d[1] = d[1] - s * P[1];
  d[2] = d[2] - s * P[2];
}

static void f32_cell_coord(const float *p, const float *P, const int *counts, int *c) {
  float f[3];
  f32_fractional(p, P, f);
  for (int d = 0; d < 3; ++d) {
    float wrapped = f[d] - floorf(f[d]);
    float scaled = wrapped * (float)counts[d];
    int v = (int)scaled;
    if (v > counts[d] - 1) v = counts[d] - 1;
    c[d] = v;
  }
}

void orc_cell_list_f32(int n, const float *pos, const float *P, const int *counts,
                       int *cell_of_atom, int *cell_start, int *cell_atoms) {
  int cells = counts[0] * counts[1] * counts[2];
  int *cnt = (int *)calloc((size_t)cells, sizeof(int));
  for (int a = 0; a < n; ++a) {
    int c[3];
    f32_cell_coord(pos + 3 * a, P, counts, c);
    int cell = (c[0] * counts[1] + c[1]) * counts[2] + c[2];
    cell_of_atom[a] = cell;
    cnt[cell]++;
  }
  cell_start[0] = 0;
  for (int c = 0; c < cells; ++c) cell_start[c + 1] = cell_start[c] + cnt[c];
  memset(cnt, 0, sizeof(int) * (size_t)cells);
  for (int a = 0; a < n; ++a) {
    int cell = cell_of_atom[a];
    cell_atoms[cell_start[cell] + cnt[cell]++] = a; /* ascending atom order per cell */
  }
  free(cnt);
}

static int wrap_cell(int v, int count) {
  int r = v % count;
  return r < 0 ? r + count : r;
}

/* neighbours.js:46-151: full both-direction list, stencil order, capacity-limited.
 * Returns the largest number of neighbours found for any atom. */
int orc_neighbour_list_f32(int n, const float *pos, const float *P, const int *counts,
                           const int *cell_start, const int *cell_atoms, const int *excl_start,
                           const int *excl_partners, int capacity, int *neighbours,
                           int *neighbour_count) {
  int required = 0;
  int base_o[3], count_o[3];
  for (int d = 0; d < 3; ++d) {
    if (counts[d] >= 3) { base_o[d] = -1; count_o[d] = 3; }
    else if (counts[d] == 2) { base_o[d] = 0; count_o[d] = 2; }
    else { base_o[d] = 0; count_o[d] = 1; }
  }
  float lc = P[25];
  float lc2 = lc * lc;
  for (int a = 0; a < n; ++a) {
    const float *ce = pos + 3 * a;
    int c[3];
    f32_cell_coord(ce, P, counts, c);
    int stored = 0, found = 0;
    for (int ox = 0; ox < count_o[0]; ++ox) {
      int cx = wrap_cell(c[0] + base_o[0] + ox, counts[0]);
      for (int oy = 0; oy < count_o[1]; ++oy) {
        int cy = wrap_cell(c[1] + base_o[1] + oy, counts[1]);
        for (int oz = 0; oz < count_o[2]; ++oz) {
          int cz = wrap_cell(c[2] + base_o[2] + oz, counts[2]);
          int cell = (cx * counts[1] + cy) * counts[2] + cz;
          for (int slot = cell_start[cell]; slot < cell_start[cell + 1]; ++slot) {
            int o = cell_atoms[slot];
            if (o == a) continue;
            float d[3] = {ce[0] - pos[3 * o], ce[1] - pos[3 * o + 1], ce[2] - pos[3 * o + 2]};
            f32_min_image(d, P);
            float t0 = d[0] * d[0], t1 = d[1] * d[1], t2 = d[2] * d[2];
            float r2 = (t0 + t1) + t2;
            if (r2 > lc2) continue;
            int lo = excl_start[a], hi = excl_start[a + 1], ex = 0;
            while (lo < hi) {
              int mid = lo + (hi - lo) / 2, v = excl_partners[mid];
              if (v == o) { ex = 1; break; }
              if (v < o) lo = mid + 1; else hi = mid;
            }
            if (ex) continue;
            found++;
            if (stored < capacity) neighbours[(size_t)a * capacity + stored++] = o;
          }
        }
      }
    }
    neighbour_count[a] = stored;
    if (found > required) required = found;
  }
  return required;
}
