/* CPU oracle of the headless structure renderer: test infrastructure only (it checks
 * rainmd_b200/csrc/raster.cu; nothing in the product links it).
 *
 * Restates the viewer's two WGSL programs (web/viewer.js:83-228 the ribbon sweep,
 * viewer.js:230-308 the sphere impostors) and the rasterisation rules the device renderer
 * states: pixel centres at (x + 0.5, y + 0.5), y downwards, edge functions with an
 * antisymmetric tie rule, perspective-correct attributes, the primitive's z/w clipped to
 * [0, 1], the depth test "less" against 1.0 with the earlier primitive winning a tie, a
 * sphere's written depth clamped to [0, 1], unorm8 by round-half-even. Scalar loops in draw
 * order; compiled without floating-point contraction, each expression evaluated in the order
 * written. The reference's own WebGPU pipeline cannot run here (no graphics stack), so this
 * restatement is the oracle and pixel parity with a browser's rasteriser is not claimed.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { float x, y, z; } v3;

static v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static v3 vadd(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 vsub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3 vscale(v3 a, float k) { return mk(a.x * k, a.y * k, a.z * k); }
static float vdot(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static float vlen(v3 a) { return sqrtf(vdot(a, a)); }
static v3 vnorm(v3 a) { float l = vlen(a); return mk(a.x / l, a.y / l, a.z / l); }
static v3 vcross(v3 a, v3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
/* WGSL mix(a, b, t) = a * (1 - t) + b * t */
static float mixs(float a, float b, float t) { return a * (1.0f - t) + b * t; }
static v3 mixv(v3 a, v3 b, float t) { return mk(mixs(a.x, b.x, t), mixs(a.y, b.y, t), mixs(a.z, b.z, t)); }

typedef struct { float vp[16], right[4], up[4], forward[4], centre[4]; } cam_t;

static void proj(const cam_t *c, v3 v, float out[4]) {
  for (int r = 0; r < 4; ++r)
    out[r] = ((c->vp[r] * v.x + c->vp[4 + r] * v.y) + c->vp[8 + r] * v.z) + c->vp[12 + r];
}
static v3 light(void) { return vnorm(mk(0.35f, 0.55f, 0.78f)); }

/* ---- the ribbon's vertex program */
static float cm1(float a0, float a1, float a2, float a3, float t, float t2, float t3) {
  float A = 2.0f * a1;
  float B = (-a0 + a2) * t;
  float C = (((2.0f * a0 - 5.0f * a1) + 4.0f * a2) - a3) * t2;
  float D = (((-a0 + 3.0f * a1) - 3.0f * a2) + a3) * t3;
  return 0.5f * (((A + B) + C) + D);
}
static v3 catmull(v3 p0, v3 p1, v3 p2, v3 p3, float t) {
  float t2 = t * t, t3 = t2 * t;
  return mk(cm1(p0.x, p1.x, p2.x, p3.x, t, t2, t3), cm1(p0.y, p1.y, p2.y, p3.y, t, t2, t3),
            cm1(p0.z, p1.z, p2.z, p3.z, t, t2, t3));
}
typedef struct { v3 centre, side, up, colour; float hw, ht; } sample_t;

static sample_t sample_at(const float *guides, const unsigned *ctl, float t) {
  const float *g0 = guides + 12 * ctl[0], *g1 = guides + 12 * ctl[1], *g2 = guides + 12 * ctl[2],
              *g3 = guides + 12 * ctl[3];
  v3 p0 = mk(g0[0], g0[1], g0[2]), p1 = mk(g1[0], g1[1], g1[2]), p2 = mk(g2[0], g2[1], g2[2]),
     p3 = mk(g3[0], g3[1], g3[2]);
  sample_t s;
  s.centre = catmull(p0, p1, p2, p3, t);
  v3 ahead = catmull(p0, p1, p2, p3, fminf(t + 0.01f, 1.0f));
  v3 behind = catmull(p0, p1, p2, p3, fmaxf(t - 0.01f, 0.0f));
  v3 tangent = vsub(ahead, behind);
  if (vlen(tangent) < 1e-7f) tangent = mk(0.0f, 0.0f, 1.0f);
  tangent = vnorm(tangent);
  v3 side = vnorm(mixv(mk(g1[4], g1[5], g1[6]), mk(g2[4], g2[5], g2[6]), t));
  side = vsub(side, vscale(tangent, vdot(side, tangent)));
  if (vlen(side) < 1e-6f) side = vnorm(vcross(tangent, mk(0.0f, 0.0f, 1.0f)));
  s.side = vnorm(side);
  s.up = vnorm(vcross(tangent, s.side));
  s.hw = mixs(g1[3], g2[3], t);
  s.ht = mixs(g1[7], g2[7], t);
  s.colour = mixv(mk(g1[8], g1[9], g1[10]), mk(g2[8], g2[9], g2[10]), t);
  return s;
}
static v3 corner(v3 side, v3 up, float hw, float ht, unsigned k) {
  float w = (k == 0u || k == 3u) ? hw : -hw;
  float h = (k == 0u || k == 1u) ? ht : -ht;
  return vadd(vscale(side, w), vscale(up, h));
}
/* vertex `v` of the sweep: clip[4], colour[3], normal[3] */
static void ribbon_vertex(const cam_t *c, const float *guides, const unsigned *segments, long v, float out[10]) {
  unsigned quad = (unsigned)(v / 24), within = (unsigned)(v % 24);
  unsigned face = within / 6u, which = within % 6u, seg = quad / 8u, step = quad % 8u;
  const unsigned *ctl = segments + 4 * seg;
  float t0 = (float)step / 8.0f, t1 = (float)(step + 1u) / 8.0f;
  sample_t a = sample_at(guides, ctl, t0), b = sample_at(guides, ctl, t1);
  int far_end = which == 2u || which == 3u || which == 5u;
  int next_corner = which == 1u || which == 4u || which == 5u;
  unsigned k = (face + (next_corner ? 1u : 0u)) % 4u;
  sample_t at = far_end ? b : a;
  v3 offset = corner(at.side, at.up, at.hw, at.ht, k);
  v3 outward = vadd(corner(a.side, a.up, a.hw, a.ht, face % 4u), corner(a.side, a.up, a.hw, a.ht, (face + 1u) % 4u));
  v3 world = vsub(vadd(at.centre, offset), mk(c->centre[0], c->centre[1], c->centre[2]));
  v3 normal = vlen(outward) < 1e-9f ? a.up : vnorm(outward);
  proj(c, world, out);
  out[4] = at.colour.x; out[5] = at.colour.y; out[6] = at.colour.z;
  out[7] = normal.x; out[8] = normal.y; out[9] = normal.z;
}

/* ---- triangle setup and coverage */
typedef struct { float px[3], py[3], z[3], iw[3]; int ord[3]; float area; } tri_t;

static float edgef(float ax, float ay, float bx, float by, float qx, float qy) {
  return (bx - ax) * (qy - ay) - (by - ay) * (qx - ax);
}
static int owns(float ax, float ay, float bx, float by) {
  float dy = by - ay, dx = bx - ax;
  return dy < 0.0f || (dy == 0.0f && dx > 0.0f);
}
static int setup(const float c[3][4], int width, int height, tri_t *t) {
  float px[3], py[3], z[3], iw[3];
  for (int k = 0; k < 3; ++k) {
    if (!(c[k][3] > 0.0f)) return 0;
    float nx = c[k][0] / c[k][3], ny = c[k][1] / c[k][3];
    px[k] = (nx + 1.0f) * (0.5f * (float)width);
    py[k] = (1.0f - ny) * (0.5f * (float)height);
    z[k] = c[k][2] / c[k][3];
    iw[k] = 1.0f / c[k][3];
  }
  float area = edgef(px[0], py[0], px[1], py[1], px[2], py[2]);
  if (!(area != 0.0f) || !isfinite(area)) return 0;
  int ord[3] = {0, 1, 2};
  if (area < 0.0f) { ord[1] = 2; ord[2] = 1; area = -area; }
  for (int k = 0; k < 3; ++k) {
    t->px[k] = px[ord[k]]; t->py[k] = py[ord[k]]; t->z[k] = z[ord[k]]; t->iw[k] = iw[ord[k]]; t->ord[k] = ord[k];
  }
  t->area = area;
  return 1;
}
static int cover(const tri_t *t, int x, int y, float l[3], float b[3]) {
  float qx = (float)x + 0.5f, qy = (float)y + 0.5f;
  float e0 = edgef(t->px[1], t->py[1], t->px[2], t->py[2], qx, qy);
  float e1 = edgef(t->px[2], t->py[2], t->px[0], t->py[0], qx, qy);
  float e2 = edgef(t->px[0], t->py[0], t->px[1], t->py[1], qx, qy);
  if (e0 < 0.0f || e1 < 0.0f || e2 < 0.0f) return 0;
  if (e0 == 0.0f && !owns(t->px[1], t->py[1], t->px[2], t->py[2])) return 0;
  if (e1 == 0.0f && !owns(t->px[2], t->py[2], t->px[0], t->py[0])) return 0;
  if (e2 == 0.0f && !owns(t->px[0], t->py[0], t->px[1], t->py[1])) return 0;
  float w[3] = {e0 / t->area, e1 / t->area, e2 / t->area};
  float pb[3] = {w[0] * t->iw[0], w[1] * t->iw[1], w[2] * t->iw[2]};
  float s = (pb[0] + pb[1]) + pb[2];
  for (int k = 0; k < 3; ++k) { l[t->ord[k]] = w[k]; b[t->ord[k]] = pb[k] / s; }
  return 1;
}
static float depth_at(const tri_t *t, const float l[3]) {
  return (l[t->ord[0]] * t->z[0] + l[t->ord[1]] * t->z[1]) + l[t->ord[2]] * t->z[2];
}

/* ---- the sphere impostor */
static const float CX[4] = {-1.0f, 1.0f, -1.0f, 1.0f}, CY[4] = {-1.0f, -1.0f, 1.0f, 1.0f};
static const int TRI[2][3] = {{0, 1, 2}, {2, 1, 3}};

static void sphere_corners(const cam_t *c, const float *pos, const float *style, float out[4][4]) {
  v3 centre = vsub(mk(pos[0], pos[1], pos[2]), mk(c->centre[0], c->centre[1], c->centre[2]));
  v3 right = mk(c->right[0], c->right[1], c->right[2]), up = mk(c->up[0], c->up[1], c->up[2]);
  for (int k = 0; k < 4; ++k) {
    v3 spread = vadd(vscale(right, CX[k]), vscale(up, CY[k]));
    proj(c, vadd(centre, vscale(spread, style[3])), out[k]);
  }
}
/* returns 1 when kept; depth and colour out */
static int sphere_fragment(const cam_t *c, const float *pos, const float *style, int tri, const float b[3],
                           float *depth, v3 *colour) {
  float ox = (b[0] * CX[TRI[tri][0]] + b[1] * CX[TRI[tri][1]]) + b[2] * CX[TRI[tri][2]];
  float oy = (b[0] * CY[TRI[tri][0]] + b[1] * CY[TRI[tri][1]]) + b[2] * CY[TRI[tri][2]];
  float squared = ox * ox + oy * oy;
  if (squared > 1.0f) return 0;
  float height = sqrtf(1.0f - squared);
  v3 centre = vsub(mk(pos[0], pos[1], pos[2]), mk(c->centre[0], c->centre[1], c->centre[2]));
  v3 right = mk(c->right[0], c->right[1], c->right[2]), up = mk(c->up[0], c->up[1], c->up[2]),
     fwd = mk(c->forward[0], c->forward[1], c->forward[2]);
  v3 dir = vadd(vadd(vscale(right, ox), vscale(up, oy)), vscale(fwd, height));
  float clip[4];
  proj(c, vadd(centre, vscale(dir, style[3])), clip);
  v3 n = mk(ox, oy, height);
  float diffuse = fmaxf(vdot(n, light()), 0.0f);
  float r = 1.0f - height;
  float rim = (r * r) * sqrtf(r);
  float shade = 0.22f + 0.78f * diffuse;
  *depth = fminf(fmaxf(clip[2] / clip[3], 0.0f), 1.0f);
  *colour = vadd(vscale(mk(style[0], style[1], style[2]), shade), vscale(mk(0.10f, 0.10f, 0.10f), rim));
  return 1;
}

static void bbox(const tri_t *t, int width, int height, int *x0, int *x1, int *y0, int *y1) {
  float a = fminf(fminf(t->px[0], t->px[1]), t->px[2]), b = fmaxf(fmaxf(t->px[0], t->px[1]), t->px[2]);
  float c = fminf(fminf(t->py[0], t->py[1]), t->py[2]), d = fmaxf(fmaxf(t->py[0], t->py[1]), t->py[2]);
  *x0 = (int)fmaxf(floorf(a - 0.5f), 0.0f);
  *x1 = (int)fminf(ceilf(b - 0.5f), (float)(width - 1));
  *y0 = (int)fmaxf(floorf(c - 0.5f), 0.0f);
  *y1 = (int)fminf(ceilf(d - 0.5f), (float)(height - 1));
}

void orc_render(const float *positions, int n, const float *camera, const float *styles, const float *guides,
                int guide_count, const unsigned *segments, int segment_count, int draw_spheres, int draw_ribbon,
                int width, int height, unsigned char *rgba) {
  (void)guide_count;
  cam_t c;
  memcpy(&c, camera, sizeof c);
  const long pixels = (long)width * height;
  uint64_t *keys = (uint64_t *)malloc(sizeof(uint64_t) * pixels);
  for (long p = 0; p < pixels; ++p) keys[p] = ~(uint64_t)0;
  const int spheres = draw_spheres && n > 0;
  const long sphere_prims = spheres ? 2L * n : 0;
  const long ribbon_tris = (draw_ribbon && segment_count > 0) ? 8L * 8 * segment_count : 0;
  float *rv = NULL;
  if (ribbon_tris) {
    rv = (float *)malloc(sizeof(float) * 10 * 3 * ribbon_tris);
    for (long v = 0; v < 3 * ribbon_tris; ++v) ribbon_vertex(&c, guides, segments, v, rv + 10 * v);
  }
  /* draw */
  for (long prim = 0; prim < sphere_prims + ribbon_tris; ++prim) {
    float cl[3][4];
    int atom = 0, tri = 0;
    if (prim < sphere_prims) {
      atom = (int)(prim >> 1);
      tri = (int)(prim & 1);
      if (!(styles[4 * atom + 3] > 0.0f)) continue;
      float q[4][4];
      sphere_corners(&c, positions + 3 * atom, styles + 4 * atom, q);
      for (int k = 0; k < 3; ++k) memcpy(cl[k], q[TRI[tri][k]], sizeof cl[k]);
    } else {
      long r = prim - sphere_prims;
      for (int k = 0; k < 3; ++k) memcpy(cl[k], rv + 10 * (3 * r + k), sizeof cl[k]);
    }
    tri_t t;
    if (!setup(cl, width, height, &t)) continue;
    int x0, x1, y0, y1;
    bbox(&t, width, height, &x0, &x1, &y0, &y1);
    for (int y = y0; y <= y1; ++y)
      for (int x = x0; x <= x1; ++x) {
        float l[3], b[3];
        if (!cover(&t, x, y, l, b)) continue;
        float zq = depth_at(&t, l);
        if (!(zq >= 0.0f && zq <= 1.0f)) continue;
        float depth = zq;
        if (prim < sphere_prims) {
          v3 unused;
          if (!sphere_fragment(&c, positions + 3 * atom, styles + 4 * atom, tri, b, &depth, &unused)) continue;
        }
        if (!(depth < 1.0f)) continue;
        uint32_t bits;
        memcpy(&bits, &depth, 4);
        uint64_t key = ((uint64_t)bits << 32) | (uint32_t)prim;
        if (key < keys[(long)y * width + x]) keys[(long)y * width + x] = key;
      }
  }
  /* resolve */
  for (long p = 0; p < pixels; ++p) {
    v3 colour = mk(0.071f, 0.078f, 0.086f);
    if (keys[p] != ~(uint64_t)0) {
      long prim = (long)(keys[p] & 0xffffffffu);
      int x = (int)(p % width), y = (int)(p / width);
      float cl[3][4], l[3], b[3];
      tri_t t;
      if (prim < sphere_prims) {
        int atom = (int)(prim >> 1), tri = (int)(prim & 1);
        float q[4][4];
        sphere_corners(&c, positions + 3 * atom, styles + 4 * atom, q);
        for (int k = 0; k < 3; ++k) memcpy(cl[k], q[TRI[tri][k]], sizeof cl[k]);
        float depth;
        if (setup(cl, width, height, &t) && cover(&t, x, y, l, b))
          sphere_fragment(&c, positions + 3 * atom, styles + 4 * atom, tri, b, &depth, &colour);
      } else {
        long r = prim - sphere_prims;
        const float *v = rv + 10 * 3 * r;
        for (int k = 0; k < 3; ++k) memcpy(cl[k], v + 10 * k, sizeof cl[k]);
        if (setup(cl, width, height, &t) && cover(&t, x, y, l, b)) {
          v3 cc = mk((b[0] * v[4] + b[1] * v[14]) + b[2] * v[24], (b[0] * v[5] + b[1] * v[15]) + b[2] * v[25],
                     (b[0] * v[6] + b[1] * v[16]) + b[2] * v[26]);
          v3 nn = mk((b[0] * v[7] + b[1] * v[17]) + b[2] * v[27], (b[0] * v[8] + b[1] * v[18]) + b[2] * v[28],
                     (b[0] * v[9] + b[1] * v[19]) + b[2] * v[29]);
          float facing = fabsf(vdot(vnorm(nn), light()));
          colour = vscale(cc, 0.26f + 0.74f * facing);
        }
      }
    }
    float rgb[3] = {colour.x, colour.y, colour.z};
    for (int k = 0; k < 3; ++k) rgba[4 * p + k] = (unsigned char)rintf(fminf(fmaxf(rgb[k], 0.0f), 1.0f) * 255.0f);
    rgba[4 * p + 3] = 255;
  }
  free(rv);
  free(keys);
}
