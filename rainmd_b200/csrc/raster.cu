// Headless rasteriser for the structure viewer's two passes (web/viewer.js): sphere impostors
// (SHADER, viewer.js:230-308: one camera-facing quad per atom, the sphere solved per fragment,
// depth written from the solved surface) and the cartoon ribbon swept from per-residue guides
// (RIBBON_SHADER, viewer.js:83-228: Catmull-Rom centre line, box cross-section, 24 vertices a
// step, 8 steps a segment), into a device RGBA8 image with no graphics API.
//
// Pipeline: a vertex stage writes every vertex's clip position and attributes once; a raster
// stage (one warp per triangle, lanes over the triangle's pixel box) tests coverage at pixel
// centres and keeps, per pixel, the 64-bit minimum of (depth bits << 32 | primitive order) with
// atomicMin, which is the depth test "less" against a cleared 1.0 with the earlier primitive
// winning a tie, as draw order decides it; a resolve stage re-evaluates the winning primitive's
// fragment shader at each pixel. Every floating-point expression has one stated evaluation
// order (this file is compiled without multiply-add contraction), so the image is a pure
// function of the inputs.
//
// Rasterisation rules: pixel centres at (x + 0.5, y + 0.5); framebuffer y downwards;
// coverage by edge functions with an antisymmetric tie rule (an edge is owned by exactly one
// of the two triangles that share it); attributes perspective-correct; the quad depth z/w
// clipped to [0, 1] per fragment; a sphere's written depth clamped to [0, 1]; no face
// culling. A triangle with a vertex at or behind the camera plane (w <= 0) is not drawn.
#include <cstdint>

#include "common.cuh"
#include "kernels.h"

namespace rmd {

namespace {

constexpr int RIBBON_STEPS = 8;  // RIBBON_SUBDIV (viewer.js:81)

struct F3 {
  float x, y, z;
};
__device__ __forceinline__ F3 f3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ F3 add(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 mul(F3 a, float k) { return {a.x * k, a.y * k, a.z * k}; }
__device__ __forceinline__ float dot3(F3 a, F3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ float len3(F3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ F3 normalize3(F3 a) {
  const float l = len3(a);
  return {a.x / l, a.y / l, a.z / l};
}
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ F3 mix3(F3 a, F3 b, float t) { return {mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)}; }

// clip = VP * (v, 1), VP column-major, each row summed left to right
__device__ __forceinline__ float4 project(const RenderCamera &c, F3 v) {
  float r[4];
#pragma unroll
  for (int k = 0; k < 4; ++k)
    r[k] = ((c.vp[k] * v.x + c.vp[4 + k] * v.y) + c.vp[8 + k] * v.z) + c.vp[12 + k];
  return make_float4(r[0], r[1], r[2], r[3]);
}

__device__ __forceinline__ F3 light_direction() { return normalize3(f3(0.35f, 0.55f, 0.78f)); }

// --------------------------------------------------------------------------- ribbon sweep
__device__ F3 catmull(F3 p0, F3 p1, F3 p2, F3 p3, float t) {
  const float t2 = t * t, t3 = t2 * t;
  auto one = [&](float a0, float a1, float a2, float a3) {
    const float A = 2.0f * a1;
    const float B = (-a0 + a2) * t;
    const float C = (((2.0f * a0 - 5.0f * a1) + 4.0f * a2) - a3) * t2;
    const float D = (((-a0 + 3.0f * a1) - 3.0f * a2) + a3) * t3;
    return 0.5f * (((A + B) + C) + D);
  };
  return {one(p0.x, p1.x, p2.x, p3.x), one(p0.y, p1.y, p2.y, p3.y), one(p0.z, p1.z, p2.z, p3.z)};
}

struct Sample {
  F3 centre, side, up, colour;
  float half_width, half_thick;
};

__device__ F3 guide_pos(const float *g) { return f3(g[0], g[1], g[2]); }

__device__ Sample sample_at(const float *guides, uint4 control, float t) {
  const float *g0 = guides + 12 * control.x, *g1 = guides + 12 * control.y, *g2 = guides + 12 * control.z,
              *g3 = guides + 12 * control.w;
  const F3 p0 = guide_pos(g0), p1 = guide_pos(g1), p2 = guide_pos(g2), p3 = guide_pos(g3);
  Sample s;
  s.centre = catmull(p0, p1, p2, p3, t);
  const F3 ahead = catmull(p0, p1, p2, p3, fminf(t + 0.01f, 1.0f));
  const F3 behind = catmull(p0, p1, p2, p3, fmaxf(t - 0.01f, 0.0f));
  F3 tangent = sub(ahead, behind);
  if (len3(tangent) < 1e-7f) tangent = f3(0.0f, 0.0f, 1.0f);
  tangent = normalize3(tangent);
  F3 side = normalize3(mix3(f3(g1[4], g1[5], g1[6]), f3(g2[4], g2[5], g2[6]), t));
  side = sub(side, mul(tangent, dot3(side, tangent)));
  if (len3(side) < 1e-6f) side = normalize3(cross3(tangent, f3(0.0f, 0.0f, 1.0f)));
  s.side = normalize3(side);
  s.up = normalize3(cross3(tangent, s.side));
  s.half_width = mixf(g1[3], g2[3], t);
  s.half_thick = mixf(g1[7], g2[7], t);
  s.colour = mix3(f3(g1[8], g1[9], g1[10]), f3(g2[8], g2[9], g2[10]), t);
  return s;
}

__device__ F3 corner(F3 side, F3 up, float half_width, float half_thick, unsigned k) {
  const float w = (k == 0u || k == 3u) ? half_width : -half_width;
  const float h = (k == 0u || k == 1u) ? half_thick : -half_thick;
  return add(mul(side, w), mul(up, h));
}

}  // namespace

// One thread per ribbon vertex (viewer.js:168-210): clip position, colour and normal.
__global__ void k_ribbon_vertices(RenderArgs a) {
  const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= 24ll * RIBBON_STEPS * a.segment_count) return;
  const unsigned quad = (unsigned)(v / 24), within = (unsigned)(v % 24);
  const unsigned face = within / 6u, which = within % 6u;
  const unsigned segment = quad / RIBBON_STEPS, step = quad % RIBBON_STEPS;
  const uint4 control = a.segments[segment];
  const float t0 = (float)step / (float)RIBBON_STEPS, t1 = (float)(step + 1u) / (float)RIBBON_STEPS;
  const Sample s0 = sample_at(a.guides, control, t0);
  const Sample s1 = sample_at(a.guides, control, t1);
  const bool far_end = which == 2u || which == 3u || which == 5u;
  const bool next_corner = which == 1u || which == 4u || which == 5u;
  const unsigned k = (face + (next_corner ? 1u : 0u)) % 4u;
  const Sample &at = far_end ? s1 : s0;
  const F3 offset = corner(at.side, at.up, at.half_width, at.half_thick, k);
  const F3 outward = add(corner(s0.side, s0.up, s0.half_width, s0.half_thick, face % 4u),
                         corner(s0.side, s0.up, s0.half_width, s0.half_thick, (face + 1u) % 4u));
  const F3 world = sub(add(at.centre, offset), f3(a.camera.centre[0], a.camera.centre[1], a.camera.centre[2]));
  const F3 normal = len3(outward) < 1e-9f ? s0.up : normalize3(outward);
  float *o = a.ribbon_vertices + 12 * v;
  const float4 clip = project(a.camera, world);
  o[0] = clip.x;
  o[1] = clip.y;
  o[2] = clip.z;
  o[3] = clip.w;
  o[4] = at.colour.x;
  o[5] = at.colour.y;
  o[6] = at.colour.z;
  o[7] = normal.x;
  o[8] = normal.y;
  o[9] = normal.z;
  o[10] = 0.0f;
  o[11] = 0.0f;
}

// One thread per atom (viewer.js:250-275): the quad's four corners in clip space, in the order
// (-1,-1), (1,-1), (-1,1), (1,1).
__global__ void k_sphere_vertices(RenderArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.atom_count) return;
  const float4 st = a.styles[i];
  const float4 p = a.positions[i];
  const F3 centre = sub(f3(p.x, p.y, p.z), f3(a.camera.centre[0], a.camera.centre[1], a.camera.centre[2]));
  const F3 right = f3(a.camera.right[0], a.camera.right[1], a.camera.right[2]);
  const F3 up = f3(a.camera.up[0], a.camera.up[1], a.camera.up[2]);
  const float cx[4] = {-1.0f, 1.0f, -1.0f, 1.0f}, cy[4] = {-1.0f, -1.0f, 1.0f, 1.0f};
  float4 *o = a.sphere_corners + 4 * (long long)i;
  for (int k = 0; k < 4; ++k) {
    const F3 spread = add(mul(right, cx[k]), mul(up, cy[k]));
    o[k] = project(a.camera, add(centre, mul(spread, st.w)));
  }
}

namespace {

struct Tri {
  float2 p[3];   // framebuffer positions
  float z[3];    // z / w
  float iw[3];   // 1 / w
  int order[3];  // which input vertex each of p[] is (after orientation)
  float area;
};

__device__ __forceinline__ float edge(float2 a, float2 b, float2 q) {
  return (b.x - a.x) * (q.y - a.y) - (b.y - a.y) * (q.x - a.x);
}
// the tie rule: a pixel centre exactly on edge a->b is inside when the edge points up the
// screen, or along it to the right; the shared edge of two triangles runs the other way in
// the neighbour, so exactly one of them owns it
__device__ __forceinline__ bool owns(float2 a, float2 b) {
  const float dy = b.y - a.y, dx = b.x - a.x;
  return dy < 0.0f || (dy == 0.0f && dx > 0.0f);
}

// Screen setup of a triangle from three clip positions; false when it is not drawn.
__device__ bool setup(const RenderCamera &, float4 c0, float4 c1, float4 c2, int width, int height, Tri &t) {
  const float4 c[3] = {c0, c1, c2};
  float2 p[3];
  float z[3], iw[3];
  for (int k = 0; k < 3; ++k) {
    if (!(c[k].w > 0.0f)) return false;
    const float nx = c[k].x / c[k].w, ny = c[k].y / c[k].w;
    p[k] = make_float2((nx + 1.0f) * (0.5f * (float)width), (1.0f - ny) * (0.5f * (float)height));
    z[k] = c[k].z / c[k].w;
    iw[k] = 1.0f / c[k].w;
  }
  float area = edge(p[0], p[1], p[2]);
  if (!(area != 0.0f) || !isfinite(area)) return false;
  int ord[3] = {0, 1, 2};
  if (area < 0.0f) {  // orient every triangle the same way round
    ord[1] = 2;
    ord[2] = 1;
    area = -area;
  }
  for (int k = 0; k < 3; ++k) {
    t.p[k] = p[ord[k]];
    t.z[k] = z[ord[k]];
    t.iw[k] = iw[ord[k]];
    t.order[k] = ord[k];
  }
  t.area = area;
  return true;
}

// Coverage of pixel (x, y); on success the screen-linear weights l[] (for depth) and the
// perspective-correct weights b[] (for attributes), both indexed by input vertex.
__device__ bool cover(const Tri &t, int x, int y, float l[3], float b[3]) {
  const float2 q = make_float2((float)x + 0.5f, (float)y + 0.5f);
  const float e0 = edge(t.p[1], t.p[2], q), e1 = edge(t.p[2], t.p[0], q), e2 = edge(t.p[0], t.p[1], q);
  if (e0 < 0.0f || e1 < 0.0f || e2 < 0.0f) return false;
  if (e0 == 0.0f && !owns(t.p[1], t.p[2])) return false;
  if (e1 == 0.0f && !owns(t.p[2], t.p[0])) return false;
  if (e2 == 0.0f && !owns(t.p[0], t.p[1])) return false;
  const float w[3] = {e0 / t.area, e1 / t.area, e2 / t.area};
  const float pb[3] = {w[0] * t.iw[0], w[1] * t.iw[1], w[2] * t.iw[2]};
  const float s = (pb[0] + pb[1]) + pb[2];
  for (int k = 0; k < 3; ++k) {
    l[t.order[k]] = w[k];
    b[t.order[k]] = pb[k] / s;
  }
  return true;
}

__device__ __forceinline__ float depth_at(const Tri &t, const float l_by_input[3]) {
  // the same weights back in oriented order
  float z = 0.0f;
  z = (l_by_input[t.order[0]] * t.z[0] + l_by_input[t.order[1]] * t.z[1]) + l_by_input[t.order[2]] * t.z[2];
  return z;
}

// The sphere fragment (viewer.js:286-307) at weights b[] of triangle `tri` (0 or 1) of a quad.
struct SphereFragment {
  bool kept;
  float depth;
  F3 colour;
};
__device__ SphereFragment sphere_fragment(const RenderArgs &a, int atom, int tri, const float b[3]) {
  const float cx[4] = {-1.0f, 1.0f, -1.0f, 1.0f}, cy[4] = {-1.0f, -1.0f, 1.0f, 1.0f};
  const int vs[2][3] = {{0, 1, 2}, {2, 1, 3}};  // corners of the two triangles, in vertex order
  float ox = 0.0f, oy = 0.0f;
  ox = (b[0] * cx[vs[tri][0]] + b[1] * cx[vs[tri][1]]) + b[2] * cx[vs[tri][2]];
  oy = (b[0] * cy[vs[tri][0]] + b[1] * cy[vs[tri][1]]) + b[2] * cy[vs[tri][2]];
  SphereFragment f{false, 1.0f, f3(0.0f, 0.0f, 0.0f)};
  const float squared = ox * ox + oy * oy;
  if (squared > 1.0f) return f;
  const float height = sqrtf(1.0f - squared);
  const float4 st = a.styles[atom];
  const float4 p = a.positions[atom];
  const RenderCamera &c = a.camera;
  const F3 centre = sub(f3(p.x, p.y, p.z), f3(c.centre[0], c.centre[1], c.centre[2]));
  const F3 right = f3(c.right[0], c.right[1], c.right[2]), up = f3(c.up[0], c.up[1], c.up[2]),
           fwd = f3(c.forward[0], c.forward[1], c.forward[2]);
  const F3 dir = add(add(mul(right, ox), mul(up, oy)), mul(fwd, height));
  const float4 clip = project(c, add(centre, mul(dir, st.w)));
  const F3 n = f3(ox, oy, height);
  const float diffuse = fmaxf(dot3(n, light_direction()), 0.0f);
  const float r = 1.0f - height;
  const float rim = (r * r) * sqrtf(r);  // r^2.5
  const float shade = 0.22f + 0.78f * diffuse;
  f.kept = true;
  f.depth = fminf(fmaxf(clip.z / clip.w, 0.0f), 1.0f);
  f.colour = add(mul(f3(st.x, st.y, st.z), shade), mul(f3(0.10f, 0.10f, 0.10f), rim));
  return f;
}

__device__ __forceinline__ unsigned long long pixel_key(float depth, unsigned prim) {
  return ((unsigned long long)__float_as_uint(depth) << 32) | prim;
}

__device__ void sphere_triangle(const RenderArgs &a, int atom, int tri, Tri &t, bool &ok) {
  const float4 *c = a.sphere_corners + 4 * (long long)atom;
  ok = tri == 0 ? setup(a.camera, c[0], c[1], c[2], a.width, a.height, t)
                : setup(a.camera, c[2], c[1], c[3], a.width, a.height, t);
}

__device__ void ribbon_triangle(const RenderArgs &a, long long prim, Tri &t, bool &ok) {
  const float *v = a.ribbon_vertices + 12 * (3 * prim);
  ok = setup(a.camera, make_float4(v[0], v[1], v[2], v[3]), make_float4(v[12], v[13], v[14], v[15]),
             make_float4(v[24], v[25], v[26], v[27]), a.width, a.height, t);
}

// Raster one triangle with one warp; `emit` returns whether a covered pixel keeps a fragment
// and its depth.
template <typename Emit>
__device__ void raster(const RenderArgs &a, const Tri &t, unsigned prim, Emit emit) {
  const float x0 = fminf(fminf(t.p[0].x, t.p[1].x), t.p[2].x), x1 = fmaxf(fmaxf(t.p[0].x, t.p[1].x), t.p[2].x);
  const float y0 = fminf(fminf(t.p[0].y, t.p[1].y), t.p[2].y), y1 = fmaxf(fmaxf(t.p[0].y, t.p[1].y), t.p[2].y);
  // clamped as floats first, so an off-screen vertex cannot overflow the conversion
  const int px0 = (int)fmaxf(floorf(x0 - 0.5f), 0.0f), px1 = (int)fminf(ceilf(x1 - 0.5f), (float)(a.width - 1));
  const int py0 = (int)fmaxf(floorf(y0 - 0.5f), 0.0f), py1 = (int)fminf(ceilf(y1 - 0.5f), (float)(a.height - 1));
  if (px0 > px1 || py0 > py1) return;
  const int bw = px1 - px0 + 1;
  const long long pixels = (long long)bw * (py1 - py0 + 1);
  for (long long k = threadIdx.x & 31; k < pixels; k += 32) {
    const int x = px0 + (int)(k % bw), y = py0 + (int)(k / bw);
    float l[3], b[3];
    if (!cover(t, x, y, l, b)) continue;
    const float zq = depth_at(t, l);
    if (!(zq >= 0.0f && zq <= 1.0f)) continue;  // the near and far clip planes
    float depth;
    if (!emit(l, b, zq, depth)) continue;
    if (!(depth < 1.0f)) continue;  // "less" against the cleared 1.0
    atomicMin(a.keys + (long long)y * a.width + x, pixel_key(depth, prim));
  }
}

}  // namespace

__global__ void k_render_clear(RenderArgs a) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < (long long)a.width * a.height) a.keys[p] = ~0ull;
}

// One warp per sphere triangle: primitive order 2 * atom + triangle.
__global__ void k_sphere_raster(RenderArgs a) {
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= 2ll * a.atom_count) return;
  const int atom = (int)(w >> 1), tri = (int)(w & 1);
  if (!(a.styles[atom].w > 0.0f)) return;  // a zero radius collapses the quad
  Tri t;
  bool ok;
  sphere_triangle(a, atom, tri, t, ok);
  if (!ok) return;
  raster(a, t, (unsigned)w, [&](const float *, const float *b, float, float &depth) {
    const SphereFragment f = sphere_fragment(a, atom, tri, b);
    depth = f.depth;
    return f.kept;
  });
}

// One warp per ribbon triangle: primitive order after every sphere triangle.
__global__ void k_ribbon_raster(RenderArgs a) {
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long tris = 8ll * RIBBON_STEPS * a.segment_count;
  if (w >= tris) return;
  Tri t;
  bool ok;
  ribbon_triangle(a, w, t, ok);
  if (!ok) return;
  raster(a, t, (unsigned)(2ll * a.atom_count * a.draw_spheres + w), [&](const float *, const float *, float zq,
                                                                          float &depth) {
    depth = zq;
    return true;
  });
}

// One thread per pixel: the background, or the winning primitive's fragment colour.
__global__ void k_render_resolve(RenderArgs a) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (long long)a.width * a.height) return;
  const unsigned long long key = a.keys[p];
  F3 colour = f3(0.071f, 0.078f, 0.086f);
  if (key != ~0ull) {
    const unsigned prim = (unsigned)(key & 0xffffffffull);
    const int x = (int)(p % a.width), y = (int)(p / a.width);
    const long long sphere_prims = a.draw_spheres ? 2ll * a.atom_count : 0;
    Tri t;
    bool ok;
    float l[3], b[3];
    if ((long long)prim < sphere_prims) {
      const int atom = (int)(prim >> 1), tri = (int)(prim & 1u);
      sphere_triangle(a, atom, tri, t, ok);
      if (ok && cover(t, x, y, l, b)) colour = sphere_fragment(a, atom, tri, b).colour;
    } else {
      const long long r = (long long)prim - sphere_prims;
      ribbon_triangle(a, r, t, ok);
      if (ok && cover(t, x, y, l, b)) {
        const float *v = a.ribbon_vertices + 12 * (3 * r);
        F3 c = f3(0.0f, 0.0f, 0.0f), n = f3(0.0f, 0.0f, 0.0f);
        c.x = (b[0] * v[4] + b[1] * v[16]) + b[2] * v[28];
        c.y = (b[0] * v[5] + b[1] * v[17]) + b[2] * v[29];
        c.z = (b[0] * v[6] + b[1] * v[18]) + b[2] * v[30];
        n.x = (b[0] * v[7] + b[1] * v[19]) + b[2] * v[31];
        n.y = (b[0] * v[8] + b[1] * v[20]) + b[2] * v[32];
        n.z = (b[0] * v[9] + b[1] * v[21]) + b[2] * v[33];
        const float facing = fabsf(dot3(normalize3(n), light_direction()));
        colour = mul(c, 0.26f + 0.74f * facing);
      }
    }
  }
  const float rgb[3] = {colour.x, colour.y, colour.z};
  uchar4 out;
  unsigned char u[3];
  for (int k = 0; k < 3; ++k) u[k] = (unsigned char)rintf(fminf(fmaxf(rgb[k], 0.0f), 1.0f) * 255.0f);
  out.x = u[0];
  out.y = u[1];
  out.z = u[2];
  out.w = 255;
  a.image[p] = out;
}

void launch_render(const RenderArgs &a, cudaStream_t stream) {
  const long long pixels = (long long)a.width * a.height;
  k_render_clear<<<(unsigned)((pixels + 255) / 256), 256, 0, stream>>>(a);
  if (a.draw_spheres && a.atom_count > 0) {
    k_sphere_vertices<<<(a.atom_count + 127) / 128, 128, 0, stream>>>(a);
    const long long warps = 2ll * a.atom_count;
    k_sphere_raster<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, stream>>>(a);
  }
  if (a.draw_ribbon && a.segment_count > 0) {
    const long long verts = 24ll * RIBBON_STEPS * a.segment_count;
    k_ribbon_vertices<<<(unsigned)((verts + 127) / 128), 128, 0, stream>>>(a);
    const long long warps = 8ll * RIBBON_STEPS * a.segment_count;
    k_ribbon_raster<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, stream>>>(a);
  }
  k_render_resolve<<<(unsigned)((pixels + 255) / 256), 256, 0, stream>>>(a);
}

}  // namespace rmd
