// kernels_render.cu — wavefront path tracing and general-scene ray casting.
//
// A wave of paths (up to the context's wave size, 2^22 by default) lives in SoA buffers. Each bounce runs three kernels over
// queues of path indices: extend (nearest hit), shade (emission, light sampling, BSDF
// sampling, Russian roulette; pushes the surviving paths to the next queue and at most one
// shadow ray per path to the shadow queue, both with one atomicAdd per warp) and shadow
// (any hit; adds the light sample's contribution when unoccluded). Radiance is added to a
// path in exactly the order PathIntegrator::li adds it (src/integrators/path.rs:55-113):
// emission, then the light sample, then the next vertex's emission or the background. At
// the end of a wave, accumulate adds every path's FP32 radiance into the FP64 film.
#include <cfloat>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "kernels.hpp"
#include "render.hpp"
#include "scene_device.cuh"

namespace pbrt {

constexpr float kPiF = 3.14159265358979323846f;
constexpr float kShadowEps = 0.00001f;  // SHADOW_RAY_EPSILON (src/lights.rs:21)
constexpr uint32_t kSpecularBit = 0x80000000u;

// ---- sampler: PCG32, one stream per pixel, re-keyed per (pixel, sample) ------------------
PBRT_DEV uint32_t pcg_next(unsigned long long& state, unsigned long long inc) {
  const unsigned long long old = state;
  state = old * 6364136223846793005ULL + inc;
  const uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
  const uint32_t rot = uint32_t(old >> 59u);
  return (xs >> rot) | (xs << ((32u - rot) & 31u));
}
PBRT_DEV float pcg_uniform(unsigned long long& state, unsigned long long inc) {
  return float(pcg_next(state, inc) >> 8) * (1.0f / 16777216.0f);
}
PBRT_DEV unsigned long long splitmix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
PBRT_DEV unsigned long long pcg_inc(uint32_t pixel) { return (((unsigned long long)pixel) << 1u) | 1u; }
PBRT_DEV unsigned long long pcg_seed(unsigned long long seed, uint32_t pixel, uint32_t sample) {
  const unsigned long long inc = pcg_inc(pixel);
  unsigned long long state = 0;
  pcg_next(state, inc);
  state += splitmix64(seed ^ splitmix64((((unsigned long long)pixel) << 32u) | sample));
  pcg_next(state, inc);
  return state;
}

// ---- warp-aggregated queue push ----------------------------------------------------------
PBRT_DEV uint32_t warp_push(uint32_t* count, bool want) {
  const unsigned mask = __activemask();
  const unsigned b = __ballot_sync(mask, want);
  if (!want) return 0;
  const int leader = __ffs(b) - 1;
  const unsigned lane = threadIdx.x & 31u;
  uint32_t base = 0;
  if (int(lane) == leader) base = atomicAdd(count, uint32_t(__popc(b)));
  base = __shfl_sync(b, base, leader);
  return base + __popc(b & ((1u << lane) - 1u));
}

// ---- lights -----------------------------------------------------------------------------------
PBRT_DEV F3 gradient(const LightRec& L, const F3& dir) {
  const float f = fm(0.5f, fa(dir.y, 1.f));
  const float g = fs(1.f, f);
  return mk3(fa(fm(L.bottom[0], g), fm(L.top[0], f)), fa(fm(L.bottom[1], g), fm(L.top[1], f)),
             fa(fm(L.bottom[2], g), fm(L.top[2], f)));
}

// Σ le over the infinite lights (path.rs:117-124)
PBRT_DEV F3 background(const SceneView& s, const F3& dir) {
  F3 res = mk3(0.f, 0.f, 0.f);
  for (uint32_t i = 0; i < s.light_count; ++i) {
    const LightRec& L = s.lights[i];
    if (L.kind == kLightBackground) res = add3(res, gradient(L, normalize3(dir)));
    else if (L.kind == kLightUniform) res = add3(res, mk3(L.rad[0], L.rad[1], L.rad[2]));
  }
  return res;
}

// SpherePdf::generate (pdfs/sphere.rs:10-23)
PBRT_DEV F3 sphere_dir(unsigned long long& st, unsigned long long inc) {
  const float two_pi = fm(2.f, kPiF);
  const float phi = fm(two_pi, pcg_uniform(st, inc));
  const float ct = fs(1.f, fm(2.f, pcg_uniform(st, inc)));
  const float sn = fsq(fs(1.f, fm(ct, ct)));
  return mk3(fm(cosf(phi), sn), fm(sinf(phi), sn), ct);
}

struct LiSample {
  F3 spectrum, wi, ro, rd;
  float pdf, dist;
};

PBRT_DEV bool sample_li(const SceneView& s, const LightRec& L, const Isect& it, unsigned long long& st,
                        unsigned long long inc, LiSample& out) {
  if (L.kind == kLightPoint) {  // point_light.rs:23-35, VisibilityTester::between (lights.rs:40-47)
    const F3 pos = mk3(L.pos[0], L.pos[1], L.pos[2]);
    const F3 wi = sub3(pos, it.p);
    const float sl = dot3(wi, wi);
    out.spectrum = mk3(fdv(L.rad[0], sl), fdv(L.rad[1], sl), fdv(L.rad[2], sl));
    out.wi = normalize3(wi);
    out.pdf = 1.f;
    out.ro = it.p;
    out.rd = normalize3(normalize3(sub3(pos, it.p)));
    out.dist = length3(sub3(pos, it.p));
    return true;
  }
  if (L.kind == kLightBackground || L.kind == kLightUniform) {  // towards_infinity (lights.rs:55-60)
    const F3 wi = sphere_dir(st, inc);
    out.pdf = fdv(1.f, fm(4.f, kPiF));
    out.spectrum = L.kind == kLightBackground ? gradient(L, wi) : mk3(L.rad[0], L.rad[1], L.rad[2]);
    out.wi = wi;
    out.ro = it.p;
    out.rd = normalize3(wi);
    out.dist = FLT_MAX;
    return true;
  }
  // area light: uniform on the emitter's area, p(ω) = p(A)·d²/|cos θ_l| (ideas/area_light.md §3)
  const ObjRec& ob = s.objects[L.object];
  F3 pl, nl;
  if (ob.shape == kShapeMesh) {
    const float u0 = fm(pcg_uniform(st, inc), L.area);
    // first triangle whose running area exceeds u0 (upper_bound)
    uint32_t lo = 0, hi = L.tri_count;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (s.light_cdf[L.tri_first + mid] <= u0) lo = mid + 1;
      else hi = mid;
    }
    const uint32_t t = lo < L.tri_count ? lo : L.tri_count - 1;
    const float su = fsq(pcg_uniform(st, inc));
    const float u2 = pcg_uniform(st, inc);
    const float b0 = fs(1.f, su), b1 = fm(u2, su);
    const float* tp = s.light_tris + 9 * size_t(L.tri_first + t);
    const F3 p0 = mk3(tp[0], tp[1], tp[2]), p1 = mk3(tp[3], tp[4], tp[5]), p2 = mk3(tp[6], tp[7], tp[8]);
    pl = add3(add3(mul3(p0, b0), mul3(p1, b1)), mul3(p2, fs(fs(1.f, b0), b1)));
    nl = normalize3(cross3(sub3(p2, p1), sub3(p1, p0)));
  } else {
    const F3 dir = sphere_dir(st, inc);
    const F3 lp = mul3(dir, ob.p[0]);
    pl = ob.xf_count ? xf_point(ob.to_world, lp) : lp;  // emitters sit under at most one transform
    nl = ob.xf_count ? normalize3(xf_normal(ob.to_local, dir)) : dir;
  }
  const F3 w = sub3(pl, it.p);
  const float d2 = dot3(w, w);
  const float dist = fsq(d2);
  const F3 wi = normalize3(w);
  const float cosl = fabsf(dot3(nl, wi));
  const float pdf = fdv(fm(fdv(1.f, L.area), d2), cosl);
  if (!(pdf > 0.f) || !isfinite(pdf)) return false;
  const MatRec& m = s.materials[ob.material];
  out.spectrum = mk3(m.color[0], m.color[1], m.color[2]);
  out.wi = wi;
  out.pdf = pdf;
  out.ro = it.p;
  out.rd = normalize3(wi);
  out.dist = fm(dist, fs(1.f, 1e-4f));
  return true;
}

// ---- materials --------------------------------------------------------------------------------
// Material::f (materials.rs:32-34, lambertian.rs:40-52)
PBRT_DEV F3 bsdf_f(const MatRec& m, const F3& alb, const F3& wo, const F3& wi, const Isect& it) {
  if (m.kind != kMatLambertian) return mk3(0.f, 0.f, 0.f);
  const F3 lwi = to_local(it, wi), lwo = to_local(it, wo);
  if (fm(lwo.z, lwi.z) > 0.f) return mk3(fdv(alb.x, kPiF), fdv(alb.y, kPiF), fdv(alb.z, kPiF));
  return mk3(0.f, 0.f, 0.f);
}

// random_in_unit_sphere (utils.rs:24-32), bounded at 64 draws
PBRT_DEV F3 in_unit_sphere(unsigned long long& st, unsigned long long inc) {
  F3 p = mk3(0.f, 0.f, 0.f);
  for (int k = 0; k < 64; ++k) {
    const float x = pcg_uniform(st, inc), y = pcg_uniform(st, inc), z = pcg_uniform(st, inc);
    p = mk3(fs(fm(x, 2.f), 1.f), fs(fm(y, 2.f), 1.f), fs(fm(z, 2.f), 1.f));
    if (dot3(p, p) < 1.f) return p;
  }
  return mul3(p, 0.5f);
}

struct ScatterOut {
  F3 att, ro, rd;
  float pdf;
};

PBRT_DEV bool scatter(const MatRec& m, const F3& col, const Isect& it, unsigned long long& st, unsigned long long inc,
                      ScatterOut& s) {
  if (m.kind == kMatLambertian) {  // lambertian.rs:24-38, pdfs/cosine.rs:10-24
    const float two_pi = fm(2.f, kPiF);
    const float phi = fm(two_pi, pcg_uniform(st, inc));
    const float r2 = pcg_uniform(st, inc);
    const float r2s = fsq(r2);
    const float ct = fsq(fs(1.f, r2));
    const F3 lwi = mk3(fm(cosf(phi), r2s), fm(sinf(phi), r2s), ct);
    const F3 wi = to_world(it, lwi);
    s.ro = add3(it.p, mul3(it.n, 0.001f));
    s.rd = normalize3(wi);
    s.att = mk3(fdv(col.x, kPiF), fdv(col.y, kPiF), fdv(col.z, kPiF));
    s.pdf = fabsf(fdv(lwi.z, kPiF));
    return true;
  }
  if (m.kind == kMatMetal) {  // metal.rs:22-59
    const F3 lwo = normalize3(to_local(it, it.wo));
    const F3 refl = mk3(-lwo.x, -lwo.y, lwo.z);
    const F3 tgt = normalize3(add3(refl, mul3(in_unit_sphere(st, inc), m.fuzz)));
    if (!(tgt.z > 0.f)) return false;
    const F3 w = to_world(it, tgt);
    s.ro = add3(it.p, mul3(it.n, 0.001f));
    s.rd = normalize3(w);
    const float ac = fabsf(tgt.z);
    s.att = mk3(fdv(col.x, ac), fdv(col.y, ac), fdv(col.z, ac));
    s.pdf = 1.f;
    return true;
  }
  if (m.kind == kMatDielectric) {  // dielectric.rs:32-182
    const F3 lwo = normalize3(to_local(it, it.wo));
    const F3 refl = mk3(-lwo.x, -lwo.y, lwo.z);
    F3 ln, wn;
    float ni, nt;
    if (lwo.z <= 0.f) { ln = mk3(0.f, 0.f, -1.f); wn = mul3(it.n, -1.f); ni = m.ior; nt = 1.f; }
    else { ln = mk3(0.f, 0.f, 1.f); wn = it.n; ni = 1.f; nt = m.ior; }
    const float nint = fdv(ni, nt);
    const float ci = dot3(lwo, ln);
    const float s2i = fs(1.f, fm(ci, ci));
    const float s2t = fm(fm(nint, nint), s2i);
    const float disc = fs(1.f, s2t);
    F3 ldir, origin;
    if (disc > 0.f) {
      const float ctt = fsq(disc);
      const F3 wi = mul3(lwo, -1.f);
      const F3 refr = normalize3(add3(mul3(wi, nint), mul3(ln, fs(fm(nint, ci), ctt))));
      const float n12 = fdv(ni, nt);
      const float cti = fm(lwo.z, ln.z);
      const float ctf = fsq(fs(1.f, fm(fm(n12, n12), fs(1.f, fm(cti, cti)))));
      const float ro = fdv(fs(fm(ni, cti), fm(nt, ctf)), fa(fm(ni, cti), fm(nt, ctf)));
      const float rp = fdv(fs(fm(nt, cti), fm(ni, ctf)), fa(fm(nt, cti), fm(ni, ctf)));
      const float reflectance = fm(fa(fm(ro, ro), fm(rp, rp)), 0.5f);
      if (pcg_uniform(st, inc) < reflectance) { ldir = refl; origin = add3(it.p, mul3(wn, 0.001f)); }
      else { ldir = refr; origin = add3(it.p, mul3(wn, -0.001f)); }
    } else {
      ldir = refl;
      origin = add3(it.p, mul3(wn, 0.001f));
    }
    s.ro = origin;
    s.rd = normalize3(to_world(it, ldir));
    const float ac = fabsf(ldir.z);
    s.att = mk3(fdv(col.x, ac), fdv(col.y, ac), fdv(col.z, ac));
    s.pdf = 1.f;
    return true;
  }
  return false;
}

// ---- the camera ------------------------------------------------------------------------------
// random_in_unit_disk (utils.rs:9-17): rejection on [-1, 1)^2, bounded at 64 draws
PBRT_DEV void in_unit_disk(unsigned long long& st, unsigned long long inc, float& x, float& y) {
  for (int k = 0; k < 64; ++k) {
    x = fs(fm(pcg_uniform(st, inc), 2.f), 1.f);
    y = fs(fm(pcg_uniform(st, inc), 2.f), 1.f);
    if (fa(fm(x, x), fm(y, y)) < 1.f) return;
  }
  x = fm(x, 0.5f);
  y = fm(y, 0.5f);
}

// PinHoleCamera::get_ray (pin_hole.rs:42-50): raster -> screen through the inverse
// perspective (w != 1 divides), normalise, camera -> world, Ray::new normalises again.
// ThinLensCamera::get_ray (thin_lens.rs:60-75): from a point of the lens disk through the
// pinhole ray's point at focal_distance / cv.z, both to world (the lens sample is drawn after
// the pixel jitter).
PBRT_DEV void camera_ray(const CameraRec& c, float px, float py, unsigned long long& st, unsigned long long inc,
                         F3& o, F3& d) {
  const float* m = c.raster_to_screen;
  F3 v = mk3(fa(fa(fa(fm(m[0], px), fm(m[1], py)), fm(m[2], 0.f)), m[3]),
             fa(fa(fa(fm(m[4], px), fm(m[5], py)), fm(m[6], 0.f)), m[7]),
             fa(fa(fa(fm(m[8], px), fm(m[9], py)), fm(m[10], 0.f)), m[11]));
  const float w = fa(fa(fa(fm(m[12], px), fm(m[13], py)), fm(m[14], 0.f)), m[15]);
  if (w != 1.f) v = mul3(v, frcp(w));
  const F3 cv = normalize3(v);
  if (!c.thin_lens) {
    o = xf_point(c.cam_to_world, mk3(0.f, 0.f, 0.f));
    d = normalize3(xf_dir(c.cam_to_world, cv));
    return;
  }
  const F3 rd = normalize3(cv);  // Ray::new(0, camera_vector)
  float lx, ly;
  in_unit_disk(st, inc, lx, ly);
  const F3 lens = mk3(fm(lx, c.lens_radius), fm(ly, c.lens_radius), 0.f);
  const float ft = fdv(c.focal_distance, cv.z);
  const F3 dir = normalize3(sub3(add3(mk3(0.f, 0.f, 0.f), mul3(rd, ft)), lens));  // ray.point_at(ft) - origin
  o = xf_point(c.cam_to_world, lens);
  d = normalize3(xf_dir(c.cam_to_world, dir));
}

// ---- the radiance cache's records ---------------------------------------------------------------
PBRT_DEV void write_record(float* rec, const F3& p, float rough, const F3& wo, const F3& n, const F3& alb) {
  float4* r = reinterpret_cast<float4*>(rec);
  r[0] = make_float4(p.x, p.y, p.z, rough);
  r[1] = make_float4(wo.x, wo.y, wo.z, 0.f);
  r[2] = make_float4(n.x, n.y, n.z, 0.f);
  r[3] = make_float4(alb.x, alb.y, alb.z, 0.f);
}

// ---- where a path's scene comes from ------------------------------------------------------------
// The wavefront kernels are written once over a scene source: one scene passed as a kernel
// parameter (pbrt_render, the cached render), or the batch table indexed by the path's scene.
struct PathSettings {
  uint32_t max_depth, rr_start, integrator;  // integrator: 0 path, 1 naive, 2 normal
  float near, far;
};

struct OneScene {
  SceneView v;
  PathSettings ps;
  PBRT_DEV const SceneView& view(const WaveBuffers&, uint32_t) const { return v; }
  PBRT_DEV PathSettings settings(const WaveBuffers&, uint32_t) const { return ps; }
};

struct ManyScenes {
  const BatchScene* b;
  PBRT_DEV const SceneView& view(const WaveBuffers& w, uint32_t p) const { return b[w.scene[p]].view; }
  PBRT_DEV PathSettings settings(const WaveBuffers& w, uint32_t p) const {
    const BatchScene& e = b[w.scene[p]];
    return PathSettings{e.max_depth, e.rr_start, e.integrator, e.cam.near, e.cam.far};
  }
};

// ---- kernels ---------------------------------------------------------------------------------
// A new path for image pixel `pixel`, sample `sample`: jitter, camera ray, fresh state.
PBRT_DEV void begin_path(const CameraRec& cam, unsigned long long seed, uint32_t pixel, uint32_t sample,
                         F3& o, F3& d, unsigned long long& st) {
  const unsigned long long inc = pcg_inc(pixel);
  st = pcg_seed(seed, pixel, sample);
  const float jx = pcg_uniform(st, inc), jy = pcg_uniform(st, inc);  // Sampler2::sample (mt.rs:145-150)
  camera_ray(cam, fa(float(pixel % cam.width), jx), fa(float(pixel / cam.width), jy), st, inc, o, d);
}

PBRT_DEV void start_path(const WaveBuffers& w, uint32_t i, const CameraRec& cam, unsigned long long seed,
                         uint32_t pixel, uint32_t sample) {
  F3 o, d;
  unsigned long long st;
  begin_path(cam, seed, pixel, sample, o, d, st);
  w.ox[i] = o.x; w.oy[i] = o.y; w.oz[i] = o.z;
  w.dx[i] = d.x; w.dy[i] = d.y; w.dz[i] = d.z;
  w.br[i] = 1.f; w.bg[i] = 1.f; w.bb[i] = 1.f;
  w.lr[i] = 0.f; w.lg[i] = 0.f; w.lb[i] = 0.f;
  w.rng[i] = st;
  w.pixel[i] = pixel;
  w.flags[i] = kSpecularBit;  // is_last_bounce_specular starts true (path.rs:52)
  w.qa[i] = i;
}

// The table entry holding path g of a batch frame: the last scene whose range starts at or
// before g (the table is in path order).
PBRT_DEV uint32_t batch_scene_of(const BatchScene* __restrict__ b, uint32_t nscenes, unsigned long long g) {
  uint32_t lo = 0, hi = nscenes - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (b[mid].begin <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Path g of a batch frame: its scene's pixel and sample (frame f takes samples
// sample_offset + f * spp ... of every pixel).
PBRT_DEV void batch_pixel_sample(const BatchScene& e, unsigned long long g, uint32_t f, uint32_t& pixel,
                                 uint32_t& sample) {
  const unsigned long long l = g - e.begin;
  const uint32_t q = uint32_t(l % e.npix);
  pixel = (q / e.film_w) * e.stride * e.cam.width + (q % e.film_w) * e.stride;
  sample = e.sample_offset + f * e.spp + uint32_t(l / e.npix);
}

__global__ void __launch_bounds__(256) k_generate(WaveBuffers w, CameraRec cam, uint64_t wave_base, uint32_t n,
                                                  uint32_t npix, uint32_t sample_offset, unsigned long long seed,
                                                  uint32_t random_pixels, uint32_t stride, uint32_t film_w,
                                                  unsigned long long* stats) {
  if (stats && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(stats + 2, (unsigned long long)n);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint64_t g = wave_base + i;
    const uint32_t q = uint32_t(g % npix);  // film pixel
    uint32_t pixel = (q / film_w) * stride * cam.width + (q % film_w) * stride;
    uint32_t sample = sample_offset + uint32_t(g / npix);
    if (random_pixels) {  // training paths: a pixel per path, the path's index keys its stream
      pixel = uint32_t(splitmix64(seed + g) % (unsigned long long)(cam.width * cam.height));
      sample = uint32_t(g);
    }
    start_path(w, i, cam, seed, pixel, sample);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) w.counts[0] = n;
}

__global__ void __launch_bounds__(256) k_generate_batch(WaveBuffers w, const BatchScene* __restrict__ b,
                                                        uint32_t nscenes, uint64_t wave_base, uint32_t n,
                                                        const uint32_t* __restrict__ frame, unsigned long long* stats) {
  if (stats && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(stats + 2, (unsigned long long)n);
  const uint32_t f = *frame;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned long long g = wave_base + i;
    const uint32_t lo = batch_scene_of(b, nscenes, g);
    const BatchScene& e = b[lo];
    uint32_t pixel, sample;
    batch_pixel_sample(e, g, f, pixel, sample);
    start_path(w, i, e.cam, e.seed, pixel, sample);
    w.scene[i] = lo;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) w.counts[0] = n;
}

// Scene::find_nearest for the queued paths, one thread per path (scene_closest). At least 4
// resident 256-thread blocks per SM (at most 64 registers a thread) for the traversal kernels:
// measured 2-4% faster than the compiler's 86 registers on the Cornell, many-spheres and
// torus-knot renders.
template <class Src, bool kCsg>
__global__ void __launch_bounds__(256, 4) k_extend(WaveBuffers w, Src src, const uint32_t* __restrict__ q,
                                                const uint32_t* __restrict__ qcount, uint32_t* err,
                                                unsigned long long* stats, uint32_t defer) {
  const uint32_t n = *qcount;
  if (stats && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(stats, (unsigned long long)n);
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const uint32_t p = q[k];
    const SceneView& s = src.view(w, p);
    const PathSettings ps = src.settings(w, p);
    const F3 o = mk3(w.ox[p], w.oy[p], w.oz[p]), d = mk3(w.dx[p], w.dy[p], w.dz[p]);
    float t = 0.f;
    uint32_t obj = 0xFFFFFFFFu, prim = 0;
    if (!scene_closest<kCsg>(s, o, d, ps.near, ps.far, t, obj, prim, err, defer ? s.defer_leaf : kNoLeaf))
      obj = 0xFFFFFFFFu;
    w.ht[p] = t;
    w.hobj[p] = obj;
    w.hprim[p] = prim;
  }
}

// Scene::find_nearest for the queued paths (scene_closest_t, visit for visit), restated as a
// persistent walk of the top-level BVH with one warp-voted step per iteration: a node step
// (or a pop) for the lanes not standing on a leaf, or, once at least `leaf_min` lanes stand on
// a leaf they must visit (or no lane has anything else to do), a leaf step for those; idle
// lanes take the next queued paths (one atomicAdd on `fetch` per warp) once at least
// `refill_min` of them are idle. Hit t / object / primitive are those of scene_closest: the
// same boxes, the same order, the same adoptions. It pays where the top-level tree is deep
// (10,000 spheres) and costs where a path's query is a few nodes (a 4-object box), hence
// kWalkMinTopNodes. At 2 resident blocks per SM it keeps its walk state in registers.
template <class Src, bool kCsg>
__global__ void __launch_bounds__(256, 2) k_extend_walk(WaveBuffers w, Src src, const uint32_t* __restrict__ q,
                                                     const uint32_t* __restrict__ qcount, uint32_t* __restrict__ fetch,
                                                     uint32_t* err, unsigned long long* stats, int leaf_min,
                                                     int refill_min, uint32_t defer) {
  const uint32_t n = *qcount;
  if (stats && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(stats, (unsigned long long)n);
  const unsigned lane = threadIdx.x & 31u, lt_mask = (1u << lane) - 1u;
  bool active = false, exhausted = false;  // exhausted is warp-uniform
  uint32_t p = 0;
  F3 o = mk3(0.f, 0.f, 0.f), d = o;
  PRay r;
  float near = 0.f, min_t = 0.f, cur_e = 0.f;
  bool have = false;
  uint32_t leaf_out = 0, prim_out = 0, lf = 0, count = 0, budget = 0;
  int sp = 0;
  uint32_t stk_lf[kTraceStack], stk_cnt[kTraceStack];
  float stk_e[kTraceStack];
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (!exhausted && idle && (__popc(idle) >= refill_min || idle == 0xffffffffu)) {
      const int leader = __ffs(idle) - 1;
      uint32_t base = 0;
      if (int(lane) == leader) base = atomicAdd(fetch, uint32_t(__popc(idle)));
      base = __shfl_sync(0xffffffffu, base, leader);
      exhausted = uint64_t(base) + __popc(idle) >= n;
      const uint64_t k = uint64_t(base) + __popc(idle & lt_mask);
      if (!active && k < n) {
        p = q[k];
        const SceneView& s = src.view(w, p);
        const PathSettings ps = src.settings(w, p);
        o = mk3(w.ox[p], w.oy[p], w.oz[p]);
        d = mk3(w.dx[p], w.dy[p], w.dz[p]);
        near = ps.near;
        min_t = ps.far;
        have = false;
        prim_out = 0;
        for (uint32_t u = 0; u < s.unbounded_count; ++u) {  // nearest_among + closer (scene.rs:222-249)
          float t;
          uint32_t leaf, prim;
          if (prim_closest<kCsg>(s, __ldg(&s.unbounded[u]), o, d, near, ps.far, t, leaf, prim, err) &&
              (!have || t < min_t)) {
            have = true;
            min_t = t;
            leaf_out = leaf;
            prim_out = prim;
          }
        }
        bool walk = false;
        if (s.top_node_count != 0) {
          r = prepare_ray(o, d);
          const float4 rlo = __ldg(&s.top[0]);
          const float4 rhi = __ldg(&s.top[1]);
          float entry;
          if (box_hit(r, rlo, rhi, near, min_t, entry)) {
            lf = __float_as_uint(rlo.w);
            count = __float_as_uint(rhi.w);
            cur_e = entry;
            sp = 0;
            budget = 2u * s.top_node_count + 2u;  // every node is pushed (and popped) at most once
            walk = true;
          }
        }
        if (walk) {
          active = true;
        } else {
          w.ht[p] = have ? min_t : 0.f;
          w.hobj[p] = have ? leaf_out : 0xFFFFFFFFu;
          w.hprim[p] = prim_out;
        }
      }
    }
    const unsigned act = __ballot_sync(0xffffffffu, active);
    if (act == 0) {
      if (exhausted) break;
      continue;  // all idle and the queue not yet drained: the next iteration refills
    }
    const bool at_leaf = active && cur_e < min_t && count > 0;  // a leaf this lane must visit
    const unsigned on_leaf = __ballot_sync(0xffffffffu, at_leaf);
    const bool leaf_step = __popc(on_leaf) >= leaf_min || on_leaf == act;
    bool done = false;
    if (active && at_leaf == leaf_step) {
      const SceneView& s = src.view(w, p);
      if (budget-- == 0) {
        atomicOr(err, kErrBudget);
        done = true;
      } else if (leaf_step) {
        // A leaf: its primitives over [near, min_t], a candidate adopted only when strictly nearer.
        for (uint32_t k = lf; k < lf + count; ++k) {
          const uint32_t ref = __ldg(&s.order[k]);
          if (defer && ref == s.defer_leaf) continue;  // answered by k_defer_closest
          float t;
          uint32_t leaf, prim;
          if (prim_closest<kCsg>(s, ref, o, d, near, min_t, t, leaf, prim, err) && (!have || t < min_t)) {
            have = true;
            min_t = t;
            leaf_out = leaf;
            prim_out = prim;
          }
        }
        if (sp == 0) {
          done = true;
        } else {
          --sp;
          lf = stk_lf[sp];
          count = stk_cnt[sp];
          cur_e = stk_e[sp];
        }
      } else {
        // One node of the walk: an interior node's children (the farther pushed, the nearer
        // taken), or a pop when the current entry is dropped (>= min_t) or no child was hit.
        bool pop = true;
        if (cur_e < min_t) {
          float4 l0, l1, r0, r1;
          load_node(&s.top[2 * lf], l0, l1);
          load_node(&s.top[2 * lf + 2], r0, r1);
          float dl, dr;
          const bool hl = box_hit(r, l0, l1, near, min_t, dl);
          const bool hr = box_hit(r, r0, r1, near, min_t, dr);
          const bool swap = hl && hr && dr < dl;
          const bool hn = swap ? hr : hl, hf = swap ? hl : hr;
          const float dn = swap ? dr : dl, df = swap ? dl : dr;
          if (hf) {
            if (sp >= kTraceStack) {
              atomicOr(err, kErrStack);
              done = true;
            } else {
              stk_lf[sp] = __float_as_uint(swap ? l0.w : r0.w);
              stk_cnt[sp] = __float_as_uint(swap ? l1.w : r1.w);
              stk_e[sp] = df;
              ++sp;
            }
          }
          if (hn) {
            lf = __float_as_uint(swap ? r0.w : l0.w);
            count = __float_as_uint(swap ? r1.w : l1.w);
            cur_e = dn;
            pop = false;
          }
        }
        if (pop && !done) {
          if (sp == 0) {
            done = true;
          } else {
            --sp;
            lf = stk_lf[sp];
            count = stk_cnt[sp];
            cur_e = stk_e[sp];
          }
        }
      }
    }
    if (done) {
      w.ht[p] = have ? min_t : 0.f;  // the adopted hit's distance (min_t = c.d)
      w.hobj[p] = have ? leaf_out : 0xFFFFFFFFu;
      w.hprim[p] = prim_out;
      active = false;
    }
  }
}

// kStage: the path and shadow queues are pushed per block instead of per warp: a block-wide
// scan of the warps' ballots and one atomicAdd per block and queue, the path indices written
// as one contiguous run, and the shadow records (11 planes) staged in shared memory and
// copied out as one contiguous SoA run per block (thread t writes entry t of each plane).
// One path vertex of PathIntegrator::li (path.rs:48-115): the hit (obj 0xFFFFFFFF: the
// background) of the path's ray, its emission, the light sample (a shadow ray to trace, with
// the contribution it adds if unoccluded), the BSDF sample and Russian roulette. `P` is updated
// in place (radiance always; ray, throughput, stream and flags when the path goes on: alive).
// With the cache on, a cacheable vertex's record is returned and the path may end into it.
struct PathState {
  F3 o, d, beta, L;
  unsigned long long st;
  uint32_t pixel, flags;  // flags: bounce count | kSpecularBit
};

struct VertexOut {
  bool alive = false, shadow = false, query = false, train = false;
  F3 sro, srd, contrib;
  float stmax = 0.f;
  F3 cp, cwo, cn, calb, cL, cB;  // the cache record of this vertex
  float crough = 0.f;
};

PBRT_DEV void shade_vertex(const SceneView& s, const PathSettings& ps, PathState& P, uint32_t obj, uint32_t prim,
                           float t, uint32_t cache_mode, uint32_t term_hit, VertexOut& v) {
  const uint32_t max_depth = ps.max_depth, rr_start = ps.rr_start, naive = ps.integrator;
  const bool normal_only = ps.integrator == 2u;
  F3 o = P.o, d = P.d;
  F3 beta = P.beta;
  F3 L = P.L;
  unsigned long long st = P.st;
  const unsigned long long inc = pcg_inc(P.pixel);
  uint32_t flags = P.flags;
  const bool spec = naive || (flags & kSpecularBit);
  uint32_t bounce = flags & 0xFFFFu;
  bool alive = false;
  if (obj == 0xFFFFFFFFu) {
    if (spec && !normal_only) {  // NormalIntegrator's background is black (integrators.rs:9-11)
      const F3 bg = background(s, d);
      L = add3(L, mk3(fm(bg.x, beta.x), fm(bg.y, beta.y), fm(bg.z, beta.z)));
    }
  } else {
    const MatRec m = s.materials[material_index(s, obj, prim)];
    const Isect it = interaction(s, obj, prim, o, d, t, m.texture != kTexColor);
    const F3 alb = texel(m, it);  // albedo, or emitted radiance (DiffuseLight::emit)
    if (normal_only) {  // NormalIntegrator::li (normal.rs:17-27): (n + (1, 1, 1)) * 0.5, one hit
      const F3 nn = add3(it.n, mk3(1.f, 1.f, 1.f));
      L = mul3(nn, 0.5f);
      bounce = max_depth - 1u;  // the hit ends the path
    }
    if (spec && !normal_only && m.kind == kMatDiffuseLight)
      L = add3(L, mk3(fm(alb.x, beta.x), fm(alb.y, beta.y), fm(alb.z, beta.z)));
    bounce++;
    // PathIntegrator stops at the max_depth-th hit, before sampling a light (path.rs:64-67);
    // the naive estimator also ends there, its emission counted: after max_depth hits its
    // recursion reaches li(.., 0), which is black (naive.rs:29-52). Paths of every scene of
    // a batch stop at their own depth, whatever the number of bounce launches.
    const bool depth_cut = bounce == max_depth;
    const bool cacheable = m.kind == kMatLambertian || m.kind == kMatMetal;
    if (!depth_cut && cacheable && cache_mode != kCacheOff) {
      v.cp = it.p;
      v.cwo = mul3(d, -1.f);
      v.cn = dot3(it.n, v.cwo) < 0.f ? mul3(it.n, -1.f) : it.n;
      v.calb = alb;
      v.crough = m.kind == kMatMetal ? m.fuzz : 1.f;
      v.cL = L;
      v.cB = beta;
      v.query = bounce >= term_hit;  // the path ends here, into the cache
      v.train = cache_mode == kCacheRecord && !v.query;
    }
    if (!depth_cut && !v.query) {
      if (!naive && s.light_count > 0) {  // sample_light (path.rs:31-44) and the light sample
        const float cnt = float(s.light_count);
        const float pick = fminf(fm(pcg_uniform(st, inc), cnt), fs(cnt, 1.f));
        const uint32_t li = uint32_t(pick);
        const float pl = fdv(1.f, cnt);
        LiSample ls;
        if (sample_li(s, s.lights[li], it, st, inc, ls)) {
          const F3 f0 = bsdf_f(m, alb, mul3(d, -1.f), ls.wi, it);
          const float ac = fabsf(dot3(ls.wi, it.n));
          const F3 f = mk3(fm(f0.x, ac), fm(f0.y, ac), fm(f0.z, ac));
          if (f.x != 0.f || f.y != 0.f || f.z != 0.f) {
            const float den = fm(pl, ls.pdf);
            v.contrib = mk3(fdv(fm(fm(ls.spectrum.x, f.x), beta.x), den),
                            fdv(fm(fm(ls.spectrum.y, f.y), beta.y), den),
                            fdv(fm(fm(ls.spectrum.z, f.z), beta.z), den));
            v.sro = ls.ro;
            v.srd = ls.rd;
            v.stmax = ls.dist;
            v.shadow = true;
          }
        }
      }
      ScatterOut sc;
      if (scatter(m, alb, it, st, inc, sc)) {
        const float ac = fabsf(dot3(sc.rd, it.n));
        const F3 kk = mk3(fdv(fm(sc.att.x, ac), sc.pdf), fdv(fm(sc.att.y, ac), sc.pdf), fdv(fm(sc.att.z, ac), sc.pdf));
        beta = mk3(fm(beta.x, kk.x), fm(beta.y, kk.y), fm(beta.z, kk.z));
        o = sc.ro;
        d = sc.rd;
        const bool sp = m.kind == kMatMetal || m.kind == kMatDielectric;
        alive = true;
        if (rr_start && bounce >= rr_start) {  // Russian roulette (path.rs:92-101, q clamped to 1)
          const float qq = fminf(1.f, fmaxf(fmaxf(beta.x, beta.y), beta.z));
          if (pcg_uniform(st, inc) > qq) {
            alive = false;
          } else {
            const float iq = frcp(qq);
            beta = mul3(beta, iq);
          }
        }
        flags = (sp ? kSpecularBit : 0u) | bounce;
      }
    }
  }
  P.L = L;
  v.alive = alive;
  if (alive) {
    P.o = o;
    P.d = d;
    P.beta = beta;
    P.st = st;
    P.flags = flags;
  }
}

template <class Src, bool kStage>
__global__ void __launch_bounds__(256) k_shade(WaveBuffers w, Src src, const uint32_t* __restrict__ q,
                                               const uint32_t* __restrict__ qcount, uint32_t* __restrict__ qout,
                                               uint32_t* __restrict__ qout_count, CacheWave cw, uint32_t cache_mode,
                                               uint32_t term_hit) {
  constexpr int kMaxThreads = 256, kMaxWarps = kMaxThreads / 32;
  __shared__ uint32_t st_off[2][kMaxWarps], st_base[2], st_total[2];
  __shared__ uint32_t st_path[kStage ? kMaxThreads : 1];
  __shared__ float st_rec[kStage ? 10 : 1][kStage ? kMaxThreads : 1];
  const uint32_t n = *qcount;
  // every lane runs the same trip count so the warp-aggregated pushes see full warps
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t iters = (n + stride - 1) / stride;
  for (uint32_t it_ = 0; it_ < iters; ++it_) {
    const uint32_t k = it_ * stride + blockIdx.x * blockDim.x + threadIdx.x;
    bool push_path = false, push_shadow = false, push_query = false, push_train = false;
    uint32_t p = 0;
    F3 sro, srd, contrib;
    float stmax = 0.f;
    F3 cp, cwo, cn, calb, cL, cB;  // the cache record of this vertex
    float crough = 0.f;
    if (k < n) {
      p = q[k];
      const SceneView& s = src.view(w, p);
      const PathSettings ps = src.settings(w, p);
      PathState P;
      P.o = mk3(w.ox[p], w.oy[p], w.oz[p]);
      P.d = mk3(w.dx[p], w.dy[p], w.dz[p]);
      P.beta = mk3(w.br[p], w.bg[p], w.bb[p]);
      P.L = mk3(w.lr[p], w.lg[p], w.lb[p]);
      P.st = w.rng[p];
      P.pixel = w.pixel[p];
      P.flags = w.flags[p];
      VertexOut v;
      shade_vertex(s, ps, P, w.hobj[p], w.hprim[p], w.ht[p], cache_mode, term_hit, v);
      push_shadow = v.shadow;
      push_query = v.query;
      push_train = v.train;
      sro = v.sro; srd = v.srd; contrib = v.contrib; stmax = v.stmax;
      cp = v.cp; cwo = v.cwo; cn = v.cn; calb = v.calb; cL = v.cL; cB = v.cB; crough = v.crough;
      w.lr[p] = P.L.x; w.lg[p] = P.L.y; w.lb[p] = P.L.z;
      if (v.alive) {
        w.ox[p] = P.o.x; w.oy[p] = P.o.y; w.oz[p] = P.o.z;
        w.dx[p] = P.d.x; w.dy[p] = P.d.y; w.dz[p] = P.d.z;
        w.br[p] = P.beta.x; w.bg[p] = P.beta.y; w.bb[p] = P.beta.z;
        w.rng[p] = P.st;
        w.flags[p] = P.flags;
        push_path = true;
      }
    }
    if (kStage) {
      const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, lt = (1u << lane) - 1u;
      const unsigned bp = __ballot_sync(0xffffffffu, push_path), bs = __ballot_sync(0xffffffffu, push_shadow);
      if (lane == 0) {
        st_off[0][warp] = __popc(bp);
        st_off[1][warp] = __popc(bs);
      }
      __syncthreads();
      if (threadIdx.x < 2) {  // exclusive scan over the warps, one atomicAdd per queue
        uint32_t run = 0;
        for (uint32_t v = 0; v < blockDim.x / 32u; ++v) {
          const uint32_t c = st_off[threadIdx.x][v];
          st_off[threadIdx.x][v] = run;
          run += c;
        }
        st_total[threadIdx.x] = run;
        st_base[threadIdx.x] = run ? atomicAdd(threadIdx.x == 0 ? qout_count : w.counts + 2, run) : 0u;
      }
      __syncthreads();
      if (push_path) qout[st_base[0] + st_off[0][warp] + __popc(bp & lt)] = p;
      if (push_shadow) {
        const uint32_t slot = st_off[1][warp] + __popc(bs & lt);
        st_path[slot] = p;
        st_rec[0][slot] = sro.x; st_rec[1][slot] = sro.y; st_rec[2][slot] = sro.z;
        st_rec[3][slot] = srd.x; st_rec[4][slot] = srd.y; st_rec[5][slot] = srd.z;
        st_rec[6][slot] = stmax;
        st_rec[7][slot] = contrib.x; st_rec[8][slot] = contrib.y; st_rec[9][slot] = contrib.z;
      }
      __syncthreads();
      const uint32_t total = st_total[1], base = st_base[1];
      for (uint32_t t = threadIdx.x; t < total; t += blockDim.x) {
        const uint32_t si = base + t;
        w.s_path[si] = st_path[t];
        w.s_ox[si] = st_rec[0][t]; w.s_oy[si] = st_rec[1][t]; w.s_oz[si] = st_rec[2][t];
        w.s_dx[si] = st_rec[3][t]; w.s_dy[si] = st_rec[4][t]; w.s_dz[si] = st_rec[5][t];
        w.s_tmax[si] = st_rec[6][t];
        w.s_cr[si] = st_rec[7][t]; w.s_cg[si] = st_rec[8][t]; w.s_cb[si] = st_rec[9][t];
      }
      __syncthreads();  // the staging arrays are reused by the next iteration
    } else {
      const uint32_t qi = warp_push(qout_count, push_path);
      if (push_path) qout[qi] = p;
      const uint32_t si = warp_push(w.counts + 2, push_shadow);
      if (push_shadow) {
        w.s_path[si] = p;
        w.s_ox[si] = sro.x; w.s_oy[si] = sro.y; w.s_oz[si] = sro.z;
        w.s_dx[si] = srd.x; w.s_dy[si] = srd.y; w.s_dz[si] = srd.z;
        w.s_tmax[si] = stmax;
        w.s_cr[si] = contrib.x; w.s_cg[si] = contrib.y; w.s_cb[si] = contrib.z;
      }
    }
    if (cache_mode != kCacheOff) {  // uniform over the grid, so the pushes see whole warps
      const uint32_t ci = warp_push(cw.counts, push_query);
      if (push_query && ci < cw.qcap) {  // at most one query per path, and qcap covers the wave
        write_record(cw.qrec + size_t(ci) * kCacheRecordFloats, cp, crough, cwo, cn, calb);
        cw.qpath[ci] = p;
      }
      const uint32_t ti = warp_push(cw.counts + 1, push_train);
      if (push_train && ti < cw.tcap) {
        write_record(cw.trec + size_t(ti) * kCacheRecordFloats, cp, crough, cwo, cn, calb);
        float* ts = cw.tstate + 6 * size_t(ti);
        ts[0] = cL.x; ts[1] = cL.y; ts[2] = cL.z;
        ts[3] = cB.x; ts[4] = cB.y; ts[5] = cB.z;
        cw.tpath[ti] = p;
      }
    }
  }
}

// The network's answer, clamped to [0, the scene's largest emitted radiance].
PBRT_DEV float cache_value(float o, float max_l) { return fminf(fmaxf(o, 0.f), max_l); }

__global__ void __launch_bounds__(256) k_apply_cache(WaveBuffers w, CacheWave cw, uint32_t paths, float max_l) {
  const uint32_t n = min(cw.counts[0], cw.qcap);
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const uint32_t p = cw.qpath[k];
    if (p >= paths) continue;
    const float* o = cw.qout + 3 * size_t(k);
    w.lr[p] = fa(w.lr[p], fm(w.br[p], cache_value(o[0], max_l)));
    w.lg[p] = fa(w.lg[p], fm(w.bg[p], cache_value(o[1], max_l)));
    w.lb[p] = fa(w.lb[p], fm(w.bb[p], cache_value(o[2], max_l)));
  }
}

__global__ void __launch_bounds__(256) k_train_batch(WaveBuffers w, CacheWave cw, uint32_t batch, uint32_t step,
                                                     unsigned long long seed, float max_l, float* __restrict__ rec,
                                                     float* __restrict__ tgt) {
  const uint32_t m = min(cw.counts[1], cw.tcap);
  if (blockIdx.x == 0 && threadIdx.x == 0) cw.counts[2] = m > 0 ? 1u : 0u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < batch; i += gridDim.x * blockDim.x) {
    if (m == 0) {
      float4* dst = reinterpret_cast<float4*>(rec + size_t(i) * kCacheRecordFloats);
      dst[0] = dst[1] = dst[2] = dst[3] = make_float4(0.f, 0.f, 0.f, 0.f);
      tgt[3 * size_t(i)] = tgt[3 * size_t(i) + 1] = tgt[3 * size_t(i) + 2] = 0.f;
      continue;
    }
    const uint32_t j = uint32_t(splitmix64(seed ^ ((((unsigned long long)step) << 32) | i)) % m);
    const float4* src = reinterpret_cast<const float4*>(cw.trec + size_t(j) * kCacheRecordFloats);
    float4* dst = reinterpret_cast<float4*>(rec + size_t(i) * kCacheRecordFloats);
    dst[0] = src[0]; dst[1] = src[1]; dst[2] = src[2]; dst[3] = src[3];
    const uint32_t p = cw.tpath[j];
    const float* ts = cw.tstate + 6 * size_t(j);
    const float le[3] = {w.lr[p], w.lg[p], w.lb[p]};
    for (int c = 0; c < 3; ++c) {
      const float b = ts[3 + c];
      tgt[3 * size_t(i) + c] = b > 0.f ? cache_value(fdv(fs(le[c], ts[c]), b), max_l) : 0.f;
    }
  }
}

// 3 resident blocks per SM (the torus-knot frame 54.1 -> 52.9 ms against 4; 2 gained nothing
// more; with the solids' code, 48 of 770 bytes still spill).
// With `defer`, a scene's deferred leaf is left out: an occluded entry is resolved (its t_max
// set to -1), an unoccluded one of a scene without a deferred leaf adds its light sample and
// is resolved, and the others wait for k_defer_any.
template <class Src, bool kCsg>
__global__ void __launch_bounds__(256, 3) k_shadow(WaveBuffers w, Src src, uint32_t* err, unsigned long long* stats,
                                                uint32_t defer) {
  const uint32_t n = w.counts[2];
  if (stats && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(stats + 1, (unsigned long long)n);
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const uint32_t p = w.s_path[k];
    const SceneView& s = src.view(w, p);
    const F3 o = mk3(w.s_ox[k], w.s_oy[k], w.s_oz[k]), d = mk3(w.s_dx[k], w.s_dy[k], w.s_dz[k]);
    const uint32_t skip = defer ? s.defer_leaf : kNoLeaf;
    if (scene_any<kCsg>(s, o, d, kShadowEps, w.s_tmax[k], err, skip)) {
      if (defer) w.s_tmax[k] = -1.f;
    } else if (skip == kNoLeaf) {  // VisibilityTester::unoccluded (lights.rs:67-69)
      w.lr[p] = fa(w.lr[p], w.s_cr[k]);
      w.lg[p] = fa(w.lg[p], w.s_cg[k]);
      w.lb[p] = fa(w.lb[p], w.s_cb[k]);
      if (defer) w.s_tmax[k] = -1.f;
    }
  }
}

// ---- the deferred leaf ----------------------------------------------------------------------
// Resident 128-thread blocks per SM the deferred passes are compiled for (8: at most 64
// registers a thread).
#ifndef PBRT_DEFER_MIN_BLOCKS
#define PBRT_DEFER_MIN_BLOCKS 8
#endif

// A scene's largest mesh, when it is placed untransformed in the top-level tree, is left out
// of the per-path queries above and answered here for all queued paths at once by persistent
// warps over the paths (the ray-cast kernel's while-while schedule: idle lanes refilled with
// one atomicAdd per warp, interior nodes walked until every lane stands on a leaf, the leaves
// of all lanes tested in one pass). Each lane walks its own scene's mesh (batches mix scenes).
//
// Nearest hit: the mesh is offered [near, nearest hit so far] and its hit adopted only when
// strictly nearer, which is what Scene::find_nearest does with it wherever it comes in the
// top-level order (scene.rs:186-220); an object's own answer does not depend on the interval
// it is offered as long as its hit lies inside, so the result is the per-path query's, up to
// which of two objects hit at exactly the same distance is kept.
template <class Src>
__global__ void __launch_bounds__(128, PBRT_DEFER_MIN_BLOCKS) k_defer_closest(WaveBuffers w, Src src, const uint32_t* __restrict__ q,
                                                       const uint32_t* __restrict__ qcount,
                                                       uint32_t* __restrict__ fetch, uint32_t* err) {
  const uint32_t n = *qcount;
  const unsigned lane = threadIdx.x & 31u, lt_mask = (1u << lane) - 1u;
  bool active = false;
  uint32_t p = 0, leaf = 0, best = 0xFFFFFFFFu, lf = 0, count = 0, budget = 0;
  MeshView m{};
  PRay r;
  float near = 0.f, far = 0.f, min_t = FLT_MAX;
  bool have = false;
  int sp = 0;
  uint32_t stk_lf[kTraceStack], stk_cnt[kTraceStack];
  float stk_e[kTraceStack];
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    bool exhausted = false;
    if (idle) {
      const int leader = __ffs(idle) - 1;
      uint32_t base = 0;
      if (int(lane) == leader) base = atomicAdd(fetch, uint32_t(__popc(idle)));
      base = __shfl_sync(0xffffffffu, base, leader);
      exhausted = uint64_t(base) + __popc(idle) >= n;
      const uint64_t k = uint64_t(base) + __popc(idle & lt_mask);
      if (!active && k < n) {
        p = q[k];
        const SceneView& s = src.view(w, p);
        leaf = s.defer_leaf;
        if (leaf != kNoLeaf) {
          const PathSettings ps = src.settings(w, p);
          m = s.meshes[s.objects[leaf].mesh];
          r = prepare_ray(mk3(w.ox[p], w.oy[p], w.oz[p]), mk3(w.dx[p], w.dy[p], w.dz[p]));
          near = ps.near;
          have = w.hobj[p] != 0xFFFFFFFFu;
          far = have ? w.ht[p] : ps.far;
          const float4 rlo = __ldg(&m.nodes[0]);
          const float4 rhi = __ldg(&m.nodes[1]);
          float entry;
          // the root is pushed, then dropped at pop if its entry is >= min_t = FLT_MAX (bvh.rs:462-472)
          if (box_hit(r, rlo, rhi, near, far, entry) && entry < FLT_MAX) {
            lf = __float_as_uint(rlo.w);
            count = __float_as_uint(rhi.w);
            min_t = FLT_MAX;
            best = 0xFFFFFFFFu;
            sp = 0;
            budget = m.node_count;
            active = true;
          }
        }
      }
    }
    if (__ballot_sync(0xffffffffu, active) == 0) {
      if (exhausted) break;
      continue;
    }
    if (active) {
      bool done = false;
      while (count == 0) {  // interior nodes until this lane stands on a leaf
        if (budget-- == 0) {
          atomicOr(err, kErrBudget);
          done = true;
          break;
        }
        float4 l0, l1, r0, r1;
        load_node(&m.nodes[2 * lf], l0, l1);
        load_node(&m.nodes[2 * lf + 2], r0, r1);
        float dl, dr;
        const bool hl = box_hit(r, l0, l1, near, far, dl);
        const bool hr = box_hit(r, r0, r1, near, far, dr);
        const bool swap = hl && hr && dr < dl;  // right first only when strictly nearer
        const bool hn = swap ? hr : hl, hf = swap ? hl : hr;
        const float dn = swap ? dr : dl, df = swap ? dl : dr;
        const bool take_f = hf && df < min_t, take_n = hn && dn < min_t;
        if (take_n) {
          if (take_f) {
            if (sp >= kTraceStack) {
              atomicOr(err, kErrStack);
              done = true;
              break;
            }
            stk_lf[sp] = __float_as_uint(swap ? l0.w : r0.w);
            stk_cnt[sp] = __float_as_uint(swap ? l1.w : r1.w);
            stk_e[sp] = df;
            ++sp;
          }
          lf = __float_as_uint(swap ? r0.w : l0.w);
          count = __float_as_uint(swap ? r1.w : l1.w);
        } else if (take_f) {
          lf = __float_as_uint(swap ? l0.w : r0.w);
          count = __float_as_uint(swap ? l1.w : r1.w);
        } else {
          bool found = false;  // pop, dropping entries at or beyond the nearest hit (bvh.rs:470-472)
          while (sp > 0) {
            --sp;
            if (stk_e[sp] < min_t) {
              lf = stk_lf[sp];
              count = stk_cnt[sp];
              found = true;
              break;
            }
          }
          if (!found) {
            done = true;
            break;
          }
        }
      }
      if (!done) {  // the leaves of every lane standing on one
        if (budget-- == 0) {
          atomicOr(err, kErrBudget);
          done = true;
        } else {
          for (uint32_t k = lf; k < lf + count; ++k) {
            const float4 A = __ldg(&m.tri_a[k]);
            const float4 B = __ldg(&m.tri_b[k]);
            const float2 C = __ldg(&m.tri_c[k]);
            float t;
            if (tri_hit(r, A, B, C.x, t) && t < min_t && t >= near && t <= far) {
              min_t = t;
              best = __float_as_uint(C.y);
            }
          }
          bool found = false;
          while (sp > 0) {
            --sp;
            if (stk_e[sp] < min_t) {
              lf = stk_lf[sp];
              count = stk_cnt[sp];
              found = true;
              break;
            }
          }
          if (!found) done = true;
        }
      }
      if (done) {
        if (best != 0xFFFFFFFFu && (!have || min_t < far)) {  // adopted only when strictly nearer
          w.ht[p] = min_t;
          w.hobj[p] = leaf;
          w.hprim[p] = best;
        }
        active = false;
      }
    }
  }
}

// Shadow rays against the deferred leaf: the entries k_shadow left open (t_max >= 0) add their
// light sample when the mesh does not block [kShadowEps, t_max]; any hit ends the walk.
template <class Src>
__global__ void __launch_bounds__(128, PBRT_DEFER_MIN_BLOCKS) k_defer_any(WaveBuffers w, Src src, uint32_t* __restrict__ fetch,
                                                   uint32_t* err) {
  const uint32_t n = w.counts[2];
  const unsigned lane = threadIdx.x & 31u, lt_mask = (1u << lane) - 1u;
  bool active = false;
  uint32_t k = 0, p = 0, lf = 0, count = 0, budget = 0;
  MeshView m{};
  PRay r;
  float far = 0.f;
  int sp = 0;
  uint32_t stk_lf[kTraceStack], stk_cnt[kTraceStack];
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    bool exhausted = false;
    if (idle) {
      const int leader = __ffs(idle) - 1;
      uint32_t base = 0;
      if (int(lane) == leader) base = atomicAdd(fetch, uint32_t(__popc(idle)));
      base = __shfl_sync(0xffffffffu, base, leader);
      exhausted = uint64_t(base) + __popc(idle) >= n;
      const uint64_t kk = uint64_t(base) + __popc(idle & lt_mask);
      if (!active && kk < n) {
        k = uint32_t(kk);
        far = w.s_tmax[k];
        if (far >= 0.f) {  // still open
          p = w.s_path[k];
          const SceneView& s = src.view(w, p);
          m = s.meshes[s.objects[s.defer_leaf].mesh];
          r = prepare_ray(mk3(w.s_ox[k], w.s_oy[k], w.s_oz[k]), mk3(w.s_dx[k], w.s_dy[k], w.s_dz[k]));
          const float4 rlo = __ldg(&m.nodes[0]);
          const float4 rhi = __ldg(&m.nodes[1]);
          float entry;
          if (box_hit(r, rlo, rhi, kShadowEps, far, entry)) {
            lf = __float_as_uint(rlo.w);
            count = __float_as_uint(rhi.w);
            sp = 0;
            budget = m.node_count;
            active = true;
          } else {  // misses the mesh: unoccluded
            w.lr[p] = fa(w.lr[p], w.s_cr[k]);
            w.lg[p] = fa(w.lg[p], w.s_cg[k]);
            w.lb[p] = fa(w.lb[p], w.s_cb[k]);
          }
        }
      }
    }
    if (__ballot_sync(0xffffffffu, active) == 0) {
      if (exhausted) break;
      continue;
    }
    if (active) {
      bool done = false, hit = false;
      while (count == 0) {
        if (budget-- == 0) {
          atomicOr(err, kErrBudget);
          done = true;
          hit = true;  // a malformed tree: reported, the sample dropped
          break;
        }
        float4 l0, l1, r0, r1;
        load_node(&m.nodes[2 * lf], l0, l1);
        load_node(&m.nodes[2 * lf + 2], r0, r1);
        float dl, dr;
        const bool hl = box_hit(r, l0, l1, kShadowEps, far, dl);
        const bool hr = box_hit(r, r0, r1, kShadowEps, far, dr);
        const bool swap = hl && hr && dr < dl;  // the nearer child first: the likelier blocker
        const bool hn = swap ? hr : hl, hf = swap ? hl : hr;
        if (hn) {
          if (hf) {
            if (sp >= kTraceStack) {
              atomicOr(err, kErrStack);
              done = true;
              hit = true;
              break;
            }
            stk_lf[sp] = __float_as_uint(swap ? l0.w : r0.w);
            stk_cnt[sp] = __float_as_uint(swap ? l1.w : r1.w);
            ++sp;
          }
          lf = __float_as_uint(swap ? r0.w : l0.w);
          count = __float_as_uint(swap ? r1.w : l1.w);
        } else if (hf) {
          lf = __float_as_uint(swap ? l0.w : r0.w);
          count = __float_as_uint(swap ? l1.w : r1.w);
        } else if (sp > 0) {
          --sp;
          lf = stk_lf[sp];
          count = stk_cnt[sp];
        } else {
          done = true;
          break;
        }
      }
      if (!done) {
        for (uint32_t j = lf; j < lf + count && !hit; ++j) {
          const float4 A = __ldg(&m.tri_a[j]);
          const float4 B = __ldg(&m.tri_b[j]);
          const float2 C = __ldg(&m.tri_c[j]);
          float t;
          if (tri_hit(r, A, B, C.x, t) && t >= kShadowEps && t <= far) hit = true;
        }
        if (hit || sp == 0) {
          done = true;
        } else {
          --sp;
          lf = stk_lf[sp];
          count = stk_cnt[sp];
        }
      }
      if (done) {
        if (!hit) {
          w.lr[p] = fa(w.lr[p], w.s_cr[k]);
          w.lg[p] = fa(w.lg[p], w.s_cg[k]);
          w.lb[p] = fa(w.lb[p], w.s_cb[k]);
        }
        active = false;
      }
    }
  }
}

__global__ void __launch_bounds__(256) k_accumulate(WaveBuffers w, uint32_t n, double* __restrict__ film,
                                                    uint32_t image_w, uint32_t stride, uint32_t film_w) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t px = w.pixel[i];
    const uint32_t pix = stride == 1 ? px : ((px / image_w) / stride) * film_w + (px % image_w) / stride;
    atomicAdd(film + 3 * size_t(pix), double(w.lr[i]));
    atomicAdd(film + 3 * size_t(pix) + 1, double(w.lg[i]));
    atomicAdd(film + 3 * size_t(pix) + 2, double(w.lb[i]));
  }
}

// A finished path's radiance into its scene's film (FP64 sums: the FP32 radiances of a pixel
// add exactly, so the order of the adds does not matter).
PBRT_DEV void batch_film_add(const BatchScene& e, uint32_t px, float r, float g, float bl) {
  const uint32_t iw = e.cam.width;
  const uint32_t pix = e.stride == 1 ? px : ((px / iw) / e.stride) * e.film_w + (px % iw) / e.stride;
  double* film = e.film + 3 * size_t(pix);
  atomicAdd(film, double(r));
  atomicAdd(film + 1, double(g));
  atomicAdd(film + 2, double(bl));
}

__global__ void __launch_bounds__(256) k_accumulate_batch(WaveBuffers w, uint32_t n, const BatchScene* __restrict__ b) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    batch_film_add(b[w.scene[i]], w.pixel[i], w.lr[i], w.lg[i], w.lb[i]);
}

// ---- batches: every path to its end in one persistent launch -------------------------------
PBRT_DEV unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__global__ void k_batch_clock(unsigned long long* t) { *t = global_ns(); }

// The batch frame as persistent warps over all scenes' paths (table order, cheapest scene
// first): a lane takes path g (one atomicAdd on `fetch` per warp, once at least `refill_min`
// lanes are idle or all are), and each iteration runs one vertex of its path: the nearest
// hit (Scene::find_nearest, the full query), the vertex's shading (shade_vertex, the shading
// kernel's code), the shadow ray (Scene::any_hit) and, when the path ends, the film add. The
// arithmetic is the wavefront's, so films are the same. `done[s]` counts scene s's finished
// paths (one atomicAdd per warp and scene); the lane that finishes a scene's last path stamps
// `done_ns[s]` with the GPU clock. stats: rays, shadow rays, paths (one atomicAdd per warp).
// kTight: at most 64 registers (8 resident blocks per SM, more spills; the default) instead
// of the compiler's choice (96: 5 blocks per SM).
//
// Measured against the wavefront batch (one B200): the 64-scene icosphere batch (512x512,
// 4-64 spp) 4.72 s a frame against 2.36 s, 64 small scenes (128x128) 45.4 ms against 25.6 ms
// at the same mean completion time (19.6 against 20.5 ms). Each iteration runs the nearest-hit
// walk, the shading and the shadow ray for lanes at different depths of different paths, so
// the warps diverge where the wavefront's kernels each run one stage over a queue.
template <bool kCsg, bool kTight>
__global__ void __launch_bounds__(128, kTight ? 8 : 0) k_batch_paths(const BatchScene* __restrict__ b, uint32_t nscenes,
                                                     unsigned long long total, const uint32_t* __restrict__ frame,
                                                     unsigned long long* __restrict__ fetch,
                                                     unsigned long long* __restrict__ done,
                                                     unsigned long long* __restrict__ done_ns, int refill_min,
                                                     unsigned long long* stats, uint32_t* err) {
  const unsigned lane = threadIdx.x & 31u, lt = (1u << lane) - 1u;
  const uint32_t f = *frame;
  bool active = false, exhausted = false;  // exhausted is warp-uniform
  PathState P;
  uint32_t sc = 0, n_rays = 0, n_shadow = 0, n_paths = 0;
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (!exhausted && idle && (__popc(idle) >= refill_min || idle == 0xffffffffu)) {
      const int leader = __ffs(idle) - 1;
      unsigned long long base = 0;
      if (int(lane) == leader) base = atomicAdd(fetch, (unsigned long long)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, leader);
      exhausted = base + __popc(idle) >= total;
      if (!active) {
        const unsigned long long g = base + __popc(idle & lt);
        if (g < total) {
          sc = batch_scene_of(b, nscenes, g);
          const BatchScene& e = b[sc];
          uint32_t pixel, sample;
          batch_pixel_sample(e, g, f, pixel, sample);
          begin_path(e.cam, e.seed, pixel, sample, P.o, P.d, P.st);
          P.beta = mk3(1.f, 1.f, 1.f);
          P.L = mk3(0.f, 0.f, 0.f);
          P.pixel = pixel;
          P.flags = kSpecularBit;  // is_last_bounce_specular starts true (path.rs:52)
          active = true;
          ++n_paths;
        }
      }
    }
    if (__ballot_sync(0xffffffffu, active) == 0) {
      if (exhausted) break;
      continue;  // all idle and paths left: the next iteration refills
    }
    bool finished = false;
    if (active) {
      const BatchScene& e = b[sc];
      const PathSettings ps{e.max_depth, e.rr_start, e.integrator, e.cam.near, e.cam.far};
      float t = 0.f;
      uint32_t obj = 0xFFFFFFFFu, prim = 0;
      if (!scene_closest<kCsg>(e.view, P.o, P.d, ps.near, ps.far, t, obj, prim, err)) obj = 0xFFFFFFFFu;
      ++n_rays;
      VertexOut v;
      shade_vertex(e.view, ps, P, obj, prim, t, kCacheOff, 0, v);
      if (v.shadow) {  // VisibilityTester::unoccluded (lights.rs:67-69)
        ++n_shadow;
        if (!scene_any<kCsg>(e.view, v.sro, v.srd, kShadowEps, v.stmax, err)) {
          P.L.x = fa(P.L.x, v.contrib.x);
          P.L.y = fa(P.L.y, v.contrib.y);
          P.L.z = fa(P.L.z, v.contrib.z);
        }
      }
      if (!v.alive) {
        batch_film_add(e, P.pixel, P.L.x, P.L.y, P.L.z);
        active = false;
        finished = true;
      }
    }
    const unsigned fin = __ballot_sync(0xffffffffu, finished);
    if (finished) {  // per scene: one count per warp, and the clock when the scene is complete
      const unsigned same = __match_any_sync(fin, sc);
      if (int(lane) == __ffs(same) - 1) {
        const unsigned long long k = __popc(same);
        const BatchScene& e = b[sc];
        if (atomicAdd(done + sc, k) + k == (unsigned long long)e.npix * e.spp) done_ns[sc] = global_ns();
      }
    }
  }
  if (stats) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      n_rays += __shfl_xor_sync(0xffffffffu, n_rays, off);
      n_shadow += __shfl_xor_sync(0xffffffffu, n_shadow, off);
      n_paths += __shfl_xor_sync(0xffffffffu, n_paths, off);
    }
    if (lane == 0) {
      atomicAdd(stats, (unsigned long long)n_rays);
      atomicAdd(stats + 1, (unsigned long long)n_shadow);
      atomicAdd(stats + 2, (unsigned long long)n_paths);
    }
  }
}

// Every scene's film: zero (scale 0) or divide the sums by spp; blockIdx.y is the scene.
__global__ void k_films_batch(const BatchScene* __restrict__ b, int zero) {
  const BatchScene& e = b[blockIdx.y];
  const size_t n = size_t(e.npix) * 3;
  const double s = zero ? 0.0 : 1.0 / double(e.spp);
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    e.film[i] = zero ? 0.0 : e.film[i] * s;
}

__global__ void k_scale_film(double* film, size_t n, double s) {
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    film[i] *= s;
}

// ---- general-scene ray casting ---------------------------------------------------------------
// Adds a thread's counters to cnt[0..2] (one atomic per warp and counter).
PBRT_DEV void flush_counts(const SceneCount& c, unsigned long long* cnt) {
  unsigned long long v[3] = {c.nodes, c.boxes, c.objects};
  for (int k = 0; k < 3; ++k) {
    for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_down_sync(0xFFFFFFFFu, v[k], off);
    if ((threadIdx.x & 31) == 0 && v[k]) atomicAdd(cnt + k, v[k]);
  }
}

// Nearest hit per ray; object ids are the description's (the leaf's desc_id). kCount adds
// the scene accelerator's counters (Scene::intersect_instrumented) into cnt.
template <bool kCount, bool kCsg>
__global__ void __launch_bounds__(128) k_scene_closest(SceneView s, const float* __restrict__ rays, uint64_t stride,
                                                       uint64_t n, uint32_t* __restrict__ prim, float* __restrict__ tout,
                                                       uint32_t* __restrict__ obj, unsigned long long* cnt,
                                                       uint32_t* err) {
  SceneCount c{0, 0, 0};
  // whole warps run the same trip count so the counter reduction sees full warps
  const uint64_t step = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t iters = (n + step - 1) / step;
  for (uint64_t it = 0; it < iters; ++it) {
    const uint64_t i = it * step + uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) continue;
    const F3 o = mk3(__ldcs(rays + i), __ldcs(rays + stride + i), __ldcs(rays + 2 * stride + i));
    const F3 d = mk3(__ldcs(rays + 3 * stride + i), __ldcs(rays + 4 * stride + i), __ldcs(rays + 5 * stride + i));
    const float near = __ldcs(rays + 6 * stride + i), far = __ldcs(rays + 7 * stride + i);
    float t = 0.f;
    uint32_t leaf = 0, pr = 0;
    const bool hit = scene_closest_t<kCount, kCsg>(s, o, d, near, far, t, leaf, pr, err, &c);
    __stcs(prim + i, hit ? pr : 0xFFFFFFFFu);
    __stcs(tout + i, hit ? t : __int_as_float(0x7f800000));
    if (obj) __stcs(obj + i, hit ? s.objects[leaf].desc_id : 0xFFFFFFFFu);
  }
  if (kCount) flush_counts(c, cnt);
}

template <bool kCount, bool kCsg>
__global__ void __launch_bounds__(128) k_scene_any(SceneView s, const float* __restrict__ rays, uint64_t stride,
                                                   uint64_t n, uint8_t* __restrict__ occ, unsigned long long* cnt,
                                                   uint32_t* err) {
  SceneCount c{0, 0, 0};
  const uint64_t step = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t iters = (n + step - 1) / step;
  for (uint64_t it = 0; it < iters; ++it) {
    const uint64_t i = it * step + uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) continue;
    const F3 o = mk3(__ldcs(rays + i), __ldcs(rays + stride + i), __ldcs(rays + 2 * stride + i));
    const F3 d = mk3(__ldcs(rays + 3 * stride + i), __ldcs(rays + 4 * stride + i), __ldcs(rays + 5 * stride + i));
    occ[i] = scene_any_t<kCount, kCsg>(s, o, d, __ldcs(rays + 6 * stride + i), __ldcs(rays + 7 * stride + i), err, &c)
                 ? 1
                 : 0;
  }
  if (kCount) flush_counts(c, cnt);
}

// ---- launchers -------------------------------------------------------------------------------
static unsigned grid_cap(uint64_t n, int threads, int sm_count, int per_sm) {
  const uint64_t want = (n + threads - 1) / threads;
  const uint64_t cap = uint64_t(sm_count) * per_sm;
  return unsigned(want < cap ? (want ? want : 1) : cap);
}

cudaError_t launch_scene_closest(const SceneView& s, const float* rays, uint64_t stride, uint64_t n, uint32_t* prim,
                                 float* t, uint32_t* obj, unsigned long long* cnt, uint32_t* err, int sm_count,
                                 cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const unsigned g = grid_cap(n, 128, sm_count, 32);
  if (cnt) k_scene_closest<true, true><<<g, 128, 0, st>>>(s, rays, stride, n, prim, t, obj, cnt, err);
  else if (s.has_csg) k_scene_closest<false, true><<<g, 128, 0, st>>>(s, rays, stride, n, prim, t, obj, nullptr, err);
  else k_scene_closest<false, false><<<g, 128, 0, st>>>(s, rays, stride, n, prim, t, obj, nullptr, err);
  return cudaGetLastError();
}

cudaError_t launch_scene_any(const SceneView& s, const float* rays, uint64_t stride, uint64_t n, uint8_t* occ,
                             unsigned long long* cnt, uint32_t* err, int sm_count, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const unsigned g = grid_cap(n, 128, sm_count, 32);
  if (cnt) k_scene_any<true, true><<<g, 128, 0, st>>>(s, rays, stride, n, occ, cnt, err);
  else if (s.has_csg) k_scene_any<false, true><<<g, 128, 0, st>>>(s, rays, stride, n, occ, nullptr, err);
  else k_scene_any<false, false><<<g, 128, 0, st>>>(s, rays, stride, n, occ, nullptr, err);
  return cudaGetLastError();
}

// The persistent walk (k_extend_walk) for scenes whose top-level tree has at least this many
// nodes; one thread per path (k_extend) below it.
constexpr uint32_t kWalkMinTopNodes = 64;

// The walk's step schedule: a leaf step once `leaf_min` lanes of a warp stand on a leaf, a
// refill once `refill_min` lanes are idle. PBRT_WALK_SCHEDULE="leaf_min,refill_min" (each in
// 1..32) overrides the default for measurements; films do not depend on it.
struct WalkSchedule {
  int leaf_min = 8, refill_min = 8;
};

static WalkSchedule walk_schedule() {
  static const WalkSchedule v = [] {
    WalkSchedule d;
    if (const char* e = std::getenv("PBRT_WALK_SCHEDULE")) {
      int a = 0, b = 0;
      if (std::sscanf(e, "%d,%d", &a, &b) == 2 && a >= 1 && a <= 32 && b >= 1 && b <= 32) {
        d.leaf_min = a;
        d.refill_min = b;
      }
    }
    return d;
  }();
  return v;
}

// Queue pushes of the shading kernel per block through shared memory (k_shade<.., true>)
// instead of per warp: PBRT_SHADE_STAGING=1 / 0 selects it for measurements; films do not
// depend on it beyond the order of queue entries.
static bool shade_staging() {
  static const bool v = [] {
    const char* e = std::getenv("PBRT_SHADE_STAGING");
    return e && e[0] == '1';
  }();
  return v;
}

// extend -> shade -> shadow, `loops` times, over the ping-pong queues. `top_nodes`: the largest
// top-level tree among the scenes rendered; `csg`: some scene holds a constructive solid (the
// traversal kernels are also built without the solids' code, which takes registers and spills
// from every other query).
// Scenes' deferred leaves are answered by their own passes (k_defer_closest, k_defer_any)
// unless PBRT_DEFER=0 (for measurements; the films differ at most where two objects are hit
// at exactly the same distance).
static bool defer_enabled() {
  static const bool v = [] {
    const char* e = std::getenv("PBRT_DEFER");
    return !(e && e[0] == '0');
  }();
  return v;
}

template <class Src>
static cudaError_t bounce_loop(const WaveBuffers& w, const Src& src, const CacheWave& cw, uint32_t loops, bool shadows,
                               uint32_t cache_mode, uint32_t term_hit, const LaunchShape& sh, unsigned long long* stats,
                               uint32_t* err, int sm_count, cudaStream_t st, uint32_t top_nodes, bool csg,
                               bool defer) {
  cudaError_t e;
  const unsigned gt = unsigned(sm_count) * sh.trace_blocks_per_sm, gs = unsigned(sm_count) * sh.shade_blocks_per_sm;
  // the deferred passes: persistent, PBRT_DEFER_MIN_BLOCKS blocks of 128 per SM
  const unsigned gd = unsigned(sm_count) * unsigned(PBRT_DEFER_MIN_BLOCKS);
  const uint32_t df = defer ? 1u : 0u;
  for (uint32_t b = 0; b < loops; ++b) {
    uint32_t* qin = (b & 1) ? w.qb : w.qa;
    uint32_t* qout = (b & 1) ? w.qa : w.qb;
    uint32_t* cin = w.counts + (b & 1);
    uint32_t* cout = w.counts + ((b + 1) & 1);
    if ((e = cudaMemsetAsync(cout, 0, sizeof(uint32_t), st)) != cudaSuccess) return e;
    // counts[2]: shadow rays queued by k_shade; counts[3]: k_extend_walk's fetch position;
    // counts[4], [5]: the deferred passes' fetch positions
    if ((e = cudaMemsetAsync(w.counts + 2, 0, 4 * sizeof(uint32_t), st)) != cudaSuccess) return e;
    const WalkSchedule ws = walk_schedule();
    if (top_nodes >= kWalkMinTopNodes && csg)
      k_extend_walk<Src, true><<<gt, sh.trace_threads, 0, st>>>(w, src, qin, cin, w.counts + 3, err, stats,
                                                                ws.leaf_min, ws.refill_min, df);
    else if (top_nodes >= kWalkMinTopNodes)
      k_extend_walk<Src, false><<<gt, sh.trace_threads, 0, st>>>(w, src, qin, cin, w.counts + 3, err, stats,
                                                                 ws.leaf_min, ws.refill_min, df);
    else if (csg)
      k_extend<Src, true><<<gt, sh.trace_threads, 0, st>>>(w, src, qin, cin, err, stats, df);
    else
      k_extend<Src, false><<<gt, sh.trace_threads, 0, st>>>(w, src, qin, cin, err, stats, df);
    if (defer) k_defer_closest<Src><<<gd, 128, 0, st>>>(w, src, qin, cin, w.counts + 4, err);
    if (shade_staging())
      k_shade<Src, true><<<gs, sh.shade_threads, 0, st>>>(w, src, qin, cin, qout, cout, cw, cache_mode, term_hit);
    else
      k_shade<Src, false><<<gs, sh.shade_threads, 0, st>>>(w, src, qin, cin, qout, cout, cw, cache_mode, term_hit);
    // (a persistent walk for the shadow rays measured 2.6% slower on 10,000 spheres: any-hit
    // rays end early, so one thread per ray wastes little)
    if (shadows && csg) k_shadow<Src, true><<<gt, sh.trace_threads, 0, st>>>(w, src, err, stats, df);
    else if (shadows) k_shadow<Src, false><<<gt, sh.trace_threads, 0, st>>>(w, src, err, stats, df);
    if (shadows && defer) k_defer_any<Src><<<gd, 128, 0, st>>>(w, src, w.counts + 5, err);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Paths from which a batch scene gets waves of its own (it fills a B200 alone: 148 SMs keep
// about 0.3M threads resident).
constexpr unsigned long long kBatchOwnWavePaths = 1ull << 20;

// The waves of a batch frame, (first path, paths), in path order and covering every path,
// none longer than `wave`: a scene of at least kBatchOwnWavePaths paths, or of more than
// `wave`, gets waves of its own (the single-scene kernels, its own depth, its completion as
// soon as it is done); smaller scenes are packed whole into shared waves.
static std::vector<std::pair<unsigned long long, uint32_t>> batch_waves(const BatchScene* host_table,
                                                                        uint32_t nscenes, uint32_t wave) {
  std::vector<std::pair<unsigned long long, uint32_t>> waves;
  unsigned long long pack_begin = 0, pack_n = 0;
  auto flush = [&]() {
    if (pack_n) waves.emplace_back(pack_begin, uint32_t(pack_n));
    pack_n = 0;
  };
  for (uint32_t i = 0; i < nscenes; ++i) {
    const unsigned long long b = host_table[i].begin, np = (unsigned long long)host_table[i].npix * host_table[i].spp;
    if (np >= kBatchOwnWavePaths || np > wave) {
      flush();
      for (unsigned long long o = 0; o < np; o += wave) waves.emplace_back(b + o, uint32_t(np - o < wave ? np - o : wave));
    } else {
      if (pack_n + np > wave) flush();
      if (!pack_n) pack_begin = b;
      pack_n += np;
    }
  }
  flush();
  return waves;
}

std::vector<BatchWave> batch_plan(const BatchScene* host_table, uint32_t nscenes, uint32_t wave, uint32_t branches) {
  const std::vector<std::pair<unsigned long long, uint32_t>> waves = batch_waves(host_table, nscenes, wave);
  std::vector<BatchWave> plan;
  plan.reserve(waves.size());
  std::vector<unsigned long long> load(branches ? branches : 1, 0);
  uint32_t first = 0, prev_last = ~0u, branch = 0;
  for (const auto& wv : waves) {
    while (host_table[first].begin + (unsigned long long)host_table[first].npix * host_table[first].spp <= wv.first)
      ++first;
    uint32_t last = first, depth = host_table[first].max_depth;
    while (last + 1 < nscenes && host_table[last + 1].begin < wv.first + wv.second) {
      ++last;
      depth = depth > host_table[last].max_depth ? depth : host_table[last].max_depth;
    }
    if (first != prev_last) {  // a new group of waves: the least loaded branch (lowest on ties)
      branch = 0;
      for (uint32_t k = 1; k < load.size(); ++k)
        if (load[k] < load[branch]) branch = k;
    }
    load[branch] += (unsigned long long)wv.second * depth;
    plan.push_back(BatchWave{wv.first, wv.second, branch});
    prev_last = last;
  }
  return plan;
}

cudaError_t render_batch(const BatchScene* table, const BatchScene* host_table, uint32_t nscenes,
                         const std::vector<BatchWave>& plan, const WaveBuffers* bw, const cudaStream_t* bst,
                         uint32_t nbranch, const uint32_t* frame, uint32_t max_depth, bool any_path_integrator,
                         const LaunchShape& shape, unsigned long long* stats, uint32_t* err, int sm_count,
                         cudaStream_t st, cudaEvent_t fork, const cudaEvent_t* joins, cudaEvent_t* done) {
  cudaError_t e;
  uint32_t max_npix = 0;
  for (uint32_t i = 0; i < nscenes; ++i) max_npix = max_npix > host_table[i].npix ? max_npix : host_table[i].npix;
  const dim3 fgrid(unsigned((size_t(max_npix) * 3 + 255) / 256 < 1024 ? (size_t(max_npix) * 3 + 255) / 256 : 1024),
                   nscenes);
  k_films_batch<<<fgrid, 256, 0, st>>>(table, 1);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (nbranch > 1) {
    if ((e = cudaEventRecord(fork, st)) != cudaSuccess) return e;
    for (uint32_t k = 1; k < nbranch; ++k)
      if ((e = cudaStreamWaitEvent(bst[k], fork, 0)) != cudaSuccess) return e;
  }
  const ManyScenes src{table};
  uint32_t top_nodes = 0;
  bool csg = false;
  for (uint32_t i = 0; i < nscenes; ++i) {
    top_nodes = top_nodes > host_table[i].view.top_node_count ? top_nodes : host_table[i].view.top_node_count;
    csg = csg || host_table[i].view.has_csg;
  }
  uint32_t first = 0;
  for (const BatchWave& wv : plan) {
    const unsigned long long base = wv.base;
    const uint32_t n = wv.n;
    const WaveBuffers& w = bw[wv.branch];
    cudaStream_t s = bst[wv.branch];
    // the scenes holding the wave's first and last paths (the table is in path order)
    while (host_table[first].begin + (unsigned long long)host_table[first].npix * host_table[first].spp <= base) ++first;
    uint32_t last = first;
    while (last + 1 < nscenes && host_table[last + 1].begin < base + n) ++last;
    k_generate_batch<<<grid_cap(n, 256, sm_count, 16), 256, 0, s>>>(w, table, nscenes, base, n, frame, stats);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (first == last) {
      // a wave of one scene runs the single-scene kernels: its view is a kernel parameter
      // instead of a per-path table lookup, and the bounce loop stops at its own depth
      const BatchScene& h = host_table[first];
      const OneScene one{h.view, PathSettings{h.max_depth, h.rr_start, h.integrator, h.cam.near, h.cam.far}};
      e = bounce_loop(w, one, CacheWave{}, h.max_depth, !h.integrator, kCacheOff, 0, shape, stats, err, sm_count, s,
                      h.view.top_node_count, h.view.has_csg != 0, defer_enabled() && h.view.defer_leaf != kNoLeaf);
    } else {
      bool defer = false;
      for (uint32_t i = first; i <= last; ++i) defer = defer || host_table[i].view.defer_leaf != kNoLeaf;
      e = bounce_loop(w, src, CacheWave{}, max_depth, any_path_integrator, kCacheOff, 0, shape, stats, err, sm_count,
                      s, top_nodes, csg, defer_enabled() && defer);
    }
    if (e != cudaSuccess) return e;
    k_accumulate_batch<<<grid_cap(n, 256, sm_count, 16), 256, 0, s>>>(w, n, table);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // the wave's scenes whose last path was in it are done
    for (uint32_t i = first; done && i <= last; ++i)
      if (host_table[i].begin + (unsigned long long)host_table[i].npix * host_table[i].spp <= base + n)
        if ((e = cudaEventRecordWithFlags(done[i], s, cudaEventRecordExternal)) != cudaSuccess) return e;
  }
  if (nbranch > 1) {
    for (uint32_t k = 1; k < nbranch; ++k) {
      if ((e = cudaEventRecord(joins[k], bst[k])) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(st, joins[k], 0)) != cudaSuccess) return e;
    }
  }
  k_films_batch<<<fgrid, 256, 0, st>>>(table, 0);
  return cudaGetLastError();
}

// Resident 128-thread blocks per SM of the persistent batch kernel (computed once).
template <bool kCsg, bool kTight>
static int batch_paths_blocks_per_sm() {
  static const int v = [] {
    int b = 0;
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_batch_paths<kCsg, kTight>, 128, 0);
    return e == cudaSuccess && b > 0 ? b : 4;
  }();
  return v;
}

// PBRT_BATCH_REFILL (1..32, default 8): idle lanes of a warp before the persistent batch
// kernel refills them (2 and 16 measured the same); PBRT_BATCH_TIGHT=0: the 96-register build
// (10-13 % slower than the 64-register default). For measurements.
static int batch_refill_min() {
  static const int v = [] {
    const char* e = std::getenv("PBRT_BATCH_REFILL");
    const int r = e ? std::atoi(e) : 8;
    return r >= 1 && r <= 32 ? r : 8;
  }();
  return v;
}

static bool batch_tight() {
  static const bool v = [] {
    const char* e = std::getenv("PBRT_BATCH_TIGHT");
    return !(e && e[0] == '0');
  }();
  return v;
}

template <bool kCsg, bool kTight>
static void launch_batch_paths(const BatchScene* table, uint32_t nscenes, unsigned long long total,
                               const uint32_t* frame, unsigned long long* scratch, int refill,
                               unsigned long long* stats, uint32_t* err, int sm_count, cudaStream_t st) {
  k_batch_paths<kCsg, kTight><<<unsigned(sm_count * batch_paths_blocks_per_sm<kCsg, kTight>()), 128, 0, st>>>(
      table, nscenes, total, frame, scratch, scratch + 2, scratch + 2 + nscenes, refill, stats, err);
}

cudaError_t render_batch_persistent(const BatchScene* table, const BatchScene* host_table, uint32_t nscenes,
                                    const uint32_t* frame, unsigned long long* scratch, unsigned long long* stats,
                                    uint32_t* err, int sm_count, cudaStream_t st) {
  cudaError_t e;
  uint32_t max_npix = 0;
  bool csg = false;
  for (uint32_t i = 0; i < nscenes; ++i) {
    max_npix = max_npix > host_table[i].npix ? max_npix : host_table[i].npix;
    csg = csg || host_table[i].view.has_csg;
  }
  const dim3 fgrid(unsigned((size_t(max_npix) * 3 + 255) / 256 < 1024 ? (size_t(max_npix) * 3 + 255) / 256 : 1024),
                   nscenes);
  const unsigned long long total =
      host_table[nscenes - 1].begin + (unsigned long long)host_table[nscenes - 1].npix * host_table[nscenes - 1].spp;
  // scratch: [0] fetch position, [1] frame start (GPU clock), [2, 2 + n) finished paths per
  // scene, [2 + n, 2 + 2n) each scene's completion time
  if ((e = cudaMemsetAsync(scratch, 0, (2 + 2 * size_t(nscenes)) * sizeof(unsigned long long), st)) != cudaSuccess)
    return e;
  k_films_batch<<<fgrid, 256, 0, st>>>(table, 1);
  k_batch_clock<<<1, 1, 0, st>>>(scratch + 1);
  const int refill = batch_refill_min();
  const bool tight = batch_tight();
  if (csg && tight)
    launch_batch_paths<true, true>(table, nscenes, total, frame, scratch, refill, stats, err, sm_count, st);
  else if (csg)
    launch_batch_paths<true, false>(table, nscenes, total, frame, scratch, refill, stats, err, sm_count, st);
  else if (tight)
    launch_batch_paths<false, true>(table, nscenes, total, frame, scratch, refill, stats, err, sm_count, st);
  else
    launch_batch_paths<false, false>(table, nscenes, total, frame, scratch, refill, stats, err, sm_count, st);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_films_batch<<<fgrid, 256, 0, st>>>(table, 0);
  return cudaGetLastError();
}

cudaError_t trace_wave(const SceneView& s, const WaveBuffers& w, const CacheWave& cw, const CameraRec& cam,
                       uint64_t wave_base, uint32_t n, uint32_t npix, const RenderSettings& rs, uint32_t* err,
                       int sm_count, cudaStream_t st) {
  cudaError_t e;
  k_generate<<<grid_cap(n, 256, sm_count, 16), 256, 0, st>>>(w, cam, wave_base, n, npix, rs.sample_offset, rs.seed,
                                                             rs.random_pixels, rs.stride,
                                                             rs.film_w ? rs.film_w : cam.width, rs.stats);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const OneScene src{s, PathSettings{rs.max_depth, rs.rr_start, rs.integrator, cam.near, cam.far}};
  return bounce_loop(w, src, cw, rs.loop_depth ? rs.loop_depth : rs.max_depth, !rs.integrator, rs.cache_mode, rs.term_hit,
                     rs.shape, rs.stats, err, sm_count, st, s.top_node_count, s.has_csg != 0,
                     defer_enabled() && s.defer_leaf != kNoLeaf);
}

cudaError_t accumulate_wave(const WaveBuffers& w, uint32_t n, double* film, uint32_t image_w, const RenderSettings& rs,
                            int sm_count, cudaStream_t st) {
  k_accumulate<<<grid_cap(n, 256, sm_count, 16), 256, 0, st>>>(w, n, film, image_w, rs.stride,
                                                               rs.film_w ? rs.film_w : image_w);
  return cudaGetLastError();
}

cudaError_t render_wave(const SceneView& s, const WaveBuffers& w, const CameraRec& cam, uint64_t wave_base,
                        uint32_t n, uint32_t npix, const RenderSettings& rs, double* film, uint32_t* err, int sm_count,
                        cudaStream_t st) {
  RenderSettings plain = rs;
  plain.cache_mode = kCacheOff;
  const cudaError_t e = trace_wave(s, w, CacheWave{}, cam, wave_base, n, npix, plain, err, sm_count, st);
  if (e != cudaSuccess) return e;
  return accumulate_wave(w, n, film, cam.width, rs, sm_count, st);
}

cudaError_t apply_cache(const WaveBuffers& w, const CacheWave& cw, uint32_t n, float max_l, int sm_count,
                        cudaStream_t st) {
  k_apply_cache<<<grid_cap(n, 256, sm_count, 8), 256, 0, st>>>(w, cw, n, max_l);
  return cudaGetLastError();
}

cudaError_t train_batch(const WaveBuffers& w, const CacheWave& cw, uint32_t batch, uint32_t step,
                        unsigned long long seed, float max_l, float* rec, float* tgt, int sm_count, cudaStream_t st) {
  if (batch == 0) return cudaSuccess;
  k_train_batch<<<grid_cap(batch, 256, sm_count, 8), 256, 0, st>>>(w, cw, batch, step, seed, max_l, rec, tgt);
  return cudaGetLastError();
}

cudaError_t scale_film(double* film, size_t n, double s, int sm_count, cudaStream_t st) {
  k_scale_film<<<grid_cap(n, 256, sm_count, 8), 256, 0, st>>>(film, n, s);
  return cudaGetLastError();
}

}  // namespace pbrt
