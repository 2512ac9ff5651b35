// oracle_capi.cpp — TEST INFRASTRUCTURE, NOT THE PRODUCT.
//
// extern "C" surface of the CPU oracle (pbrt_oracle.hpp) for the Python tests and the
// cpu_baseline leg of bench.py. Rays cross this boundary as eight SoA planes of n values:
// ox, oy, oz, dx, dy, dz, tmin, tmax.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "mlp_oracle.hpp"
#include "pbrt_oracle.hpp"
#include "pbrt_oracle_pt.hpp"


using namespace oracle;

namespace {

template <class F>
void parallel_for(size_t n, int threads, F&& f) {
  if (threads <= 1 || n < 4096) {
    f(size_t(0), n);
    return;
  }
  std::vector<std::thread> pool;
  std::atomic<size_t> next{0};
  const size_t chunk = 4096;
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&]() {
      for (;;) {
        size_t b = next.fetch_add(chunk);
        if (b >= n) break;
        f(b, std::min(n, b + chunk));
      }
    });
  }
  for (auto& th : pool) th.join();
}

template <class R>
Ray<R> load_ray(const R* rays, size_t n, size_t i, R* tmin, R* tmax) {
  Ray<R> r;
  r.o = {rays[i], rays[n + i], rays[2 * n + i]};
  r.d = {rays[3 * n + i], rays[4 * n + i], rays[5 * n + i]};
  *tmin = rays[6 * n + i];
  *tmax = rays[7 * n + i];
  return r;
}

template <class R>
int trace(const MeshBVH<R>* m, const R* rays, size_t n, uint32_t* prim, R* t, uint64_t* stats, int threads) {
  std::atomic<uint64_t> nv{0}, bt{0}, tt{0};
  parallel_for(n, threads, [&](size_t b, size_t e) {
    TraversalStats st;
    for (size_t i = b; i < e; ++i) {
      R tmin, tmax;
      Ray<R> r = load_ray(rays, n, i, &tmin, &tmax);
      TriHit<R> h;
      uint32_t id;
      if (m->traverse(r, tmin, tmax, &h, &id, &st)) {
        prim[i] = id;
        t[i] = h.t;
      } else {
        prim[i] = 0xFFFFFFFFu;
        t[i] = std::numeric_limits<R>::infinity();
      }
    }
    nv += st.nodes_visited;
    bt += st.box_tests;
    tt += st.triangle_tests;
  });
  if (stats) {
    stats[0] = nv;
    stats[1] = bt;
    stats[2] = tt;
  }
  return 0;
}

template <class R>
int occluded(const MeshBVH<R>* m, const R* rays, size_t n, uint8_t* occ, int threads) {
  parallel_for(n, threads, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      R tmin, tmax;
      Ray<R> r = load_ray(rays, n, i, &tmin, &tmax);
      occ[i] = m->intersect_p(r, tmin, tmax) ? 1 : 0;
    }
  });
  return 0;
}

template <class R>
int brute(const MeshBVH<R>* m, const R* rays, size_t n, uint32_t* prim, R* t, int threads) {
  parallel_for(n, threads, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      R tmin, tmax;
      Ray<R> r = load_ray(rays, n, i, &tmin, &tmax);
      R tt;
      uint32_t id;
      if (m->brute_force(r, tmin, tmax, &tt, &id)) {
        prim[i] = id;
        t[i] = tt;
      } else {
        prim[i] = 0xFFFFFFFFu;
        t[i] = std::numeric_limits<R>::infinity();
      }
    }
  });
  return 0;
}

// Mesh-mode ray set of the traversal benchmark (bvh_stats.rs:345-382): 6 orbit cameras
// around the vertex bounds, 200x200 pixel-centre primary rays each, near 1e-4, far 1000.
template <class R>
void orbit_rays(const MeshBVH<R>* m, R* out) {
  const size_t n = 6 * 200 * 200;
  AABB<R> b = m->vertex_bounds();
  V3<R> c = b.centroid();
  const R PI = R(3.141592653589793238462643383279502884L);
  const R fov = R(40) * PI / R(180);
  R radius = length(b.bmax - b.bmin) * R(0.5);
  R dist = radius / std::sin(fov / R(2));
  size_t i = 0;
  for (int v = 0; v < 6; ++v) {
    PinHoleCamera<R> cam = orbit_camera<R>(v, c, dist);
    for (uint32_t py = 0; py < 200; ++py)
      for (uint32_t px = 0; px < 200; ++px, ++i) {
        Ray<R> r = cam.get_ray(R(px) + R(0.5), R(py) + R(0.5));
        out[i] = r.o.x; out[n + i] = r.o.y; out[2 * n + i] = r.o.z;
        out[3 * n + i] = r.d.x; out[4 * n + i] = r.d.y; out[5 * n + i] = r.d.z;
        out[6 * n + i] = R(0.0001); out[7 * n + i] = R(1000);
      }
  }
}

thread_local std::string g_err;

}  // namespace

extern "C" {

const char* oracle_last_error() { return g_err.c_str(); }
void oracle_free(void* p) { std::free(p); }

// ASCII PLY reader with the reference's semantics (src/loader/ply/ply_loader.rs,
// src/loader/mesh_loader.rs:13-91): float properties parse as f32 and widen to f64,
// vertex_indices lists are appended as they come (reversed when `reverse`).
int oracle_ply_read(const char* path, int reverse, double** verts_out, size_t* nv_out, uint32_t** idx_out, size_t* nidx_out) {
  std::ifstream f(path);
  if (!f) { g_err = std::string("cannot open ") + path; return -1; }
  std::string line;
  struct Prop { std::string name; std::string type; bool list; std::string count_type; };
  struct Elem { std::string name; size_t count; std::vector<Prop> props; };
  std::vector<Elem> elems;
  std::getline(f, line);
  if (line.rfind("ply", 0) != 0) { g_err = "not a ply file"; return -1; }
  while (std::getline(f, line)) {
    std::istringstream ss(line);
    std::string kw;
    ss >> kw;
    if (kw == "format") {
      std::string fmt;
      ss >> fmt;
      if (fmt != "ascii") { g_err = "only ascii ply is supported"; return -1; }
    } else if (kw == "element") {
      Elem e;
      ss >> e.name >> e.count;
      elems.push_back(e);
    } else if (kw == "property") {
      Prop p;
      std::string t;
      ss >> t;
      if (t == "list") { p.list = true; ss >> p.count_type >> p.type >> p.name; }
      else { p.list = false; p.type = t; ss >> p.name; }
      if (elems.empty()) { g_err = "property before element"; return -1; }
      elems.back().props.push_back(p);
    } else if (kw == "end_header") {
      break;
    }
  }
  std::vector<double> verts;
  std::vector<uint32_t> idx;
  for (const Elem& e : elems) {
    for (size_t r = 0; r < e.count; ++r) {
      if (!std::getline(f, line)) { g_err = "truncated ply: element " + e.name + " row " + std::to_string(r) + " of " + std::to_string(e.count); return -1; }
      std::istringstream ss(line);
      for (const Prop& p : e.props) {
        if (p.list) {
          size_t cnt;
          ss >> cnt;
          std::vector<long long> vals(cnt);
          for (size_t k = 0; k < cnt; ++k) ss >> vals[k];
          if (e.name == "face" && (p.name == "vertex_indices" || p.name == "vertex_index")) {
            if (reverse) for (size_t k = cnt; k-- > 0;) idx.push_back(uint32_t(vals[k]));
            else for (size_t k = 0; k < cnt; ++k) idx.push_back(uint32_t(vals[k]));
          }
        } else {
          std::string tok;
          ss >> tok;
          if (e.name == "vertex" && (p.name == "x" || p.name == "y" || p.name == "z")) {
            double v;
            if (p.type == "float" || p.type == "float32") v = double(std::strtof(tok.c_str(), nullptr));
            else v = std::strtod(tok.c_str(), nullptr);
            verts.push_back(v);
          }
        }
      }
    }
  }
  *nv_out = verts.size() / 3;
  *nidx_out = idx.size();
  *verts_out = (double*)std::malloc(sizeof(double) * std::max<size_t>(1, verts.size()));
  *idx_out = (uint32_t*)std::malloc(sizeof(uint32_t) * std::max<size_t>(1, idx.size()));
  std::memcpy(*verts_out, verts.data(), sizeof(double) * verts.size());
  std::memcpy(*idx_out, idx.data(), sizeof(uint32_t) * idx.size());
  return 0;
}

#define ORACLE_MESH_API(SUF, R)                                                                              \
  void* oracle_mesh_new_##SUF(const R* v, size_t nv, const uint32_t* idx, size_t nt, int bins, uint32_t max_leaf) { \
    try {                                                                                                    \
      return new MeshBVH<R>(v, nv, idx, nt, bins, max_leaf);                                                 \
    } catch (const std::exception& e) {                                                                      \
      g_err = e.what();                                                                                      \
      return nullptr;                                                                                        \
    }                                                                                                        \
  }                                                                                                          \
  void oracle_mesh_free_##SUF(void* m) { delete (MeshBVH<R>*)m; }                                            \
  void oracle_mesh_build_stats_##SUF(void* m, uint64_t* out) {                                               \
    BuildStats s = ((MeshBVH<R>*)m)->build_stats();                                                          \
    out[0] = s.node_count; out[1] = s.leaf_count; out[2] = s.max_depth;                                      \
    out[3] = s.max_leaf_tri_count; out[4] = s.total_leaf_tri_count;                                          \
  }                                                                                                          \
  size_t oracle_mesh_node_count_##SUF(void* m) { return ((MeshBVH<R>*)m)->nodes().size(); }                  \
  void oracle_mesh_nodes_##SUF(void* m, R* boxes, uint64_t* left_first, uint64_t* count) {                   \
    const auto& ns = ((MeshBVH<R>*)m)->nodes();                                                              \
    for (size_t i = 0; i < ns.size(); ++i) {                                                                 \
      boxes[6 * i + 0] = ns[i].box.bmin.x; boxes[6 * i + 1] = ns[i].box.bmin.y; boxes[6 * i + 2] = ns[i].box.bmin.z; \
      boxes[6 * i + 3] = ns[i].box.bmax.x; boxes[6 * i + 4] = ns[i].box.bmax.y; boxes[6 * i + 5] = ns[i].box.bmax.z; \
      left_first[i] = ns[i].left_first; count[i] = ns[i].count;                                              \
    }                                                                                                        \
  }                                                                                                          \
  void oracle_mesh_tri_idx_##SUF(void* m, uint32_t* out) {                                                   \
    const auto& t = ((MeshBVH<R>*)m)->tri_idx();                                                             \
    std::memcpy(out, t.data(), t.size() * sizeof(uint32_t));                                                 \
  }                                                                                                          \
  int oracle_mesh_trace_##SUF(void* m, const R* rays, size_t n, uint32_t* prim, R* t, uint64_t* stats, int threads) { \
    try {                                                                                                    \
      return trace((MeshBVH<R>*)m, rays, n, prim, t, stats, threads);                                        \
    } catch (const std::exception& e) {                                                                      \
      g_err = e.what();                                                                                      \
      return -1;                                                                                             \
    }                                                                                                        \
  }                                                                                                          \
  int oracle_mesh_occluded_##SUF(void* m, const R* rays, size_t n, uint8_t* occ, int threads) {              \
    try {                                                                                                    \
      return occluded((MeshBVH<R>*)m, rays, n, occ, threads);                                                \
    } catch (const std::exception& e) {                                                                      \
      g_err = e.what();                                                                                      \
      return -1;                                                                                             \
    }                                                                                                        \
  }                                                                                                          \
  int oracle_mesh_brute_##SUF(void* m, const R* rays, size_t n, uint32_t* prim, R* t, int threads) {         \
    return brute((MeshBVH<R>*)m, rays, n, prim, t, threads);                                                 \
  }                                                                                                          \
  void oracle_mesh_orbit_rays_##SUF(void* m, R* out) { orbit_rays((MeshBVH<R>*)m, out); }                    \
  R oracle_slab_widening_##SUF() { return Limits<R>::slab_widening(); }                                      \
  int oracle_box_hit_##SUF(const R* box, const R* ray, R tmin, R tmax, R* entry) {                           \
    AABB<R> b{{box[0], box[1], box[2]}, {box[3], box[4], box[5]}};                                           \
    Ray<R> r{{ray[0], ray[1], ray[2]}, {ray[3], ray[4], ray[5]}};                                            \
    return box_hit(b, r, tmin, tmax, entry) ? 1 : 0;                                                         \
  }                                                                                                          \
  void oracle_make_ray_##SUF(const R* o, const R* d, R* out) {                                               \
    Ray<R> r = make_ray(V3<R>{o[0], o[1], o[2]}, V3<R>{d[0], d[1], d[2]});                                   \
    out[0] = r.o.x; out[1] = r.o.y; out[2] = r.o.z; out[3] = r.d.x; out[4] = r.d.y; out[5] = r.d.z;           \
  }

ORACLE_MESH_API(f64, double)
ORACLE_MESH_API(f32, float)

}  // extern "C"

namespace {

// Sums per-chunk SceneStats into stats[3] = {nodes visited, box tests, object tests}.
struct StatSum {
  std::atomic<uint64_t> v[3] = {{0}, {0}, {0}};
  void add(const SceneStats& st) {
    v[0] += st.nodes_visited;
    v[1] += st.box_tests;
    v[2] += st.object_tests;
  }
  void out(uint64_t* stats) const {
    if (stats)
      for (int k = 0; k < 3; ++k) stats[k] = v[k].load();
  }
};

template <class R>
int scene_trace(const OScene<R>* s, const R* rays, size_t n, uint32_t* prim, uint32_t* obj, R* t, int threads,
                uint64_t* stats = nullptr) {
  StatSum sum;
  parallel_for(n, threads, [&](size_t b, size_t e) {
    SceneStats st;
    for (size_t i = b; i < e; ++i) {
      R tmin, tmax;
      Ray<R> r = load_ray(rays, n, i, &tmin, &tmax);
      Isect<R> it;
      uint32_t o = 0xFFFFFFFFu, p = 0xFFFFFFFFu;
      if (s->intersect(r, tmin, tmax, &it, &o, &p, stats ? &st : nullptr)) {
        prim[i] = p;
        obj[i] = o;
        t[i] = it.d;
      } else {
        prim[i] = 0xFFFFFFFFu;
        obj[i] = 0xFFFFFFFFu;
        t[i] = std::numeric_limits<R>::infinity();
      }
    }
    sum.add(st);
  });
  sum.out(stats);
  return 0;
}

template <class R>
int scene_occluded(const OScene<R>* s, const R* rays, size_t n, uint8_t* occ, int threads, uint64_t* stats = nullptr) {
  StatSum sum;
  parallel_for(n, threads, [&](size_t b, size_t e) {
    SceneStats st;
    for (size_t i = b; i < e; ++i) {
      R tmin, tmax;
      Ray<R> r = load_ray(rays, n, i, &tmin, &tmax);
      occ[i] = s->occluded(r, tmin, tmax, stats ? &st : nullptr) ? 1 : 0;
    }
    sum.add(st);
  });
  sum.out(stats);
  return 0;
}

// The scene mode of the traversal benchmark (src/bin/bvh_stats.rs:254-286): one primary ray
// per pixel centre through Scene::intersect_instrumented on [near, far]; from each hit, one
// shadow ray spawned towards `target` (Ray::spawn_from_through) through
// Scene::intersect_p_instrumented on [shadow_near, |target - p|].
// out[0..4] = primary rays, hits, nodes, boxes, objects; out[5..9] the same for shadow rays.
// With shadow_rays != NULL the shadow rays are written out (8 SoA planes of `primary rays`
// entries; rows of missed pixels hold NaN) so that another implementation can cast them.
template <class R>
void scene_cast_sets(const OScene<R>* s, const OCameraDesc* c, const double* target, double near, double far,
                     double shadow_near, uint64_t* out, R* shadow_rays) {
  const PinHoleCamera<R> cam = make_camera<R>(*c).pin;
  const V3<R> tgt{R(target[0]), R(target[1]), R(target[2])};
  SceneStats ps, ss;
  uint64_t np = 0, hp = 0, ns = 0, hs = 0;
  const size_t n = size_t(c->width) * c->height;
  for (uint32_t y = 0; y < c->height; ++y)
    for (uint32_t x = 0; x < c->width; ++x) {
      const size_t i = size_t(y) * c->width + x;
      const Ray<R> ray = cam.get_ray(R(x) + R(0.5), R(y) + R(0.5));
      ++np;
      Isect<R> it;
      uint32_t o, p;
      if (shadow_rays)
        for (int k = 0; k < 8; ++k) shadow_rays[k * n + i] = std::numeric_limits<R>::quiet_NaN();
      if (!s->intersect(ray, R(near), R(far), &it, &o, &p, &ps)) continue;
      ++hp;
      const Ray<R> sr = spawn_from_through(it.p, tgt);
      const R dist = length(tgt - it.p);
      ++ns;
      if (shadow_rays) {
        const R v[8] = {sr.o.x, sr.o.y, sr.o.z, sr.d.x, sr.d.y, sr.d.z, R(shadow_near), dist};
        for (int k = 0; k < 8; ++k) shadow_rays[k * n + i] = v[k];
      }
      if (s->occluded(sr, R(shadow_near), dist, &ss)) ++hs;
    }
  const uint64_t v[10] = {np, hp, ps.nodes_visited, ps.box_tests, ps.object_tests,
                          ns, hs, ss.nodes_visited, ss.box_tests, ss.object_tests};
  for (int k = 0; k < 10; ++k) out[k] = v[k];
}

// renderers::mt::compute_pixel (mt.rs:112-130): spp jittered samples through the pinhole
// camera, mean radiance per pixel (accumulated in f64, the film the judge image needs).
// `tally` (optional) receives the render's work counters summed over all threads.
template <class R>
int render(const OScene<R>* s, const ORenderParams* p, double* film, int threads, const CacheHook* cache = nullptr,
           WorkTally* tally = nullptr) {
  const Camera<R> cam = make_camera<R>(p->camera);
  const uint32_t w = p->camera.width, h = p->camera.height;
  const size_t npix = size_t(w) * h;
  std::mutex tally_mu;
  parallel_for(npix, threads, [&](size_t b, size_t e) {
    WorkTally local;
    work_tally = tally ? &local : nullptr;
    for (size_t pix = b; pix < e; ++pix) {
      const uint32_t x = uint32_t(pix % w), y = uint32_t(pix / w);
      double acc[3] = {0, 0, 0};
      for (uint32_t k = 0; k < p->spp; ++k) {
        Pcg32 rng = path_rng(p->seed, uint32_t(pix), p->sample_offset + k);
        const R jx = R(rng.uniform()), jy = R(rng.uniform());  // Sampler2::sample (mt.rs:145-150)
        const Ray<R> ray = cam.get_ray(R(x) + jx, R(y) + jy, rng);
        const R near = R(p->camera.near), far = R(p->camera.far);
        const V3<R> L = p->integrator == 1   ? s->li_naive(ray, near, far, p->max_depth, rng)
                        : p->integrator == 2 ? s->li_normal(ray, near, far)
                                             : s->li_path(ray, near, far, p->max_depth, p->rr_start, rng, cache);
        acc[0] += double(L.x);
        acc[1] += double(L.y);
        acc[2] += double(L.z);
      }
      for (int c = 0; c < 3; ++c) film[3 * pix + c] = acc[c] / double(p->spp);
    }
    work_tally = nullptr;
    if (tally) {
      std::lock_guard<std::mutex> lock(tally_mu);
      tally->add(local);
    }
  });
  return 0;
}

// The cache as the GPU evaluates it: the network in its BF16-emulating mode.
CacheHook cache_hook(const float* weights, const float* b6, uint32_t term_hit) {
  auto net = std::make_shared<oracle::mlp::Net>(weights, true);
  float lo[3], inv[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = b6[a];
    const float ext = b6[3 + a] - b6[a];
    inv[a] = ext > 0.f ? 1.0f / ext : 1.0f;
  }
  CacheHook h;
  h.term_hit = term_hit;
  h.query = [net, lo0 = lo[0], lo1 = lo[1], lo2 = lo[2], i0 = inv[0], i1 = inv[1], i2 = inv[2]](const float* rec,
                                                                                                  float* rgb) {
    const float l[3] = {lo0, lo1, lo2}, iv[3] = {i0, i1, i2};
    double f[oracle::mlp::kInPad], o[oracle::mlp::kOutPad];
    std::vector<std::vector<double>> acts;
    oracle::mlp::encode(rec, l, iv, f);
    net->forward(f, acts, o);
    for (int c = 0; c < 3; ++c) rgb[c] = float(o[c]);
  };
  return h;
}

template <class R>
void camera_rays(const OCameraDesc* c, R* out) {
  const PinHoleCamera<R> cam = make_camera<R>(*c).pin;
  const size_t n = size_t(c->width) * c->height;
  for (size_t pix = 0; pix < n; ++pix) {
    const Ray<R> r = cam.get_ray(R(pix % c->width) + R(0.5), R(pix / c->width) + R(0.5));
    out[pix] = r.o.x; out[n + pix] = r.o.y; out[2 * n + pix] = r.o.z;
    out[3 * n + pix] = r.d.x; out[4 * n + pix] = r.d.y; out[5 * n + pix] = r.d.z;
    out[6 * n + pix] = R(c->near); out[7 * n + pix] = R(c->far);
  }
}

}  // namespace

extern "C" {

#define ORACLE_SCENE_API(SUF, R)                                                                            \
  void* oracle_scene_new_##SUF(const OSceneDesc* d) {                                                       \
    try {                                                                                                   \
      return new OScene<R>(*d);                                                                             \
    } catch (const std::exception& e) {                                                                     \
      g_err = e.what();                                                                                     \
      return nullptr;                                                                                       \
    }                                                                                                       \
  }                                                                                                         \
  void oracle_scene_free_##SUF(void* s) { delete (OScene<R>*)s; }                                           \
  int oracle_scene_trace_##SUF(void* s, const R* rays, size_t n, uint32_t* prim, uint32_t* obj, R* t, int th) { \
    return scene_trace((OScene<R>*)s, rays, n, prim, obj, t, th);                                           \
  }                                                                                                         \
  int oracle_scene_occluded_##SUF(void* s, const R* rays, size_t n, uint8_t* occ, int th) {                 \
    return scene_occluded((OScene<R>*)s, rays, n, occ, th);                                                 \
  }                                                                                                         \
  int oracle_scene_trace_stats_##SUF(void* s, const R* rays, size_t n, uint32_t* prim, uint32_t* obj, R* t,  \
                                     int th, uint64_t* stats) {                                             \
    return scene_trace((OScene<R>*)s, rays, n, prim, obj, t, th, stats);                                    \
  }                                                                                                         \
  int oracle_scene_occluded_stats_##SUF(void* s, const R* rays, size_t n, uint8_t* occ, int th,             \
                                        uint64_t* stats) {                                                  \
    return scene_occluded((OScene<R>*)s, rays, n, occ, th, stats);                                          \
  }                                                                                                         \
  void oracle_scene_cast_sets_##SUF(void* s, const OCameraDesc* c, const double* target, double near,       \
                                    double far, double shadow_near, uint64_t* out, R* shadow_rays) {        \
    scene_cast_sets((OScene<R>*)s, c, target, near, far, shadow_near, out, shadow_rays);                    \
  }                                                                                                         \
  void oracle_scene_counts_##SUF(void* s, uint64_t* out) {                                                  \
    const OScene<R>* sc = (OScene<R>*)s;                                                                    \
    out[0] = sc->prim_root.size();                                                                          \
    out[1] = sc->unbounded.size();                                                                          \
    out[2] = sc->bnodes.size();                                                                             \
  }                                                                                                         \
  int oracle_render_##SUF(void* s, const ORenderParams* p, double* film, int th) {                          \
    try {                                                                                                   \
      return render((OScene<R>*)s, p, film, th);                                                            \
    } catch (const std::exception& e) {                                                                     \
      g_err = e.what();                                                                                     \
      return -1;                                                                                            \
    }                                                                                                       \
  }                                                                                                         \
  /* the render with its work counters: rays, shadow rays, top-level boxes, objects, mesh boxes,     \
     triangles, analytic shape tests */                                                                     \
  int oracle_render_counted_##SUF(void* s, const ORenderParams* p, double* film, int th, uint64_t* out7) {   \
    try {                                                                                                   \
      WorkTally t;                                                                                          \
      const int rc = render((OScene<R>*)s, p, film, th, nullptr, &t);                                       \
      const uint64_t v[7] = {t.rays, t.shadow_rays, t.top_boxes, t.objects, t.mesh_boxes, t.triangles,      \
                             t.shapes};                                                                     \
      for (int k = 0; k < 7; ++k) out7[k] = v[k];                                                           \
      return rc;                                                                                            \
    } catch (const std::exception& e) {                                                                     \
      g_err = e.what();                                                                                     \
      return -1;                                                                                            \
    }                                                                                                       \
  }                                                                                                         \
  int oracle_render_cached_##SUF(void* s, const ORenderParams* p, const float* weights, const float* bounds6,  \
                                 uint32_t term_hit, double* film, int th) {                                 \
    try {                                                                                                   \
      CacheHook hook = cache_hook(weights, bounds6, term_hit);                                              \
      hook.max_radiance = ((OScene<R>*)s)->max_radiance;                                                    \
      return render((OScene<R>*)s, p, film, th, &hook);                                                     \
    } catch (const std::exception& e) {                                                                     \
      g_err = e.what();                                                                                     \
      return -1;                                                                                            \
    }                                                                                                       \
  }                                                                                                         \
  void oracle_camera_rays_##SUF(const OCameraDesc* c, R* out) { camera_rays(c, out); }                     \
  void oracle_scene_bvh_##SUF(void* s, R* boxes, uint32_t* left_first, uint32_t* count, uint32_t* order) {  \
    const OScene<R>* sc = (OScene<R>*)s;                                                                    \
    for (size_t i = 0; i < sc->bnodes.size(); ++i) {                                                        \
      const auto& b = sc->bnodes[i].box;                                                                    \
      boxes[6 * i] = b.bmin.x; boxes[6 * i + 1] = b.bmin.y; boxes[6 * i + 2] = b.bmin.z;                    \
      boxes[6 * i + 3] = b.bmax.x; boxes[6 * i + 4] = b.bmax.y; boxes[6 * i + 5] = b.bmax.z;                \
      left_first[i] = sc->bnodes[i].left_first; count[i] = sc->bnodes[i].count;                             \
    }                                                                                                       \
    for (size_t i = 0; i < sc->order.size(); ++i) order[i] = sc->prim_root[sc->order[i]];                  \
  }                                                                                                         \
  size_t oracle_scene_bvh_nodes_##SUF(void* s) { return ((OScene<R>*)s)->bnodes.size(); }

ORACLE_SCENE_API(f64, double)
ORACLE_SCENE_API(f32, float)

}  // extern "C"

// ---- the radiance cache's network (mlp_oracle.hpp) ----------------------------------------

extern "C" {

static void mlp_bounds(const float* b6, float* lo, float* inv) {
  for (int a = 0; a < 3; ++a) {
    lo[a] = b6[a];
    const float ext = b6[3 + a] - b6[a];
    inv[a] = ext > 0.f ? 1.0f / ext : 1.0f;
  }
}

// The network's input features of n records (kInPad per record, the encoding the forward pass uses).
int oracle_mlp_encode(const float* bounds6, const float* records, size_t n, float* features) {
  float lo[3], inv[3];
  mlp_bounds(bounds6, lo, inv);
  for (size_t i = 0; i < n; ++i) {
    double f[oracle::mlp::kInPad];
    oracle::mlp::encode(records + i * oracle::mlp::kRecord, lo, inv, f);
    for (int k = 0; k < oracle::mlp::kInPad; ++k) features[i * oracle::mlp::kInPad + k] = float(f[k]);
  }
  return 0;
}

int oracle_mlp_forward(const float* weights, const float* bounds6, const float* records, size_t n, float* out,
                       int emulate, int threads) {
  const oracle::mlp::Net net(weights, emulate != 0);
  float lo[3], inv[3];
  mlp_bounds(bounds6, lo, inv);
  parallel_for(n, threads, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      double f[oracle::mlp::kInPad], o[oracle::mlp::kOutPad];
      std::vector<std::vector<double>> acts;
      oracle::mlp::encode(records + i * oracle::mlp::kRecord, lo, inv, f);
      net.forward(f, acts, o);
      for (int c = 0; c < 3; ++c) out[3 * i + c] = float(o[c]);
    }
  });
  return 0;
}

// BF16-emulating outputs with, per record, the smallest BF16 rounding margin of its forward
// pass (Net::forward) and the three outputs' term-magnitude sums.
int oracle_mlp_forward_margins(const float* weights, const float* bounds6, const float* records, size_t n,
                               float* out, double* margin, double* out_scale, int threads) {
  const oracle::mlp::Net net(weights, true);
  float lo[3], inv[3];
  mlp_bounds(bounds6, lo, inv);
  parallel_for(n, threads, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      double f[oracle::mlp::kInPad], o[oracle::mlp::kOutPad], sc[oracle::mlp::kOutPad];
      std::vector<std::vector<double>> acts;
      oracle::mlp::encode(records + i * oracle::mlp::kRecord, lo, inv, f);
      net.forward(f, acts, o, margin + i, sc);
      for (int c = 0; c < 3; ++c) {
        out[3 * i + c] = float(o[c]);
        out_scale[3 * i + c] = sc[c];
      }
    }
  });
  return 0;
}

// Exact-mode (FP64) outputs, for finite-difference checks of the gradient.
int oracle_mlp_forward_f64(const float* weights, const float* bounds6, const float* records, size_t n,
                           double* out) {
  const oracle::mlp::Net net(weights, false);
  float lo[3], inv[3];
  mlp_bounds(bounds6, lo, inv);
  for (size_t i = 0; i < n; ++i) {
    double f[oracle::mlp::kInPad], o[oracle::mlp::kOutPad];
    std::vector<std::vector<double>> acts;
    oracle::mlp::encode(records + i * oracle::mlp::kRecord, lo, inv, f);
    net.forward(f, acts, o);
    for (int c = 0; c < 3; ++c) out[3 * i + c] = o[c];
  }
  return 0;
}

int oracle_mlp_gradient(const float* weights, const float* bounds6, const float* records, const float* targets,
                        size_t n, double* grad, double* loss, int emulate) {
  const oracle::mlp::Net net(weights, emulate != 0);
  float lo[3], inv[3];
  mlp_bounds(bounds6, lo, inv);
  for (int p = 0; p < oracle::mlp::kParams; ++p) grad[p] = 0.0;
  const double scale = 1.0 / (double(n) * 3.0);
  double l = 0.0;
  for (size_t i = 0; i < n; ++i) {
    double f[oracle::mlp::kInPad];
    oracle::mlp::encode(records + i * oracle::mlp::kRecord, lo, inv, f);
    l += net.backward(f, targets + 3 * i, scale, grad);
  }
  *loss = l * scale;
  return 0;
}

void oracle_mlp_adam(float* w, float* m, float* v, const float* g, uint32_t step, float lr, float b1, float b2,
                     float eps) {
  oracle::mlp::adam(w, m, v, g, step, lr, b1, b2, eps);
}

}  // extern "C"
