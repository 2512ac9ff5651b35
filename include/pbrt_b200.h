/*
 * pbrt_b200.h — C ABI of the B200 wavefront path tracer.
 *
 * This is the drop-in boundary for nmichel/pbrt's data-parallel hot path: ray/BVH
 * traversal (Möller–Trumbore triangles, analytic spheres and cylinders) and the path
 * integrator's bounce loop with BSDF sampling/evaluation and light sampling. The reference
 * is a Rust crate whose seams are traits; a Rust binding would declare exactly these
 * functions in an `extern "C"` block. Each entry point names the reference interface it
 * replaces, as `path:line` inside nmichel/pbrt.
 *
 * Conventions
 *   - Every function returns a pbrt_status; 0 is success. pbrt_last_error() gives a
 *     human-readable message for the last failure on a context.
 *   - A context belongs to one host thread at a time; callers serialise per context.
 *   - Buffers passed to trace/render calls may live in host memory (pageable or pinned) or
 *     in device memory of the context's GPU; the library detects which. Host buffers are
 *     always complete when the call returns. Device buffers are complete when the call
 *     returns unless a stream was set with pbrt_ctx_set_stream(), in which case the work is
 *     ordered on that stream and pbrt_ctx_sync() reports any device-side error.
 *   - The library copies every scene description it is given; the caller keeps ownership
 *     of its arrays.
 *   - Rays are eight SoA planes of n floats each, one after another:
 *       ox[n] oy[n] oz[n] dx[n] dy[n] dz[n] tmin[n] tmax[n]
 *     Directions are used as given: they must be normalised the way the reference's
 *     Ray::new does it (src/geom/ray.rs:10-18: d * (1 / sqrt(dx*dx + dy*dy + dz*dz))).
 *   - All arithmetic on the path is IEEE FP32 with no fused multiply-add, in the
 *     reference's operation order; films are accumulated in FP64.
 */
#ifndef PBRT_B200_H
#define PBRT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pbrt_status {
  PBRT_OK = 0,
  PBRT_ERR_INVALID_ARGUMENT = 1,
  PBRT_ERR_OUT_OF_MEMORY = 2,
  PBRT_ERR_CUDA = 3,
  PBRT_ERR_DEVICE_BUDGET = 4, /* a device loop ran out of its iteration budget */
  PBRT_ERR_CAPACITY = 5,      /* a tree too deep for the traversal stack, a queue overflow */
  PBRT_ERR_UNSUPPORTED = 6
} pbrt_status;

typedef struct pbrt_ctx pbrt_ctx;
typedef struct pbrt_scene pbrt_scene;

/* Missing-hit marker written to prim_id / object_id. */
#define PBRT_MISS 0xFFFFFFFFu

/* ---------------------------------------------------------------------------------- */
/* Context                                                                              */
/* ---------------------------------------------------------------------------------- */

/* Opens a context on CUDA device `device`. No reference counterpart: the reference runs on
 * host threads (src/renderers/mt.rs:23-110). */
int pbrt_ctx_create(int device, pbrt_ctx** out);
void pbrt_ctx_destroy(pbrt_ctx* ctx);
/* Message of the last failure on `ctx` (never NULL; "" when none). */
const char* pbrt_last_error(const pbrt_ctx* ctx);
/* Orders subsequent device-buffer calls on `stream` (a cudaStream_t) without a host
 * synchronisation; NULL restores synchronous calls. */
int pbrt_ctx_set_stream(pbrt_ctx* ctx, void* stream);
/* Waits for the context's work and reports device-side errors raised since the last sync. */
int pbrt_ctx_sync(pbrt_ctx* ctx);

/* ---------------------------------------------------------------------------------- */
/* Scene description (flat POD; replaces building Scene/Object/Shape/Material/Light     */
/* trait objects: src/scene.rs:89-115, the files of src/objects/ and src/shapes/)       */
/* ---------------------------------------------------------------------------------- */

typedef enum pbrt_shape_kind {
  PBRT_SHAPE_MESH = 0,      /* TriangleMesh (src/shapes/triangle_mesh/triangle_mesh.rs:11-41) */
  PBRT_SHAPE_SPHERE = 1,    /* Sphere of `radius` at the origin (src/shapes/sphere.rs:11-23) */
  PBRT_SHAPE_CYLINDER = 2,  /* Cylinder along y, `radius`, `height` (src/shapes/cylinder.rs:7-21) */
  PBRT_SHAPE_RECTANGLE = 3, /* Rectangle::new(width = `radius`, height = `height`): the y = 0 plane within
                               |x| <= width/2, |z| <= height/2, facing +y (src/shapes/rectangle.rs:9-70) */
  PBRT_SHAPE_AABOX = 4,     /* AABox::new(`extent`): the box [-extent/2, extent/2] (src/shapes/aabox.rs:9-203) */
  PBRT_SHAPE_PLANE = 5,     /* Plane: the y = 0 plane, unbounded (src/shapes/plane.rs:9-94); an unbounded
                               primitive is kept out of the scene BVH and tested first (src/scene.rs:101-115) */
  PBRT_SHAPE_CSG = 6        /* a constructive solid over csg_elems[csg_first .. + csg_count) with csg_op
                               (src/shapes/csg.rs, csg/{union,intersection,substraction}.rs) */
} pbrt_shape_kind;

typedef enum pbrt_csg_op {
  PBRT_CSG_UNION = 0,        /* hits of each element outside every other element */
  PBRT_CSG_INTERSECTION = 1, /* hits of each element inside every other element */
  PBRT_CSG_SUBTRACTION = 2   /* the first element's hits outside the others, the others' hits inside the
                                first and outside the rest, their normals reversed */
} pbrt_csg_op;

/* One element of a constructive solid (csg::Elem, src/shapes/csg.rs:7-10): a plain shape
 * (not PBRT_SHAPE_CSG) with the sizes of pbrt_object_desc, placed by its transform. */
typedef struct pbrt_csg_elem_desc {
  uint32_t shape;
  uint32_t mesh;
  float radius, height;
  float extent[3];
  float to_world[12], to_local[12];
} pbrt_csg_elem_desc;

typedef enum pbrt_texture_kind {
  PBRT_TEXTURE_COLOR = 0,       /* PlainColor(color) (src/textures/plain_color.rs) */
  PBRT_TEXTURE_CHECKERBOARD = 1 /* CheckerBoard(color, color2, scale) on the hit's u, v
                                   (src/textures/checker_board.rs:17-28) */
} pbrt_texture_kind;

typedef enum pbrt_node_kind {
  PBRT_NODE_SIMPLE = 0,      /* an object of `objects` (Simple, src/objects/simple.rs) */
  PBRT_NODE_TRANSFORMED = 1, /* Transformed(child) (src/objects/transformed.rs) */
  PBRT_NODE_COMPOUND = 2     /* Compound(children): the nearest member's hit, the first on a tie
                                (src/objects/compound.rs:21-65) */
} pbrt_node_kind;

typedef enum pbrt_material_kind {
  PBRT_MAT_LAMBERTIAN = 0,    /* src/materials/lambertian.rs */
  PBRT_MAT_METAL = 1,         /* src/materials/metal.rs (fuzz) */
  PBRT_MAT_DIELECTRIC = 2,    /* src/materials/dielectric.rs (ior, albedo) */
  PBRT_MAT_DIFFUSE_LIGHT = 3  /* src/materials/diffuse_light.rs (emission in `color`) */
} pbrt_material_kind;

typedef enum pbrt_light_kind {
  PBRT_LIGHT_POINT = 0,               /* src/lights/point_light.rs */
  PBRT_LIGHT_UNIFORM_INFINITE = 1,    /* src/lights/uniform_infinite_light.rs */
  PBRT_LIGHT_BACKGROUND_INFINITE = 2, /* src/lights/background_infinite_light.rs */
  PBRT_LIGHT_AREA = 3                 /* the emissive surface of an object (the reference's
                                         planned AreaLight, ideas/area_light.md) */
} pbrt_light_kind;

typedef struct pbrt_mesh_desc {
  const float* vertices;    /* 3 * vertex_count floats, xyz */
  uint32_t vertex_count;
  const uint32_t* indices;  /* 3 * triangle_count vertex indices */
  uint32_t triangle_count;
  /* Optional material index per triangle (NULL: every triangle takes its object's
   * material). An extension: the reference binds one material per object. */
  const uint32_t* face_materials;
} pbrt_mesh_desc;

typedef struct pbrt_material_desc {
  uint32_t kind;  /* pbrt_material_kind */
  float color[3]; /* albedo (lambertian, metal, dielectric) or emitted radiance (diffuse light) */
  float fuzz;     /* metal */
  float ior;      /* dielectric */
  uint32_t texture; /* pbrt_texture_kind: where `color` comes from */
  float color2[3];  /* checkerboard: the second colour */
  float scale;      /* checkerboard: squares per unit of u and v */
} pbrt_material_desc;

typedef struct pbrt_object_desc {
  uint32_t shape;          /* pbrt_shape_kind */
  uint32_t mesh;           /* index into meshes, PBRT_SHAPE_MESH only */
  float radius, height;    /* sphere, cylinder; rectangle: width, height */
  uint32_t material;       /* index into materials */
  uint32_t transformed;    /* 0: Simple (src/objects/simple.rs); 1: Transformed(Simple)
                              (src/objects/transformed.rs) with the two matrices below */
  float to_world[12];      /* row-major 3x4 of Transform::mat (src/geom/transform.rs:7-10) */
  float to_local[12];      /* row-major 3x4 of Transform::inv_mat */
  float extent[3];         /* aabox: full size along x, y, z */
  uint32_t csg_op, csg_first, csg_count; /* PBRT_SHAPE_CSG: pbrt_csg_op and the elements */
} pbrt_object_desc;

/* One node of an object tree (the Object trait objects a scene file builds,
 * src/loader/visitors/scene_builder.rs:95-116). TRANSFORMED wraps children[first] with
 * the two matrices; COMPOUND holds children[first .. first + count); SIMPLE names
 * objects[object] (whose own `transformed` matrices, if set, apply innermost). A node may be
 * shared by several parents (the reference holds objects in Arc); the tree may not loop. */
typedef struct pbrt_node_desc {
  uint32_t kind;  /* pbrt_node_kind */
  uint32_t object;
  uint32_t first, count;
  float to_world[12], to_local[12];
} pbrt_node_desc;

typedef struct pbrt_light_desc {
  uint32_t kind;           /* pbrt_light_kind */
  float position[3];       /* point light, world space */
  float radiance[3];       /* point: intensity I; uniform infinite: L */
  float bottom[3], top[3]; /* background gradient: `f` at dir.y = -1, `t` at dir.y = +1 */
  uint32_t object;         /* area light: the emitting object (its material is DIFFUSE_LIGHT) */
} pbrt_light_desc;

typedef struct pbrt_scene_desc {
  const pbrt_mesh_desc* meshes;
  uint32_t mesh_count;
  const pbrt_material_desc* materials;
  uint32_t material_count;
  const pbrt_object_desc* objects;
  uint32_t object_count;
  const pbrt_light_desc* lights;
  uint32_t light_count;
  /* Mesh BVH build (src/shapes/triangle_mesh/bvh.rs:221-309): binned SAH with `bvh_bins`
   * bins (0 = the reference's 8) that stops splitting nodes of at most `bvh_max_leaf`
   * triangles (0 = the reference's 1, i.e. split while the SAH says so). */
  uint32_t bvh_bins;
  uint32_t bvh_max_leaf;
  /* Optional object tree. nodes == NULL: every object is one primitive of the scene, in
   * order (Scene::add_object for each). Otherwise the scene's primitives are the nodes
   * listed in `roots`, in that order; children indexes into `node_children`. Object ids
   * reported by the trace calls are indexes into `objects` (the Simple that was hit). */
  const pbrt_node_desc* nodes;
  uint32_t node_count;
  const uint32_t* node_children;
  uint32_t child_count;
  const uint32_t* roots;
  uint32_t root_count;
  /* 1: build the meshes' BVHs on the GPU (the same trees and triangle order as the host
   * build); mesh arrays (vertices, indices, face_materials) may then be device memory. */
  uint32_t device_build;
  /* The elements of the constructive solids among the objects. */
  const pbrt_csg_elem_desc* csg_elems;
  uint32_t csg_elem_count;
} pbrt_scene_desc;

/* Builds the acceleration structures on the host and uploads the scene. Replaces
 * Scene::commit (src/scene.rs:101-115), BVH::new (src/bvh.rs:109-132) and
 * TriangleMesh::new / BVHTree::build (src/shapes/triangle_mesh/triangle_mesh.rs:27-41,
 * bvh.rs:221-230). */
int pbrt_scene_create(pbrt_ctx* ctx, const pbrt_scene_desc* desc, pbrt_scene** out);
void pbrt_scene_destroy(pbrt_scene* scene);
/* n scenes at once: their host-side builds (BVHs) run on `threads` host threads (0: all
 * cores), then they are uploaded in order; out[i] receives scene i. On failure no scene is
 * left created. */
int pbrt_scene_create_many(pbrt_ctx* ctx, const pbrt_scene_desc* descs, uint32_t n, uint32_t threads,
                           pbrt_scene** out);

/* Host-only: builds one mesh's BVH exactly as pbrt_scene_create does and copies out the
 * flattened layout the GPU reads, without touching a GPU. `nodes` receives node_capacity
 * 32-byte records {float bmin[3]; uint32 left_first; float bmax[3]; uint32 count} in GPU
 * numbering (index 0 = root, index 1 = padding, sibling pairs at even indices);
 * `tri_order` receives triangle_count original triangle indices in leaf order. Call with
 * nodes = NULL to learn the node count through *node_count. Replaces BVHTree::new + build
 * (src/shapes/triangle_mesh/bvh.rs:179-230) for callers that inspect the tree. */
int pbrt_mesh_bvh_build_host(const pbrt_mesh_desc* mesh, uint32_t bvh_bins, uint32_t bvh_max_leaf, void* nodes,
                             uint64_t node_capacity, uint32_t* tri_order, uint64_t* node_count);
/* pbrt_mesh_bvh_build_host on the context's GPU: the binned-SAH build of
 * src/shapes/triangle_mesh/bvh.rs:221-309, 609-735 with every node split level by level by
 * many thread blocks (small subtrees by one thread each); it yields the same nodes, in the
 * same numbering, and the same triangle order. The mesh arrays may be host or device
 * memory; nodes and tri_order are host memory. build_ms (may be NULL) receives the device
 * time of the build, input copies included. */
int pbrt_mesh_bvh_build_device(pbrt_ctx* ctx, const pbrt_mesh_desc* mesh, uint32_t bvh_bins, uint32_t bvh_max_leaf,
                               void* nodes, uint64_t node_capacity, uint32_t* tri_order, uint64_t* node_count,
                               float* build_ms);

typedef struct pbrt_scene_info {
  uint64_t triangle_count;
  uint64_t mesh_node_count;  /* summed over meshes, reference numbering (no padding) */
  uint64_t mesh_leaf_count;
  uint32_t mesh_max_depth;   /* root = depth 1, as BuildStats::max_depth (bvh.rs:70) */
  uint32_t mesh_max_leaf_tris;
  uint64_t object_count;     /* the scene's primitives (Scene::primitive_count plus the unbounded ones) */
  uint64_t device_bytes;     /* device memory held by the scene */
} pbrt_scene_info;
int pbrt_scene_get_info(const pbrt_scene* scene, pbrt_scene_info* info);

/* ---------------------------------------------------------------------------------- */
/* Batched ray casting                                                                  */
/* ---------------------------------------------------------------------------------- */

/* Nearest hit per ray: replaces Scene::intersect (src/scene.rs:118-120, 186-220) and, for
 * a scene made of one untransformed mesh, TriangleMesh::intersect / BVHTree::query
 * (src/shapes/triangle_mesh/triangle_mesh.rs:73-132, bvh.rs:350-352, 450-526).
 * prim_id: triangle index within its mesh, cylinder piece (0 wall, 1 bottom, 2 top), box face
 * (0..5: -x, +x, -y, +y, -z, +z), for a constructive solid element << 24 | that element's
 * prim_id; 0 for the other shapes; PBRT_MISS on a miss.
 * t: hit distance, +inf on a miss. object_id may be NULL. */
int pbrt_trace_closest(pbrt_scene* scene, const float* rays, uint64_t n, uint32_t* prim_id, float* t,
                       uint32_t* object_id);

/* pbrt_trace_closest plus the traversal's work counters summed over all rays:
 * stats[0] nodes visited, stats[1] ray/box tests, stats[2] ray/triangle tests. Replaces
 * TriangleMesh::intersect_instrumented (src/shapes/triangle_mesh/triangle_mesh.rs:49-53)
 * and BVHTree::query_instrumented (bvh.rs:359-361); the counts are those of
 * TraversalStats (bvh.rs:18-47), so they equal the reference's for the same tree. */
int pbrt_trace_closest_instrumented(pbrt_scene* scene, const float* rays, uint64_t n, uint32_t* prim_id, float* t,
                                    uint64_t* stats);

/* pbrt_trace_closest for callers that cannot call cudaMalloc — a host application that
 * owns every device allocation through its own pool and budget (a renderer embedding this
 * tracer as a plugin), or code on a latency-critical path where cudaMalloc's implicit
 * synchronisation and unpredictable cost are not acceptable. No counterpart in the
 * reference. It allocates nothing: its scratch (survivor queue, counters, error word) is a
 * fixed static device array of PBRT_NOALLOC_MAX_RAYS queue entries (4 MiB + 256 B) that
 * every GPU which loads the library holds until the process exits.
 *   - rays, prim_id and t must be device memory of the context's GPU; n must not exceed
 *     PBRT_NOALLOC_MAX_RAYS (PBRT_ERR_CAPACITY otherwise; split larger batches).
 *   - pbrt_ctx_create looks the array's address up on its device; that also loads the
 *     trace kernels there, so the array's memory is committed when the context is created
 *     (a context that cannot get it fails to create) and never inside this call.
 *   - Every call shares the one array: calls that overlap on the GPU (other streams, other
 *     threads, other contexts on the same device) race and corrupt each other's results.
 *   - It runs on the context's stream (pbrt_ctx_set_stream) and returns when its results
 *     are complete, with device-side errors reported in its status. Because it waits for
 *     them, it refuses a stream that is being captured (PBRT_ERR_UNSUPPORTED, nothing
 *     enqueued) instead of invalidating the capture.
 *   - n = 0 returns PBRT_OK whatever the scene, as pbrt_trace_closest does.
 * Results are identical to pbrt_trace_closest's. */
#define PBRT_NOALLOC_MAX_RAYS 1048576u
int pbrt_trace_closest_noalloc(pbrt_scene* scene, const float* rays, uint64_t n, uint32_t* prim_id, float* t);

/* Whether anything blocks each ray within [tmin, tmax]: replaces Scene::intersect_p
 * (src/scene.rs:143-168) and BVHTree::intersect_p (src/shapes/triangle_mesh/bvh.rs:381-420). */
int pbrt_trace_any(pbrt_scene* scene, const float* rays, uint64_t n, uint8_t* occluded);

/* The scene-level queries with the scene accelerator's work counters summed over all rays
 * (any scene): stats[0] nodes visited, stats[1] ray/box tests, stats[2] object tests
 * (primitives asked, the unbounded ones included), counted as TraversalStats counts them in
 * Scene::intersect_instrumented / Scene::intersect_p_instrumented (src/scene.rs:124-153,
 * src/bvh.rs:153-275). The meshes' inner traversals are not counted, as in the reference. */
int pbrt_trace_closest_counted(pbrt_scene* scene, const float* rays, uint64_t n, uint32_t* prim_id, float* t,
                               uint32_t* object_id, uint64_t* stats /* 3 */);
int pbrt_trace_any_counted(pbrt_scene* scene, const float* rays, uint64_t n, uint8_t* occluded,
                           uint64_t* stats /* 3 */);

/* ---------------------------------------------------------------------------------- */
/* Rendering                                                                            */
/* ---------------------------------------------------------------------------------- */

/* PinHoleCamera::new(resolution, fov, near, far, Matrix4::look_at(position, look_at, up))
 * (src/cameras/pin_hole.rs:17-38, src/geom/matrix4.rs:70-98), or with thin_lens = 1
 * ThinLensCamera::new(.., lens_radius, focal_distance, ..) (src/cameras/thin_lens.rs:21-75),
 * whose rays start on a disk of lens_radius (random_in_unit_disk, drawn after the pixel
 * jitter) and pass through the point at focal_distance along the pinhole ray. near/far are
 * also every ray's [near, far] interval, as the reference passes Config::near/far to li(). */
typedef struct pbrt_camera_desc {
  uint32_t width, height;
  float fov; /* full field of view, radians */
  float near, far;
  float position[3], look_at[3], up[3];
  uint32_t thin_lens;
  float lens_radius, focal_distance;
} pbrt_camera_desc;

typedef enum pbrt_integrator {
  PBRT_INTEGRATOR_PATH = 0,  /* PathIntegrator (src/integrators/path.rs:48-115) + area-light NEE */
  PBRT_INTEGRATOR_NAIVE = 1, /* NaiveIntegrator (src/integrators/naive.rs:29-52), background = the
                                scene's infinite lights */
  PBRT_INTEGRATOR_NORMAL = 2 /* NormalIntegrator (src/integrators/normal.rs:17-30): (n + 1) / 2 of the
                                first hit, the infinite lights on a miss */
} pbrt_integrator;

typedef struct pbrt_render_params {
  pbrt_camera_desc camera;
  uint32_t spp;           /* Config::samples_ppx */
  uint32_t max_depth;     /* PathIntegrator::max_depth */
  uint32_t rr_start;      /* Russian roulette from this bounce (q = min(1, max beta)); 0 = off, as the
                             reference's is commented out (path.rs:92-101) */
  uint32_t sample_offset; /* index of the first sample: progressive rendering, resume */
  uint64_t seed;          /* PCG32, one stream per pixel, re-keyed per (pixel, sample) */
  uint32_t integrator;    /* pbrt_integrator */
  uint32_t pixel_stride;  /* 0 or 1: every pixel. s > 1: only the pixels (s*i, s*j), each rendered
                             exactly as a full render renders it (same sample streams); the film
                             is then ceil(width/s) x ceil(height/s) */
} pbrt_render_params;

/* Mean radiance per pixel over spp samples into film_rgb (width*height*3 doubles, row-major,
 * row 0 at the top; see pixel_stride), host or device memory; per-sample radiance is FP32,
 * the film FP64.
 * Replaces renderers::mt::render / st::render (src/renderers/mt.rs:23-110, 112-130). */
int pbrt_render(pbrt_scene* scene, const pbrt_render_params* params, double* film_rgb);

/* ---------------------------------------------------------------------------------- */
/* Learned radiance cache (no counterpart in the reference: an extension of the path    */
/* integrator, src/integrators/path.rs:48-115, that ends paths into a network)          */
/* ---------------------------------------------------------------------------------- */

typedef struct pbrt_cache pbrt_cache;

/* Network: 82 features (12-band sin/cos encoding of the position normalised to the scene
 * box, 72 values; outgoing direction, normal, albedo, roughness) -> 5 x 64 ReLU -> RGB, no
 * biases, BF16 weights, FP32 accumulation on the tensor cores; relative-L2 loss; Adam. */
#define PBRT_CACHE_PARAMS 23552u /* weights, row-major out x in per layer, last layer padded to 16 rows */
#define PBRT_CACHE_RECORD 16u    /* floats per query record: p.xyz, roughness, wo.xyz, 0, n.xyz, 0, albedo.xyz, 0 */

typedef struct pbrt_cache_params {
  uint64_t seed;            /* weight initialisation */
  float learning_rate;      /* Adam step size; 0 = 1e-2 */
  float beta1, beta2;       /* 0 = 0.9, 0.99 */
  float epsilon;            /* 0 = 1e-8 */
  float scene_min[3], scene_max[3]; /* the box positions are normalised to */
  uint32_t terminate_bounce; /* paths end into the cache at this hit; 0 = 2 */
  uint32_t train_samples;    /* training samples per cached frame; 0 = 65536 */
  uint32_t train_steps;      /* Adam steps per cached frame; 0 = 4 */
} pbrt_cache_params;

int pbrt_cache_create(pbrt_ctx* ctx, const pbrt_cache_params* params, pbrt_cache** out);
void pbrt_cache_destroy(pbrt_cache* cache);
/* Back to the seeded initial weights, zero Adam moments. */
int pbrt_cache_reset(pbrt_cache* cache);
int pbrt_cache_get_weights(pbrt_cache* cache, float* weights /* PBRT_CACHE_PARAMS */);
int pbrt_cache_set_weights(pbrt_cache* cache, const float* weights);
/* rgb[3*i..3*i+2] = network(record i); host or device buffers. */
int pbrt_cache_query(pbrt_cache* cache, const float* records, uint64_t n, float* rgb);
/* Gradient of the mean relative-L2 loss over a batch (grad: PBRT_CACHE_PARAMS floats); the
 * loss is reported through *loss when not NULL. Weights are not changed. */
int pbrt_cache_gradient(pbrt_cache* cache, const float* records, const float* targets, uint64_t n, float* grad,
                        float* loss);
/* One Adam step on a batch. */
int pbrt_cache_train_step(pbrt_cache* cache, const float* records, const float* targets, uint64_t n, float* loss);
/* Checkpoint of the weights and Adam state (pass buf = NULL to learn the size). */
int pbrt_cache_save(pbrt_cache* cache, void* buf, uint64_t capacity, uint64_t* size);
int pbrt_cache_load(pbrt_cache* cache, const void* buf, uint64_t size);

/* Path tracing that ends paths into the learned radiance cache (an extension of
 * PathIntegrator::li, src/integrators/path.rs:48-115; the reference has no counterpart).
 * First `train_rounds` rounds of online training. A round traces max(128, train_samples / 4)
 * path-integrator paths from random pixels; each ends into the cache itself three hits after
 * the render's cache hit (the cache's answer there closes the path), and each Lambertian or
 * metal vertex before that (at most train_samples of them) is recorded with the radiance the
 * rest of its path gathered, divided by the throughput at the vertex. The round then takes
 * train_steps Adam steps, each on max(128, train_samples / train_steps) vertices drawn with
 * replacement from the recorded ones (no step when none were recorded).
 * Then params->spp samples per pixel are rendered as pbrt_render renders them, except that a
 * path whose hit number terminate_bounce + 1 (or a later one, after a dielectric) lies on a
 * Lambertian or metal surface stops there: it takes no light sample at that hit and adds
 * its throughput times the network's output clamped to [0, Lmax]. Lmax is the largest
 * radiance an emitter of the scene gives off (diffuse-light materials, infinite lights;
 * unbounded with a point light): no energy-conserving surface reflects more. Training
 * targets are clamped the same way. spp = 0 only trains (film may be NULL). A call that
 * both trains (train_rounds > 0) and renders (spp > 0) runs its rounds beside the frame, on
 * a second stream: the frame reads the weights the cache held when the call started, and
 * the call's work ends with the weights its rounds trained. The integrator must be
 * PBRT_INTEGRATOR_PATH. A cache whose scene box is empty (scene_min ==
 * scene_max) takes the scene's bounds on first use. */
int pbrt_render_cached(pbrt_scene* scene, pbrt_cache* cache, const pbrt_render_params* params, uint32_t train_rounds,
                       double* film_rgb);

/* ---------------------------------------------------------------------------------- */
/* Tuning and batches of scenes                                                         */
/* ---------------------------------------------------------------------------------- */

/* Launch shape of the wavefront renderer (pbrt_render, pbrt_render_cached, batches created
 * afterwards). Zero fields take the defaults. */
typedef struct pbrt_tuning {
  uint32_t wave_paths;          /* paths in flight per wave (the queues' capacity), [1024, 2^26]; 0 = 2^26.
                                 * A render allocates 136 bytes of path state per path of min(its paths,
                                 * wave_paths); fewer waves leave fewer per-bounce kernel tails (10,000
                                 * spheres at 1024x768x64 spp: 139.7 ms a frame at 2^22, 103.7 ms at 2^26) */
  uint32_t trace_threads;       /* threads per block of the traversal kernels, multiple of 32 <= 256; 0 = 128 */
  uint32_t trace_blocks_per_sm; /* their grid = SMs x this, [1, 64]; 0 = 16 */
  uint32_t shade_threads;       /* the shading kernel's; 0 = 128 */
  uint32_t shade_blocks_per_sm; /* 0 = 16 */
} pbrt_tuning;

int pbrt_ctx_set_tuning(pbrt_ctx* ctx, const pbrt_tuning* tuning /* NULL: defaults */);
int pbrt_ctx_get_tuning(pbrt_ctx* ctx, pbrt_tuning* tuning);

/* Many scenes rendered together (no counterpart in the reference, whose renderer takes one
 * scene): the paths of all scenes share the waves, queues and kernel launches of one
 * wavefront (or one persistent launch, pbrt_ctx_set_batch_kernel), scene by scene, cheapest
 * first (pixels x spp x max depth; ties keep the given order, which minimises the frame's
 * mean completion time), and the launch sequence of one frame is recorded once in a CUDA
 * graph that pbrt_batch_render replays. The scenes must
 * belong to ctx and outlive the batch; params[i] (integrator path or naive) renders
 * scenes[i]; films and times are reported per caller index i. */
typedef struct pbrt_batch pbrt_batch;
int pbrt_batch_create(pbrt_ctx* ctx, pbrt_scene* const* scenes, const pbrt_render_params* params, uint32_t n,
                      pbrt_batch** out);
/* Frame `frame`: scene i takes samples sample_offset + frame * spp ... + spp - 1 of every
 * pixel. films[i] (host or device, scene i's film size; films or films[i] may be NULL)
 * receives the mean radiance. scene_ms (optional, n floats): device milliseconds from the
 * frame's start until the wave holding scene i's last paths finished (persistent batches:
 * until its last path finished). */
int pbrt_batch_render(pbrt_batch* batch, uint32_t frame, double* const* films, float* scene_ms);
void pbrt_batch_destroy(pbrt_batch* batch);
/* How batches created afterwards run a frame. PBRT_BATCH_WAVEFRONT (the default): waves of
 * paths through the wavefront's queues, one kernel per stage and bounce. PBRT_BATCH_PERSISTENT:
 * one persistent launch in which each warp lane runs a path to its end (nearest hit, shading,
 * shadow ray, film) and takes the next; scene_ms then comes from the GPU clock at the moment a
 * scene's last path finished. Films are the same either way. */
enum { PBRT_BATCH_WAVEFRONT = 0, PBRT_BATCH_PERSISTENT = 1 };
int pbrt_ctx_set_batch_kernel(pbrt_ctx* ctx, int kind);
/* Concurrent branches of the wavefront frame of batches created afterwards, [1, 8]; default 2.
 * With k > 1 the frame's waves are spread over k streams inside the graph, each with its own
 * wave buffers (136 bytes per path of its largest wave): the waves of one scene stay on one
 * branch, and each group of waves goes to the branch with the least work so far. The GPU then
 * fills one branch's per-bounce kernel tails with another's work (64 scenes of 512x512 at 4-64
 * spp: 2.19 s a frame on one branch, 1.95 s on two or more). Scenes packed into one shared wave
 * form one group. Films are the same for any k; scenes complete cheapest first within a branch. */
int pbrt_ctx_set_batch_branches(pbrt_ctx* ctx, uint32_t branches);
/* pbrt_batch_create + pbrt_batch_render(frame 0) + pbrt_batch_destroy. */
int pbrt_render_batch(pbrt_scene* const* scenes, const pbrt_render_params* params, uint32_t n, double* const* films);

/* Work of the last pbrt_render / pbrt_render_cached / pbrt_batch_render on this context: stats[0] rays traced
 * to their nearest hit (camera and bounce rays, training paths included), stats[1] shadow
 * rays, stats[2] paths started. Synchronises the context's stream. */
int pbrt_ctx_render_stats(pbrt_ctx* ctx, uint64_t* stats /* 3 */);

/* ---------------------------------------------------------------------------------- */
/* Scene files (host only, no GPU work)                                                 */
/* ---------------------------------------------------------------------------------- */

/* A parsed `.stage` scene file: Parser::parse + SceneBuilderVisitor
 * (src/loader/parser.rs:13-367, src/loader/parser/lexer.rs, src/loader/visitors/scene_builder.rs)
 * with its meshes read from ASCII PLY files (src/loader/mesh_loader.rs, src/loader/ply/). */
typedef struct pbrt_stage pbrt_stage;

/* The settings Loader::load_scene takes from its Config (src/config.rs:112-129); zero fields
 * take the reference's defaults. */
typedef struct pbrt_stage_options {
  const char* base_dir;      /* mesh file names are read relative to it (NULL or "": as given) */
  uint32_t width, height;    /* Config::output_width/height; 0 = 800 x 600 */
  double fov_deg;            /* Config::fov_deg; 0 = 90 */
  double near, far;          /* Config::near/far; 0 = 1e-4 / 1000 */
  uint32_t no_loader_lights; /* 0: add the point light at (0, 2, 1) of intensity 15 and the white-to-
                                (0.5, 0.7, 1.0) background light that Loader::load_scene adds to every
                                scene (src/loader.rs:36-42); 1: add none */
  uint32_t bvh_bins, bvh_max_leaf; /* copied into the scene description */
} pbrt_stage_options;

/* Parses `text` (a whole scene file) and reads its meshes. On failure returns
 * PBRT_ERR_INVALID_ARGUMENT (a file the reference's parser rejects) or PBRT_ERR_UNSUPPORTED
 * (a constructive solid nested in another), with a message in err. */
int pbrt_stage_parse(const char* text, const pbrt_stage_options* options, pbrt_stage** out, char* err,
                     size_t err_len);
/* The scene description (pointing into arrays the stage owns, valid until
 * pbrt_stage_destroy) and the camera (the file's pos/look/up, pin_hole or thin_lens, with
 * the options' resolution, field of view and planes). Either output may be NULL.
 * camera_lens (2 floats, may be NULL) receives the thin lens' radius and focal distance
 * (0, 0 for a pin_hole camera). */
int pbrt_stage_describe(const pbrt_stage* stage, pbrt_scene_desc* desc, pbrt_camera_desc* camera,
                        float* camera_lens);
void pbrt_stage_destroy(pbrt_stage* stage);
/* Loader::load_scene (src/loader.rs:29-45): parse + pbrt_scene_create. camera may be NULL. */
int pbrt_scene_load(pbrt_ctx* ctx, const char* text, const pbrt_stage_options* options, pbrt_scene** scene,
                    pbrt_camera_desc* camera);
/* load_ply_mesh(path, reverse) (src/loader/mesh_loader.rs:13-24): vertices (3 floats each) and
 * triangles (3 indices each; reversed winding when reverse != 0) of an ASCII PLY file,
 * allocated with malloc (release with pbrt_free). Faces must be triangles. */
int pbrt_ply_read(const char* path, int reverse, float** vertices, uint32_t* vertex_count, uint32_t** indices,
                  uint32_t* triangle_count, char* err, size_t err_len);
void pbrt_free(void* p);

/* Spectrum::gamma_correct + to_rgb (src/spectrum.rs:13-25, 134-136): sqrt gamma, clip to
 * [0, 1], truncate to 8 bits, alpha 255, as image_write stores it (mt.rs:152-167). Host
 * buffers; no GPU work. */
int pbrt_film_to_rgba8(const double* film_rgb, uint32_t width, uint32_t height, uint8_t* rgba);

/* image_write (src/renderers/mt.rs:152-167): an 8-bit RGBA PNG of width x height pixels
 * (row-major, row 0 at the top) at `path`. The pixels decode to exactly `rgba`; the
 * compressed bytes are the library's own (stored deflate blocks). Host only. */
int pbrt_write_png(const char* path, const uint8_t* rgba, uint32_t width, uint32_t height);

#ifdef __cplusplus
}
#endif

#endif /* PBRT_B200_H */
