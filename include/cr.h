/*
 * cr.h: C ABI of the B200-native Radiance path tracer (libcr_b200.so).
 *
 * Drop-in replacement for the Radiance path of xlnx/cuda-raytracer
 * ("Koishi").  Each entry point names the reference interface it replaces
 * (paths are inside that project).  Plain C types only: pointers, sizes and
 * opaque handles; no exceptions cross this boundary.  Every call returns
 * CR_OK (0) or a negative CR_ERR_* code, with a message in cr_last_error().
 *
 * Ownership: the library owns every device buffer it allocates; caller host
 * arrays are copied during the call.  A cr_scene is not thread-safe for
 * mutation; renders of distinct scenes may run concurrently on distinct
 * streams.  `stream` arguments are cudaStream_t values passed as void*
 * (NULL = the legacy default stream).
 */
#ifndef CR_H
#define CR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CR_OK 0
#define CR_ERR_INVALID -1     /* bad argument or malformed input            */
#define CR_ERR_PARSE -2       /* JSON / mesh file could not be read          */
#define CR_ERR_CUDA -3        /* a CUDA call failed                          */
#define CR_ERR_STATE -4       /* call not valid in the scene's current state */
#define CR_ERR_UNSUPPORTED -5 /* feature named in input is not implemented   */
#define CR_ERR_DEVICE -6      /* a kernel reported an internal error flag    */

/* Estimators of the Radiance kernel. */
#define CR_ESTIMATOR_KOISHI 0 /* reference semantics (radiance.cu:14-81)     */
#define CR_ESTIMATOR_MIS 1    /* power-heuristic MIS of BSDF and area NEE    */

typedef struct cr_scene cr_scene;

/* One ray query result.  prim is the primitive index in scene order (meshes
 * of an import asset in file order, spheres in asset order), tri the
 * triangle index within that mesh (-1 for spheres), prim = -1 on a miss. */
typedef struct cr_hit {
    int32_t prim;
    int32_t tri;
    float t;
    float u; /* barycentric weight of the triangle's second vertex */
    float v; /* barycentric weight of the triangle's third vertex  */
} cr_hit;

typedef struct cr_render_desc {
    uint32_t width, height, spp;
    uint32_t max_bounce;     /* UINT32_MAX: the scene's kernel "maxBounce" (default 16) */
    int32_t estimator;       /* CR_ESTIMATOR_*, or -1: the scene's kernel "estimator"   */
    uint32_t x0, y0, x1, y1; /* pixel window [x0,x1)x[y0,y1); all zero = whole image    */
    uint64_t seed;           /* Philox key for this render                             */
    uint32_t wave_paths;     /* paths in flight per wave; 0 = autotuned default        */
    int32_t guiding;         /* 1: learned path guiding (estimator MIS only)           */
    int32_t count_work;      /* 1: also count BVH nodes / triangles visited            */
    uint32_t refill_min;     /* traversal: idle lanes of 32 that trigger a refill; 0 = tuned */
    uint32_t traverse_blocks_per_sm; /* traversal grid, 1..8 blocks per SM; 0 = tuned    */
    uint32_t shade_threads;  /* shading block size: 64, 128 or 256; 0 = tuned           */
    uint32_t rr_start;       /* MIS estimator: first bounce at which Russian roulette may
                                end a path; 0 = the default: 4 (the reference's "after
                                bounce 3", which the reference estimator always uses) for
                                plain renders, none for guided renders; above max_bounce: none */
    int32_t bin_rays;        /* 1: sort each secondary and shadow traversal queue by (ray
                                octant, origin cell) before tracing; -1: trace in queue
                                order; 0 = tuned (off until cr_autotune picks it) */
    uint32_t shadow_vote;    /* any-hit traversal: a warp tests triangles once shadow_vote x
                                (lanes with triangles pending) >= its active lanes, 1..32;
                                0 = tuned (4 until cr_autotune picks it) */
    uint32_t shadow_refill_min; /* any-hit traversal: idle lanes of 32 that trigger a refill;
                                0 = tuned (refill_min until cr_autotune picks it) */
} cr_render_desc;

/* Launch configuration chosen by cr_autotune (also used by later renders of
 * the scene whose desc fields are 0). */
typedef struct cr_tuning {
    uint32_t wave_paths;
    uint32_t refill_min;
    uint32_t traverse_blocks_per_sm;
    uint32_t candidates_tried;
    double msamples_per_s;   /* rate of the chosen configuration on the sample render */
    double default_msamples_per_s; /* rate of the built-in defaults on the same sample */
    uint32_t shade_threads;  /* shading block size */
    int32_t bin_rays;        /* 1: ray binning chosen, -1: not */
    uint32_t shadow_vote;    /* any-hit triangle-step vote */
    uint32_t shadow_refill_min; /* any-hit refill threshold */
} cr_tuning;

typedef struct cr_stats {
    double ms_total;       /* device time of the whole render (CUDA events)  */
    double ms_extend;      /* closest-hit traversal kernels                   */
    double ms_shadow;      /* any-hit (shadow) traversal kernels              */
    double ms_shade;       /* shading / NEE / queue compaction kernels        */
    double ms_other;       /* generation, film accumulation, guiding          */
    double ms_guide;       /* guide inference and training (part of ms_other) */
    uint64_t samples;      /* camera paths traced                             */
    uint64_t rays_extend;  /* closest-hit queries                             */
    uint64_t rays_shadow;  /* any-hit queries                                 */
    uint64_t nodes;        /* closest-hit: wide-BVH nodes fetched (count_work = 1) */
    uint64_t tris;         /* closest-hit: triangles tested (count_work = 1)       */
    uint64_t shadow_nodes; /* any-hit: wide-BVH nodes fetched (count_work = 1)     */
    uint64_t shadow_tris;  /* any-hit: triangles tested (count_work = 1)           */
    uint32_t launches;     /* kernels launched by the call                    */
    uint32_t waves;        /* waves of paths                                  */
    uint32_t extend_launches;
    uint32_t shadow_launches;
    double ms_guide_train; /* guide training steps (part of ms_guide)         */
    uint32_t graph_nodes;  /* cr_batch_render: kernel nodes of the replayed CUDA graph
                              (an initialising kernel and the wave loop's body, which
                              runs once per wave); 0 for other calls            */
    uint32_t guide_launches; /* guide inference launches (one per guided bounce of a wave) */
    uint64_t guide_rows;     /* paths the guide's inference ran on (its rows)  */
} cr_stats;

/* ------------------------------------------------------------------ errors */
/* Message for the last failing call on this thread.                        */
const char *cr_last_error(void);
/* Library version string. */
const char *cr_version(void);
/* No counterpart in the reference.  The library's stream-ordered device
 * memory (wave state: about 140 bytes per path in flight; the BVH build's
 * scratch; upload staging; the films of host-array calls) comes from a memory
 * pool of its own per device, which keeps freed memory mapped so that the
 * next scene or render reuses it: between calls a process holds up to its
 * largest concurrent use.  This hands that cached memory back to the device
 * (scenes alive keep their own buffers). */
int cr_trim_memory(void);

/* ------------------------------------------------------------------ scenes */
/* Scene::Scene(const Properties&) (src/core/meta/scene.cu:18-219) together
 * with the Renderer's configuration read (src/core/renderer/renderer.cu:13-24,
 * renderer.hpp:17-23): parses the reference JSON schema, loads the
 * ["import", {"path"}] mesh file (OBJ, or the CRM binary mesh format,
 * resolved against base_dir), spheres, pointLight assets, shaders and
 * cameras, and makes every Emission-shaded primitive an area light.  The scene is committed
 * (uploaded, BVH built) before return. */
int cr_scene_create(const char *json_text, const char *base_dir, cr_scene **out);

/* An empty scene to be filled by the cr_scene_add_* calls below, then
 * cr_scene_commit. */
int cr_scene_create_empty(cr_scene **out);

/* Factory<Shader>::create (src/core/basic/factory.hpp:15-23) over the shader
 * registry of src/ext/shader/shader.impl.cu:15-24: Lambert, GlossyBSDF
 * (Beckmann or Cosine distribution), Emission, Transparent, Blackhole,
 * RefractionBSDF, GlassBSDF and Mixed (fac Constant or Fresnel, nested
 * Mixed up to 16 deep).  config_json is the reference's [Type, {props}]
 * array.  CR_ESTIMATOR_KOISHI renders them all with the reference's
 * semantics; CR_ESTIMATOR_MIS with physically restated BSDFs (rough
 * dielectrics after Walter et al. 2007, Transparent as a delta pass-through)
 * for microfacet shaders with the Beckmann distribution and Mixed of two
 * leaves, and refuses the rest (Cosine-distribution microfacet shaders,
 * nested Mixed).
 * Returns the shader id (>= 0) or an error code. */
int cr_scene_add_shader(cr_scene *s, const char *name, const char *config_json);

/* PolyMesh(vertices, normals, indices) (src/core/primitive/mesh.cu:404-433):
 * one triangle mesh with per-vertex normals, shaded by the named shader.
 * Returns the primitive id (>= 0) or an error code. */
int cr_scene_add_mesh(cr_scene *s, const float *vertices, uint32_t n_vertices, const float *normals,
                      const uint32_t *indices, uint32_t n_triangles, const char *shader);

/* The "sphere" asset (src/core/meta/scene.cu:136-156, sphere.hpp:9-16). */
int cr_scene_add_sphere(cr_scene *s, const float *center, float radius, const char *shader);

/* The "pointLight" asset (src/core/meta/scene.cu:156-163, pointLight.hpp:13-18):
 * emission = color (null: white) * strength, delivered to a lit point without
 * distance falloff (the reference estimator; CR_ESTIMATOR_MIS treats it as a
 * point of intensity color * strength, with 1/r^2 falloff).  Point lights
 * precede the area lights in the light list.  Returns the point light's index. */
int cr_scene_add_point_light(cr_scene *s, const float *position, const float *color, float strength);

/* CameraConfig (src/util/config.hpp:12-35), pinhole lens; `target` is a
 * direction, fovx the horizontal field of view in degrees. */
int cr_scene_set_camera(cr_scene *s, const float *position, const float *target, const float *upaxis,
                        float fovx);

/* CameraConfig::lens ("pinhole" / "orthographic", config.hpp:14-27), which
 * the Renderer turns into a PinholeLens or an OrthographicLens
 * (src/core/renderer/renderer.cu:30-38, lens.hpp:40-66).  The orthographic
 * lens shoots along the view direction from the camera position moved by
 * the image-plane offset times 4 / width.  Call after cr_scene_set_camera. */
#define CR_LENS_PINHOLE 0
#define CR_LENS_ORTHOGRAPHIC 1
int cr_scene_set_lens(cr_scene *s, int lens);

/* Upload and build the quantised 8-wide BVH on the GPU; replaces the host
 * builder createBVH / doCreateBVH (src/core/primitive/mesh.cu:35-143).
 * light_seed seeds the reference-compatible light-point tables
 * (src/core/primitive/mesh.hpp:61-84). */
int cr_scene_commit(cr_scene *s, uint64_t light_seed, void *stream);
/* cr_scene_commit with the light seed that scene loading uses (the 48-bit
 * state 0x330E) on the scene's own stream: the one-call BVH build. */
int cr_bvh_build(cr_scene *s);

/* Parses a mesh file the way an ["import", {"path"}] asset does (OBJ with
 * per-usemtl groups, PLY as one "DefaultMaterial" group, or CRM) without
 * building a scene: groups, vertices, triangles and a checksum of the
 * triangle corner positions.  Host only; replaces the Assimp::Importer read
 * of Scene::Scene (src/core/meta/scene.cu:37-44). */
int cr_mesh_file_info(const char *path, uint32_t *n_groups, uint64_t *n_vertices, uint64_t *n_triangles,
                      double *checksum);

/* Selects the kernel by its Factory<Kernel> name (kernel.impl.cu:10-15), as
 * the scene file's ["tracer", {"kernel": [name, ...]}] or `cr -k` does:
 * "Radiance" (default), or the debug kernels "Normal" (shading normal * 0.5 +
 * 0.5, normal.hpp:17-31), "Visibility" (1 where a sample of light 0 is
 * unoccluded, visibility.hpp:17-41) and "HalfVector" (angle of the view/light-0
 * half vector from the normal, * 2 / pi, halfVector.hpp:17-43). */
int cr_scene_set_kernel(cr_scene *s, const char *name);

/* No counterpart in the reference.  BVH build options, set before
 * cr_scene_commit (defaults in brackets):
 *   builder      CR_BUILD_PLOC: locally-ordered clustering [default], or
 *                CR_BUILD_LBVH: the Morton radix tree (faster build, more
 *                nodes visited per ray)
 *   ploc_radius  clustering search radius in Morton positions [10]
 *   max_leaf     triangles per leaf, 1..3 [3]
 *   cost_node, cost_tri  binary-tree SAH costs of a node visit and a triangle
 *                test [1.2, 1]
 *   collapse     CR_COLLAPSE_SAH: plan the 8-wide collapse by dynamic
 *                programming over the SAH (PLOC trees) [default], or
 *                CR_COLLAPSE_GREEDY: open the largest child first
 *   wide_cost_node, wide_cost_tri  SAH costs of a wide-node visit and a
 *                triangle test in that plan [1, 0.6] */
#define CR_BUILD_PLOC 0
#define CR_BUILD_LBVH 1
#define CR_COLLAPSE_SAH 0
#define CR_COLLAPSE_GREEDY 1
typedef struct cr_build_config {
    int32_t builder;
    uint32_t ploc_radius;
    uint32_t max_leaf;
    float cost_node;
    float cost_tri;
    int32_t collapse;
    float wide_cost_node;
    float wide_cost_tri;
} cr_build_config;
int cr_scene_set_build(cr_scene *s, const cr_build_config *cfg);

/* Counts after commit. */
int cr_scene_info(const cr_scene *s, uint64_t *n_triangles, uint32_t *n_primitives, uint32_t *n_lights,
                  uint32_t *n_bvh_nodes);

void cr_scene_destroy(cr_scene *s);

/* The 1024-point table of light `light` (mesh lights only; Mesh::samples,
 * src/core/primitive/mesh.hpp:58-84): out = 1024 x {p.xyz, n.xyz}; *pdf the
 * table's area pdf. */
int cr_light_table(const cr_scene *s, uint32_t light, float *out, float *pdf);

/* ------------------------------------------------------------- ray queries */
/* Scene::intersect(Ray, ...) (src/core/meta/scene.hpp:35-55) when any_hit = 0,
 * Scene::intersect(Seg, ...) (scene.hpp:57-67) when any_hit = 1, batched.
 * rays: n x {o.x,o.y,o.z, d.x,d.y,d.z, tmax} floats (tmax <= 0 or inf: none).
 * Host buffers; copies are part of the call. */
int cr_trace_rays(cr_scene *s, const float *rays, uint64_t n, cr_hit *hits, int any_hit);
/* No counterpart in the reference.  The traversal work of the same queries:
 * work[0] = wide-BVH nodes fetched (80 bytes each), work[1] = primitives
 * tested (48-byte records), summed over the n rays (the counting build of the
 * traversal kernel; the hits are discarded).  With the reference's own work
 * on the same rays (binary nodes of 36 bytes, faces of 36 bytes) it gives
 * the bytes per query of both layouts. */
int cr_trace_work(cr_scene *s, const float *rays, uint64_t n, int any_hit, uint64_t work[2]);
/* Mesh::samples and Mesh::pdf (src/core/primitive/mesh.hpp:58-84) handed over
 * from a reference Scene: replaces the 1024-point light table (points
 * 1024 x {p.xyz, n.xyz}) and the area pdf that the reference estimator's
 * AreaLight::sample (src/core/light/areaLight.hpp:19-31) draws from, for the
 * emissive mesh `primitive` (the id cr_scene_add_mesh returned) of a
 * committed scene.  The Tracer plugin uses it so that the GPU samples the very
 * light points the reference's CPU tracer would. */
int cr_scene_set_light_table(cr_scene *s, uint32_t primitive, const float *points, float pdf);

/* Same on device buffers, asynchronous on `stream`. */
int cr_trace_rays_device(cr_scene *s, const float *d_rays, uint64_t n, cr_hit *d_hits, int any_hit,
                         void *stream);

/* --------------------------------------------------------------- rendering */
/* Tracer::execute (src/core/tracer/tracer.hpp:20-21) with the Radiance
 * kernel (RadianceKernel::execute, src/core/kernel/radiance.cu:14-81) for
 * every pixel and sample, as CPUMulticoreTracer::execute
 * (src/core/tracer/cpuMulticore.cu:14-122) does on the CPU: per pixel the
 * mean of its finite samples.  film_rgb: host, window-sized W x H x 3
 * doubles (row-major, y down).  Blocks until the film is on the host. */
int cr_render(cr_scene *s, const cr_render_desc *desc, double *film_rgb, cr_stats *stats);

/* Device variant: accumulates into caller device buffers sized for the
 * window (sum and sum of squares W x H x 3 doubles, count W x H uint32),
 * asynchronous on `stream`; the library allocates its wave buffers. */
int cr_render_device(cr_scene *s, const cr_render_desc *desc, double *d_sum, double *d_sumsq,
                     uint32_t *d_count, void *stream, cr_stats *stats);

/* No counterpart in the reference.  Same render as cr_render_device, for
 * callers that cannot allocate device memory while they render (a frame
 * callback or real-time loop where cudaMalloc/cudaFree would synchronise the
 * device, or an application that budgets all device memory at start-up).
 * The call allocates nothing: the per-path wave state lives in one fixed
 * device array inside the library, held by every GPU that loads it until the
 * process exits (CR_NOALLOC_MAX_WAVE_PATHS paths, about 37 MB).  The scene
 * must already be committed; the caller passes the film buffers as for
 * cr_render_device.  desc->wave_paths above CR_NOALLOC_MAX_WAVE_PATHS, or a
 * max_bounce above CR_NOALLOC_MAX_BOUNCE, is rejected with CR_ERR_INVALID
 * (wave_paths 0 means the maximum); a guided request (desc->guiding) with
 * CR_ERR_UNSUPPORTED, before anything about the scene changes.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current;
 * make that first call before any stream capture.  Every call on a device
 * shares the one array, so calls whose work overlaps on the GPU (concurrent
 * streams, or host threads sharing a device) race and corrupt each other's
 * films; serialise them.  The call is asynchronous on `stream` and does not
 * read back the kernels' error word; stats are not collected. */
#define CR_NOALLOC_MAX_WAVE_PATHS 262144u
#define CR_NOALLOC_MAX_BOUNCE 64u
int cr_render_device_noalloc(cr_scene *s, const cr_render_desc *desc, double *d_sum, double *d_sumsq,
                             uint32_t *d_count, void *stream);

/* ----------------------------------------------------- per-bounce profile */
/* RadianceKernel::Slice (src/core/kernel/radiance.hpp:17-55) as the
 * reference's Profiler keeps it (src/core/kernel/kernel.hpp:35-81): one slice
 * per sample of the profiled pixel area, holding the sample's radiance, the
 * loop's bounce counter at exit, and for its first `depth` vertices one
 * BounceRecord each (radiance.cu:41-53): the ray that reached the vertex, the
 * shader's f for the light sample's direction, theta = the angle between wo
 * and that direction mirrored about the normal, the radiance gathered up to
 * and including the vertex, and the vertex's shader id. */
typedef struct cr_profile_bounce {
    float ray_o[3], ray_d[3];
    float f[3];
    float theta;
    float L[3];
    uint32_t shader;
} cr_profile_bounce;
typedef struct cr_profile_slice {
    uint32_t bounce;
    float L[3];
} cr_profile_slice;
/* Profiled render with the reference estimator (CPUMulticoreTracer::execute
 * with an enabled Profiler, src/core/tracer/cpuMulticore.cu:17,53-64):
 * renders the pixel window of `desc` (the profiler's area) and records its
 * slices, host arrays in the Profiler's order (row, column, sample):
 * slices ww x wh x spp, bounces ww x wh x spp x depth (depth <= 64).
 * film_rgb (window-sized, may be NULL) receives the per-pixel means.  For
 * the records to follow the reference's loop exactly, a profiled path is not
 * cut short when its throughput reaches zero. */
int cr_render_profile(cr_scene *s, const cr_render_desc *desc, uint32_t depth, cr_profile_slice *slices,
                      cr_profile_bounce *bounces, double *film_rgb);
/* Profiler::~Profiler (kernel.cu): writes the slices of the area
 * (x0, y0)-(x1, y1) of a profiled render at `spp` samples to `path` in the
 * reference's text format (an "at [ x, y, k ]: " line per sample; a slice's
 * records only when its radiance is at least 100 in every channel, as
 * RadianceKernel::Slice::writeSlice prints them). */
int cr_profile_write(const char *path, const uint32_t area[4], uint32_t spp, uint32_t depth,
                     const cr_profile_slice *slices, const cr_profile_bounce *bounces);

/* No counterpart in the reference (its tracer has no launch parameters).
 * Picks the wave size, the traversal refill threshold and the traversal grid
 * for this scene by timing a sample render (a band of the requested image,
 * at most 64 spp) under each candidate, coordinate by coordinate, with CUDA
 * events.  The choice is stored in the scene and returned in *out.
 * Synchronises `stream`; allocates temporary device buffers. */
int cr_autotune(cr_scene *s, const cr_render_desc *desc, void *stream, cr_tuning *out);

/* No counterpart in the reference.  Measures, on the current device, the
 * L2-resident read bandwidth (a 32 MB buffer read 64 times with 16-byte
 * loads) and the FP32 FMA throughput (8 independent chains per thread): the
 * rooflines of traversal when the scene fits in L2 and of its box and
 * triangle tests.  Synchronises `stream`; allocates 32 MB for the call. */
int cr_measure_peaks(void *stream, double *l2_read_gbs, double *fp32_tflops);

/* No counterpart in the reference.  Measures, on the current device, the
 * achievable rate of random whole-record gathers, the access pattern of BVH
 * traversal: records of record_bytes (80: a wide node, 48: a triangle) at
 * independent pseudo-random indices of an array of array_bytes (1 MB..1 GB;
 * below the 126 MB L2 it is L2-resident), read through the L1/texture path.
 * *gbs: gathered bytes per second / 1e9.  Synchronises `stream`; allocates
 * the array for the call. */
int cr_measure_gather(void *stream, uint32_t record_bytes, uint64_t array_bytes, double *gbs);

/* ------------------------------------------------------ batched renders */
/* No counterpart in the reference (its tracer renders one scene per call).
 * A batch renders many committed scenes, each at its own resolution and spp,
 * in shared waves: the paths of all jobs are concatenated, so one persistent
 * traversal launch per bounce serves every scene and small images do not
 * leave the GPU idle.  The first cr_batch_render builds one CUDA graph on
 * the batch's stream: an initialising kernel and a conditional WHILE node
 * whose body is one wave's kernels (generation, max_bounce + 1 x closest
 * hit, shading and shadow rays, accumulation); the wave index lives in
 * device memory and the body's last kernel ends the loop after the last
 * wave.  Later calls replay the graph.  Jobs render their whole image;
 * estimator and max_bounce are shared; learned guiding is not used in
 * batches. */
typedef struct cr_batch cr_batch;
typedef struct cr_batch_job {
    cr_scene *scene;         /* committed scene (may appear in several jobs) */
    uint32_t width, height;  /* image size */
    uint32_t spp;            /* samples per pixel per render call */
    uint64_t seed;           /* random seed of this job (plus the call's offset) */
    double *d_sum;           /* device film: width x height x 3 doubles, accumulated */
    double *d_sumsq;         /* width x height x 3 doubles */
    uint32_t *d_count;       /* width x height finite-sample counts */
} cr_batch_job;
/* stream: the stream the batch captures and replays on; NULL: a stream of
 * the batch's own.  The job table is copied; the films stay the caller's, and
 * the scenes must stay alive and unchanged while the batch exists. */
int cr_batch_create(const cr_batch_job *jobs, uint32_t n_jobs, uint32_t max_bounce, int32_t estimator,
                    void *stream, cr_batch **out);
/* Picks wave size, refill threshold and traversal grid for the batch by
 * timing a reduced batch (every job at spp / 16, at least 1) under each
 * candidate; the choice is kept (the next render captures a new graph).
 * Synchronises; allocates temporary films. */
int cr_batch_autotune(cr_batch *b, cr_tuning *out);
/* Sets the batch's launch configuration from `t` (wave_paths, refill_min,
 * traverse_blocks_per_sm, shade_threads; a zero field keeps the current
 * value), e.g. a tuning kept from an earlier run.  The next render builds a
 * new graph. */
int cr_batch_set_tuning(cr_batch *b, const cr_tuning *t);
/* One render of every job into its film, job seeds offset by seed_offset.
 * With stats NULL the call only enqueues the graph (asynchronous); with
 * stats it waits, checks the device error word and fills the totals and the
 * device time of the replay. */
int cr_batch_render(cr_batch *b, uint64_t seed_offset, cr_stats *stats);
void cr_batch_destroy(cr_batch *b);

/* ------------------------------------------------------ learned guiding */
/* No counterpart in the reference.  A committed scene owns one path guide:
 * a 12-level hash-grid + SH encoding feeding a 4 x 64 MLP whose output is a
 * mixture of 8 von Mises-Fisher lobes over incident directions.  Renders with
 * desc->guiding = 1 (MIS estimator) sample it by one-sample MIS with the BSDF
 * and train it online (Adam) on their own path vertices; it persists across
 * renders of the scene.  cr_guide_reset (re)initialises it from `seed`. */
int cr_guide_reset(cr_scene *s, uint64_t seed);
/* Normalisation box (x -> (x - bmin) * binv), training steps taken, and the
 * sizes (in floats) of the grid, weight and bias arrays. */
int cr_guide_info(const cr_scene *s, float *bmin, float *binv, uint32_t *step, uint32_t *sizes);
/* Training schedule of the scene's guide, defaults in brackets.  Each wave of
 * a guided render records the vertices of steps_per_wave x train_paths paths
 * spread over the wave and takes one Adam step per train_paths of them.
 *   lr              Adam step size [1e-2]
 *   select_prob     probability of sampling the guide at a vertex [0.5]
 *   train_paths     paths per training batch [32768: up to 2^18 vertices at
 *                   max_bounce 7]
 *   steps_per_wave  batches (Adam steps) per wave [64]: the 600-step budget is
 *                   spent in the first ten waves, then the guide is frozen
 *   warmup_steps    steps taken before the guide is first sampled [8]; until
 *                   then a guided render samples the BSDF only and trains
 *   product_target  1: fit the integrand Li f cos at each vertex; 0: fit the
 *                   incident (indirect) radiance Li alone [1]
 *   max_steps       training budget: after this many Adam steps renders sample
 *                   the guide without recording or training (0: no budget) [600]
 *   guided_bounces  vertices 0 .. guided_bounces-1 of a path sample the guide
 *                   (and only their bounces run the guide's inference); later
 *                   vertices sample the BSDF alone (0: every vertex but the
 *                   last) [0]
 *   learn_select    1: the network also learns, per vertex, the probability of
 *                   sampling the guide rather than the BSDF (a sigmoid output
 *                   clamped to [0.02, 0.98], trained on the density of the
 *                   one-sample mixture the renderer samples); select_prob is
 *                   then unused [0] */
typedef struct cr_guide_config {
    float lr;
    float select_prob;
    uint32_t train_paths;
    uint32_t steps_per_wave;
    uint32_t warmup_steps;
    uint32_t product_target;
    uint32_t max_steps;
    uint32_t guided_bounces;
    uint32_t learn_select;
} cr_guide_config;
/* Apply `in` (when not NULL) and report the schedule in `out` (when not NULL). */
int cr_guide_configure(cr_scene *s, const cr_guide_config *in, cr_guide_config *out);
/* Trains the scene's guide to its budget (max_steps; a guide with none is
 * refused) on guided MIS renders of desc's image or window into a scratch
 * film that is then discarded, so that a later guided render of the image
 * draws every sample with the trained, frozen guide.  Each pass has about
 * steps_per_wave x train_paths paths (desc->spp is replaced), one wave that is
 * recorded whole; the seeds run from desc->seed.  On `stream` (NULL: the
 * scene's); waits for the passes; *passes (when not NULL) = passes rendered. */
int cr_guide_train(cr_scene *s, const cr_render_desc *desc, void *stream, uint32_t *passes);
/* Weighted NLL (normalised by the batch weight) of the last training batch. */
int cr_guide_loss(const cr_scene *s, float *loss);
/* Copy the parameters out (set = 0) or in (set = 1); NULL arrays are skipped.
 * grid: [12][65536][2], W: [5][64 out][64 in], b: [5][64]. */
int cr_guide_params(cr_scene *s, float *grid, float *W, float *b, int set);
/* Network outputs (n x 64, FP32 path) for inputs n x {x, wo, n} (9 floats). */
int cr_guide_forward(cr_scene *s, const float *inputs, uint64_t n, float *out);
/* The same through the path the renderer samples with: BF16 weights and
 * activations on the tensor cores (tcgen05), FP32 accumulation. */
int cr_guide_forward_tc(cr_scene *s, const float *inputs, uint64_t n, float *out);
/* Gradients of the weighted mixture NLL over records n x {x, wo, n, w, weight}
 * (13 floats; 14 with learn_select, the 14th the BSDF density of w),
 * normalised by the total weight; parameters are not updated. */
int cr_guide_gradients(cr_scene *s, const float *records, uint64_t n, float *gW, float *gb, float *ggrid);
/* The same through the training pass the renderer uses: BF16 operands on the
 * tensor cores (tcgen05), FP32 accumulation. */
int cr_guide_gradients_tc(cr_scene *s, const float *records, uint64_t n, float *gW, float *gb, float *ggrid);

/* Renderer::render (src/core/renderer/renderer.cu:13-52): load a scene file,
 * render it with the configured kernel and tracer, write the reference's
 * clamped 8-bit PNG (src/util/image.cu:15-18) and, when pfm_path is not
 * NULL, a linear float PFM. */
int cr_render_file(const char *json_path, const char *png_path, const char *pfm_path, uint32_t spp,
                   uint32_t width, uint32_t height, const char *kernel, const char *tracer);

/* 8-bit PNG of linear radiance clamped to [0,1] as util::Image<3> stores it
 * (src/util/image.hpp:16-49). */
int cr_write_png(const char *path, uint32_t width, uint32_t height, const double *rgb);

/* ----------------------------------------------------- BSDF parity helpers */
/* Shader::execute(compute_f_by_wi_wo) (src/core/nodes/shader.hpp:17-23) for n
 * local-frame direction pairs, evaluated by the CUDA path's device code.
 * f: n x 3, pdf: n (0 for CR_ESTIMATOR_KOISHI, which has no pdf). */
int cr_bsdf_eval(int estimator, const char *shader_json, const float *wo, const float *wi, uint64_t n,
                 float *f, float *pdf);
/* Shader::execute(sample_wi_f_by_wo) for n outgoing directions and uniforms
 * u (n x 2): wi (n x 3), weight = f*|cos|/pdf (n x 3), pdf (n). */
int cr_bsdf_sample(int estimator, const char *shader_json, const float *wo, const float *u, uint64_t n,
                   float *wi, float *weight, float *pdf);
/* The two helpers above take single-node shaders without selection draws
 * (not Mixed, not GlassBSDF); cr_shader_execute takes any shader. */

/* Shader::execute(varyings, sampler, pool, target) (src/core/nodes/shader.hpp:17-23)
 * with the reference estimator's shaders, nested Mixed included, for n
 * samples in the local shading frame (z = normal), run by the CUDA path's
 * device code:
 *   CR_SHADE_EVAL   compute_f_by_wi_wo: f for (wo, wi)
 *   CR_SHADE_SAMPLE sample_wi_f_by_wo:  wi and f for wo; wi is in/out and
 *                   keeps its input where the shader leaves it unchanged
 *                   (a refraction past the critical angle)
 * u holds k uniforms per sample (k <= 64), handed out in the order the
 * reference's Sampler would serve them (sample3 draws three); used[i] is how
 * many sample i drew (draws past k read 0.5).  emission (n x 3) is what the
 * executed shader writes to varyings.emission (non-zero for Emission only).
 * Replaces direct calls of the poly::object<Shader> in scene.shaders. */
#define CR_SHADE_EVAL 0
#define CR_SHADE_SAMPLE 1
int cr_shader_execute(const char *shader_json, int target, const float *wo, float *wi, const float *u, uint32_t k,
                      uint64_t n, float *f, float *emission, uint32_t *used);

/* --------------------------------------------------- random number parity */
/* No counterpart in the reference: its Sampler is a 48-bit linear
 * congruential generator (src/core/misc/sampler.hpp:22-36), which the CUDA
 * path replaces with counter-based Philox4x32-10 (Salmon et al., SC'11).
 * Runs the render's own device generator on n (counter, key) pairs, host
 * arrays: ctr_key n x 6 words (c0, c1, c2, c3, k0, k1), out n x 4 words.
 * For known-answer tests of the generator. */
int cr_philox4x32_10(const uint32_t *ctr_key, uint64_t n, uint32_t *out);

#ifdef __cplusplus
}
#endif
#endif /* CR_H */
