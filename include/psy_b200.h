/*
 * psy_b200.h - C ABI of the B200 (sm_100a) implementation of the
 * breadth-first path-tracing hot path of the Psychopath renderer.
 *
 * Plain C types only: host pointers, device pointers (as void* / typed
 * pointers into GPU memory), sizes and an opaque cudaStream_t passed as
 * void*.  Every entry point returns an int status: PSY_OK (0) or a negative
 * PSY_ERR_* code; psy_last_error() returns the message of the last failure
 * on a context.  No exceptions cross this boundary.
 *
 * A context is used by one host thread at a time (like the reference's
 * Tracer, one per thread: integrator/path_trace_integrator.cpp:286).
 *
 * Reference interfaces replaced (paths within the reference project):
 *   psy_scene_upload   Assembly::finalize -> BVH4::build + LightTree::build
 *                      (scene/assembly.hpp:206-238, accel/bvh4.cpp:17,
 *                      accel/light_tree.cpp:99)
 *   psy_trace          Tracer::trace (tracer/tracer.hpp:76, tracer/tracer.cpp:38-121)
 *   psy_trace_host     Tracer::trace with host arrays (same seam, e2e form)
 *   psy_light_sample   LightAccel::sample / LightTree::sample
 *                      (accel/light_accel.hpp:55, accel/light_tree.cpp:30-96)
 *   psy_render         PathTraceIntegrator::integrate
 *                      (integrator/integrator.hpp:32, integrator/path_trace_integrator.cpp:28-384)
 */
#ifndef PSY_B200_H
#define PSY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Status codes                                                         */
/* ------------------------------------------------------------------ */
#define PSY_OK 0
#define PSY_ERR_ARG (-1)            /* invalid argument / malformed scene */
#define PSY_ERR_OOM (-2)            /* device or host allocation failed */
#define PSY_ERR_DEVICE (-3)         /* CUDA runtime error */
#define PSY_ERR_TIMEOUT (-4)        /* a bounded device wait gave up */
#define PSY_ERR_STACK_OVERFLOW (-5) /* a per-ray traversal stack overflowed */
#define PSY_ERR_NAN (-6)            /* non-finite input rejected */
#define PSY_ERR_NO_SCENE (-7)       /* call needs a scene; none uploaded */

typedef struct psy_ctx psy_ctx;

/* Creates a context on CUDA device `device`. */
int psy_ctx_create(int device, psy_ctx** out);
void psy_ctx_destroy(psy_ctx* ctx);
/* Message of the last failing call on ctx (never NULL). */
const char* psy_last_error(const psy_ctx* ctx);
/* Library version string. */
const char* psy_version(void);

/* ------------------------------------------------------------------ */
/* Scene description (host memory, flattened assembly tree)             */
/* ------------------------------------------------------------------ */
/*
 * The flattened form of the reference's Scene / Assembly / Instance /
 * Object / SurfaceShader graph (scene/scene.hpp:33-53,
 * scene/assembly.hpp:26-330).  Matrices are 16 floats, row-major, in the
 * reference's row-vector convention (v' = v * M; math/matrix.hpp:99-115).
 * Instance transforms map the parent space into the instance's space; the
 * camera transforms map camera space to world space.
 */
enum {
	PSY_OBJ_SPHERE = 0,       /* data: n0 time samples of (cx cy cz r)            */
	PSY_OBJ_BILINEAR = 1,     /* data: n0 time samples of 4 verts (12 floats)     */
	PSY_OBJ_BICUBIC = 2,      /* data: n0 time samples of 16 verts (48 floats)    */
	PSY_OBJ_SPHERE_LIGHT = 3, /* data: n0 positions (3), n1 radii, n2 colours (3) */
	PSY_OBJ_RECT_LIGHT = 4    /* data: n0 dimensions (x y), n1 colours (3); in its xy plane at the origin
	                             (RectangleLight, lights/rectangle_light.hpp) */
};

enum { PSY_INSTANCE_OBJECT = 0, PSY_INSTANCE_ASSEMBLY = 1 };

enum { PSY_SHADER_LAMBERT = 0, PSY_SHADER_EMIT = 1, PSY_SHADER_GTR = 2 };

typedef struct psy_object_desc {
	uint32_t kind;         /* PSY_OBJ_* */
	uint32_t n0, n1, n2;   /* time-sample counts (see PSY_OBJ_*) */
	const float* data;     /* object data, layout per kind */
} psy_object_desc;

typedef struct psy_instance_desc {
	uint32_t kind;             /* PSY_INSTANCE_* */
	uint32_t data_index;       /* object index in the assembly, or the slot in the assembly's `children` */
	uint32_t transform_index;  /* first transform in the assembly's transform list */
	uint32_t transform_count;  /* motion samples; 0 = no transform */
	int32_t shader;            /* scene shader index, -1 = none (inherit) */
} psy_instance_desc;

typedef struct psy_assembly_desc {
	uint32_t object_count;
	const psy_object_desc* objects;
	uint32_t instance_count;
	const psy_instance_desc* instances;
	uint32_t transform_count;
	const float* transforms;    /* transform_count * 16 */
	uint32_t child_count;
	const uint32_t* children;   /* scene assembly indices of the sub-assemblies */
} psy_assembly_desc;

typedef struct psy_shader_desc {
	uint32_t kind;       /* PSY_SHADER_* */
	float color[3];      /* RGB */
	float roughness, tail_shape, fresnel;  /* GTR only */
} psy_shader_desc;

typedef struct psy_scene_desc {
	uint32_t cam_transform_count;
	const float* cam_transforms;       /* camera-to-world, count * 16 */
	uint32_t cam_fov_count;
	const float* cam_fovs;             /* radians (reference parser/parser.cpp:218 conversion applied) */
	uint32_t cam_aperture_count;
	const float* cam_aperture_radii;
	uint32_t cam_focus_count;
	const float* cam_focus_distances;
	float background[3];               /* RGB */
	float dice_rate;                   /* Config::dice_rate (config.cpp:7), 0.25 default */
	float min_upoly_size;              /* Config::min_upoly_size (config.cpp:8), 1e-5 default */
	uint32_t assembly_count;           /* [0] is the root assembly */
	const psy_assembly_desc* assemblies;
	uint32_t shader_count;
	const psy_shader_desc* shaders;
} psy_scene_desc;

/*
 * Builds the acceleration structures on the host as Assembly::finalize does
 * (BVH with a midpoint split, packed to BVH4, which gives each assembly its
 * bounds; light tree) and uploads the device scene.  The device walks a
 * BVH4 of the same form built with surface-area splits: the hits are the
 * same (exact ties aside), with fewer nodes visited.  Replaces any previous
 * scene.
 */
int psy_scene_upload(psy_ctx* ctx, const psy_scene_desc* scene);

/*
 * psy_scene_upload with options (no counterpart in the reference, whose
 * builds run on the host at Assembly::finalize).  PSY_UPLOAD_GPU_BVH: the
 * root assembly's traversal BVH4 is built on the device (moving instances
 * included): the host's binned surface-area tree split for split, packed
 * four-wide as BVH4::build packs (accel/bvh4.cpp:17-159, time samples
 * included), so traces and renders are those of psy_scene_upload bit for
 * bit.  The root's
 * light tree is built on the device too, when it has two or more lights
 * (moving bounds included): LightTree::build's own tree node for node
 * (accel/light_tree.cpp:99-238, libstdc++'s partition order included), so
 * light selection is unchanged.  The nested assemblies' trees are built on
 * the host either way.
 */
#define PSY_UPLOAD_GPU_BVH 1u
int psy_scene_upload_ex(psy_ctx* ctx, const psy_scene_desc* scene, uint32_t flags);

/* Summary of the uploaded scene (for tests and tooling).  gpu_bvh4_nodes and
 * gpu_light_nodes count the nodes of bvh4_nodes and light_nodes that the
 * device built (PSY_UPLOAD_GPU_BVH), 0 when the host built them all. */
typedef struct psy_scene_stats {
	uint32_t assemblies, instances, objects, bvh4_nodes, light_nodes, lights;
	uint64_t device_bytes;
	uint32_t gpu_bvh4_nodes, gpu_light_nodes;
} psy_scene_stats;
int psy_scene_stats_get(const psy_ctx* ctx, psy_scene_stats* out);

/*
 * Host-only inspection of the scene builder (no device needed): builds the
 * scene description exactly as psy_scene_upload does and copies one
 * assembly's BVH4 in the reference's node-record form (one record per node
 * time sample, BVH4::Node in accel/bvh4.hpp:39-71): bounds[n*24] as BBox4
 * SoA, child[n*3] (children 2-4, 0 = none / leaf marker), ts[n],
 * data_index[n] (leaf instance).  Pass NULL arrays to get *count only.
 */
int psy_build_bvh4(const psy_scene_desc* scene, uint32_t assembly, uint64_t* count, float* bounds, uint64_t* child,
                   uint32_t* ts, uint64_t* data_index);

/*
 * Host-only: one assembly's light tree (LightTree nodes,
 * accel/light_tree.hpp:15-24).  meta[n*6] = is_leaf, index1, index2,
 * instance_index, bounds count, first bounds record; energy[n];
 * bounds[*nbounds*6] = min xyz, max xyz per time sample.  Indices are local
 * to the assembly's tree.  Also returns the tree's light count and total
 * energy.  Pass NULL arrays to get the counts only.
 */
int psy_build_light_tree(const psy_scene_desc* scene, uint32_t assembly, uint64_t* count, uint64_t* nbounds,
                         uint64_t* meta, float* energy, float* bounds, uint64_t* light_count, float* total_energy);

/*
 * Host-only: a .psy scene file read into a scene description, replacing the
 * reference's Parser::parse_next_frame (parser/data_tree.cpp:177-400,
 * parser/parser.cpp:37-662): the frame-th Scene node's render settings,
 * camera, background colour and root assembly (shaders, spheres, bilinear
 * and bicubic patches, sphere and rectangle lights, nested assemblies,
 * instances with motion transforms and shader bindings).  Numbers are read
 * as the reference reads them (std::stof of each -?[0-9]+[.]?[0-9]* match).
 * psy_file_parse returns PSY_ERR_ARG for a malformed file, with the reason
 * in err (err_len bytes, NULL for none), and PSY_ERR_NO_SCENE when the file
 * has no Scene node `frame` (frames count from 0: where parse_next_frame
 * returns null); the description stays valid until psy_file_free.
 */
typedef struct psy_file_scene psy_file_scene;
typedef struct psy_render_settings {
	uint32_t width, height, spp, seed;  /* RenderSettings: Resolution, SamplesPerPixel, Seed (default 1 each) */
	const char* output_path;            /* Output: Path ("" when none), owned by the psy_file_scene */
} psy_render_settings;
int psy_file_parse(const char* text, size_t len, uint32_t frame, psy_file_scene** out, char* err, size_t err_len);
const psy_scene_desc* psy_file_scene_desc(const psy_file_scene* scene);
int psy_file_render_settings(const psy_file_scene* scene, psy_render_settings* out);
void psy_file_free(psy_file_scene* scene);

/* ------------------------------------------------------------------ */
/* Ray stream tracing                                                   */
/* ------------------------------------------------------------------ */
/*
 * World rays, structure of arrays (WorldRay, basics/ray.hpp:162-186).
 * All pointers are device pointers with n elements (vec3 fields n*3).
 */
enum { PSY_RAY_CAMERA = 1, PSY_RAY_DIFFUSE = 2, PSY_RAY_OCCLUSION = 32 };

typedef struct psy_ray_soa {
	const float* o;       /* n*3 */
	const float* d;       /* n*3 */
	const float* odx;     /* n*3 origin differentials */
	const float* ody;     /* n*3 */
	const float* ddx;     /* n*3 direction differentials */
	const float* ddy;     /* n*3 */
	const float* time;    /* n */
	const uint16_t* type; /* n, WorldRay::Type values; NULL = all closest-hit */
} psy_ray_soa;

/*
 * Intersections, structure of arrays (Intersection, basics/intersection.hpp:22-49).
 * Any pointer may be NULL to skip that field.  Geometry is in the hit
 * object's space, as the reference stores it; `space` is the 4x4 transform
 * from world space into that space at the ray's time (identity when none).
 * closure: 0 none, 1 Lambert, 2 Emit, 3 GTR, with its RGB colour.
 * For occlusion rays only `hit` (and `id`) are meaningful.
 */
typedef struct psy_hit_soa {
	uint8_t* hit;         /* n */
	uint64_t* id;         /* n, InstanceID bits (basics/instance_id.hpp) */
	float* t;             /* n */
	float* uv;            /* n*2 */
	float* p;             /* n*3 */
	float* n;             /* n*3 */
	float* dpdu;          /* n*3 */
	float* dpdv;          /* n*3 */
	float* dndu;          /* n*3 */
	float* dndv;          /* n*3 */
	uint8_t* backfacing;  /* n */
	float* light_pdf;     /* n */
	float* offset;        /* n*3 */
	float* space;         /* n*16 */
	uint8_t* closure;     /* n */
	float* closure_color; /* n*3 */
} psy_hit_soa;

/*
 * Traces n rays (device SoA) and writes their intersections (device SoA)
 * on `stream` (a cudaStream_t, NULL = default stream).  Asynchronous;
 * errors from the kernel's own checks are reported by the next call that
 * synchronises (psy_sync).
 */
int psy_trace(psy_ctx* ctx, const psy_ray_soa* rays, uint32_t n, const psy_hit_soa* hits, void* stream);

/*
 * The same with host arrays: copies the rays to the device, traces, copies
 * the requested hit fields back, and synchronises.  Field layout as above,
 * host pointers.
 */
int psy_trace_host(psy_ctx* ctx, const psy_ray_soa* rays, uint32_t n, const psy_hit_soa* hits);

/*
 * psy_trace_host without any allocation.  This entry point has no
 * counterpart in the reference; it exists for callers that cannot let a
 * trace call allocate device memory (a renderer whose pool allocator already
 * holds all free device memory, or one whose other streams must not be
 * stalled by the device-wide synchronisation cudaMalloc / cudaFree can
 * cause).  The rays and hits are staged in one fixed-size device array
 * compiled into the library (about 17 MB per device) instead of the
 * context's growable scratch buffers.  Same arguments and results as
 * psy_trace_host, on `stream` (NULL = default stream), synchronised before
 * return.
 *  - n > PSY_NOALLOC_MAX_RAYS fails with PSY_ERR_ARG before any device work.
 *  - The array is one per device, shared by all contexts: calls that overlap
 *    in time on one device race on it; serialise them.
 *  - The array is made resident on a device (its module loaded, its address
 *    resolved) by psy_ctx_create on that device, or by a call with n == 0,
 *    which does only that.  Create the context, or make that call, before a
 *    pool allocator takes the device's free memory and before any stream
 *    capture begins on that device.
 *  - No device or pinned memory is allocated; only a failing call may grow
 *    the context's error message string.
 */
#define PSY_NOALLOC_MAX_RAYS 65536u
int psy_trace_host_noalloc(psy_ctx* ctx, const psy_ray_soa* rays, uint32_t n, const psy_hit_soa* hits,
                           void* stream);

/* Waits for the context's work on `stream` and reports device-side errors. */
int psy_sync(psy_ctx* ctx, void* stream);

/* ------------------------------------------------------------------ */
/* Light sampling                                                       */
/* ------------------------------------------------------------------ */
/*
 * Batched LightTree::sample queries (LightQuery, accel/light_accel.hpp:23-42)
 * against the root assembly, with a Lambert BSDF for the tree's estimate.
 * Inputs (device, n or n*3): n u v, pos, nor, d, wavelength, time.
 * Outputs (device): to_light n*3, spec n*4 (spectral sample energies),
 * selection_pdf n, light_pdf n, id n (may be NULL).
 */
typedef struct psy_light_query_soa {
	const float* n;
	const float* u;
	const float* v;
	const float* pos;
	const float* nor;
	const float* d;
	const float* wavelength;
	const float* time;
} psy_light_query_soa;

typedef struct psy_light_sample_soa {
	float* to_light;
	float* spec;
	float* selection_pdf;
	float* light_pdf;
	uint64_t* id;
} psy_light_sample_soa;

int psy_light_sample(psy_ctx* ctx, const psy_light_query_soa* q, uint32_t n, const psy_light_sample_soa* out,
                     void* stream);

/* ------------------------------------------------------------------ */
/* Rendering                                                            */
/* ------------------------------------------------------------------ */
typedef struct psy_render_desc {
	uint32_t width, height;   /* image resolution */
	uint32_t spp;             /* samples per pixel */
	uint32_t seed;            /* sampler seed (RenderSettings Seed) */
	uint32_t path_length;     /* max path segments (PathTraceIntegrator::path_length, default 4) */
	uint32_t stream_paths;    /* paths in flight per wave, 0 = automatic */
	uint32_t block_size;      /* threads per block for the wavefront kernels, 0 = automatic */
} psy_render_desc;

typedef struct psy_render_stats {
	uint64_t paths;           /* width*height*spp */
	uint64_t rays;            /* rays traced (Global::Stats::rays_shot equivalent) */
	uint32_t launches;        /* kernels launched */
	uint32_t waves;
	uint64_t occlusion_rays;  /* of rays, the shadow (occlusion) rays */
} psy_render_stats;

/*
 * Renders the uploaded scene.  xyz (device, width*height*3) receives the
 * per-pixel XYZ sums of the samples, each scaled by XYZ_NORM_FAC exactly as
 * Film::add_sample receives them (path_trace_integrator.cpp:357-359);
 * counts (device, width*height, may be NULL) the accepted sample counts.
 * Both are accumulated into (not cleared).  Stream-ordered on `stream`.
 */
int psy_render(psy_ctx* ctx, const psy_render_desc* desc, float* xyz, uint32_t* counts, psy_render_stats* stats,
               void* stream);

/*
 * Film output (Film::scanline_image_8bbc, film/film.hpp:173-225): the film
 * psy_render accumulates (device xyz sums, width*height*3, and counts,
 * width*height) to 8-bit sRGB scanlines (device rgb, width*height*3):
 * mean XYZ -> whitepoint-E sRGB, clamped, sRGB curve, x255, dither,
 * clamp, truncate; pixels without samples show the reference's grey
 * checkerboard.  The reference dithers with a clock-seeded RNG; here the
 * dither is a hash of (seed, pixel, channel) in [-0.5, 0.5) when `dithered`
 * is non-zero, else none.  Stream-ordered on `stream`.
 */
int psy_film_srgb8(psy_ctx* ctx, const float* xyz, const uint32_t* counts, uint32_t width, uint32_t height,
                   int dithered, uint32_t seed, uint8_t* rgb, void* stream);

/*
 * Self-check of the device float math (no counterpart in the reference).
 * The shading kernels evaluate sin, cos, acos, asin and exp of floats with
 * restatements of the host C library's sincosf, acosf, asinf and expf, so
 * their bits follow the reference's std::sin/cos/acos/asin/exp calls.
 * psy_math_check evaluates function `fn` on the device for the n host
 * floats x into the n host floats out (synchronous).
 */
#define PSY_MATH_SIN 0u
#define PSY_MATH_COS 1u
#define PSY_MATH_ACOS 2u
#define PSY_MATH_ASIN 3u
#define PSY_MATH_EXP 4u
int psy_math_check(psy_ctx* ctx, uint32_t fn, uint32_t n, const float* x, float* out);

/*
 * Optional timing of the traversal kernels, for roofline reports (no
 * counterpart in the reference).  While enabled, psy_render records CUDA
 * events on its stream around every traversal launch (the event pool starts
 * at PSY_PROFILE_MAX_LAUNCHES launches and grows as needed);
 * psy_profile_read waits for them and returns their summed time and count,
 * then starts a new count.
 */
#define PSY_PROFILE_MAX_LAUNCHES 4096
int psy_profile_enable(psy_ctx* ctx, int on);
int psy_profile_read(psy_ctx* ctx, double* trace_ms, uint32_t* launches);

/*
 * Work counters of the traversal kernels over the last psy_render,
 * psy_render_diff or psy_render_adjoint call on ctx, for closest-hit and
 * occlusion rays (no counterpart in the reference; always collected).
 * Synchronises the device.  Either pointer may be NULL.
 */
typedef struct psy_trace_counters {
	uint64_t rays;              /* rays traced */
	uint64_t node_visits;       /* BVH4 inner nodes visited */
	uint64_t leaf_visits;       /* leaves visited: assembly instance entries and object tests */
	uint64_t patch_iterations;  /* patch bisection iterations (a leaf test or a split each) */
	uint64_t warp_steps;        /* traversal warp-loop iterations that ran work */
	uint64_t lane_steps;        /* lanes that ran work, summed over those iterations (of 32 each) */
} psy_trace_counters;
int psy_profile_counters(psy_ctx* ctx, psy_trace_counters* closest, psy_trace_counters* occlusion);

/* ------------------------------------------------------------------ */
/* Differentiable rendering: parameters and the path-replay adjoint     */
/* ------------------------------------------------------------------ */
/*
 * No counterpart in the reference, whose shading reads fixed RGB colours.
 * A parameter vector (device memory) replaces chosen colours:
 *  - a Lambert shader with shader_param[s] = p >= 0 takes its albedo
 *    spectrum from four Gaussian basis weights params[p..p+3]:
 *      a(lambda) = sum_k params[p+k] * exp(-(lambda - c_k)^2 / (2 s^2)),
 *    c_k = PSY_ALBEDO_BASIS_C0 + k * PSY_ALBEDO_BASIS_STEP nm, s = PSY_ALBEDO_BASIS_SIGMA nm
 *    (the RGB colour's upsampled spectrum is used where shader_param is -1);
 *  - a Lambert shader with shader_scale_param[s] = q >= 0 keeps its RGB
 *    colour's upsampled spectrum, scaled by params[q] (the reference's
 *    spectral upsampling is linear in the colour's magnitude, so this is the
 *    reference's albedo with the colour scaled by params[q]); a shader takes
 *    basis weights or a scale, not both;
 *  - a sphere light with object_param[o] = q >= 0 has its emission scaled
 *    by params[q].  Light selection keeps the uploaded energies, so the
 *    estimator stays unbiased for any scale.
 * With every entry -1 the render is the reference's.  Objects are numbered
 * assembly by assembly in psy_scene_desc order, shaders as in the scene.
 */
#define PSY_ALBEDO_BASIS_C0 430.0f
#define PSY_ALBEDO_BASIS_STEP 80.0f
#define PSY_ALBEDO_BASIS_SIGMA 45.0f

typedef struct psy_diff_desc {
	uint32_t param_count;             /* length of params (and of the gradient) */
	const float* params;              /* device, param_count floats */
	uint32_t shader_count;            /* entries of shader_param: the scene's shader count */
	const int32_t* shader_param;      /* host: first albedo weight of each shader, or -1 */
	uint32_t object_count;            /* entries of object_param: the scene's object count */
	const int32_t* object_param;      /* host: emission scale of each light object, or -1 */
	uint32_t shader_scale_count;      /* entries of shader_scale_param: 0 (none) or the scene's shader count */
	const int32_t* shader_scale_param;/* host: the scale of each shader's RGB albedo, or -1 */
} psy_diff_desc;

/* psy_render with the parameterised colours (same film semantics). */
int psy_render_diff(psy_ctx* ctx, const psy_render_desc* desc, const psy_diff_desc* diff, float* xyz,
                    uint32_t* counts, psy_render_stats* stats, void* stream);

/*
 * Path-replay adjoint of psy_render_diff: replays every path from its
 * sampler seed (nothing is stored per vertex between the passes) and adds
 * to grad (device, param_count floats) the gradient of a loss whose
 * derivative with respect to the film sums is dl_dxyz (device,
 * width*height*3 floats; the film sums are what psy_render_diff accumulates).
 * The estimator is differentiated exactly: sampling decisions do not depend
 * on the parameters.  Samples the film would reject (non-finite) are not
 * excluded.  path_length must be at most PSY_ADJOINT_MAX_PATH.
 */
#define PSY_ADJOINT_MAX_PATH 8
int psy_render_adjoint(psy_ctx* ctx, const psy_render_desc* desc, const psy_diff_desc* diff, const float* dl_dxyz,
                       float* grad, psy_render_stats* stats, void* stream);

/* ------------------------------------------------------------------ */
/* Batched rendering                                                    */
/* ------------------------------------------------------------------ */
/*
 * Many renders of different scenes in one stream of waves: the renders'
 * paths are laid end to end and every wave takes the next paths of as many
 * renders as fit, so small renders share the GPU instead of running one
 * after another.  Each render's film gets exactly the samples psy_render
 * would give it (same sampler sequence, same per-pixel order).
 */
typedef struct psy_batch_desc {
	uint32_t count;                   /* renders */
	psy_ctx* const* scenes;           /* per render: a context holding its uploaded scene, on ctx's device */
	const psy_render_desc* renders;   /* per render: width, height, spp, seed, path_length */
	float* const* xyz;                /* per render: device film, width*height*3 floats, accumulated */
	uint32_t* const* counts;          /* per render: device sample counts, or NULL; the array may be NULL */
	uint32_t stream_paths;            /* paths per wave; 0 = the context's tuned value, else 2^21 */
	uint32_t block_size;              /* 64, 128 or 256 threads per block; 0 = tuned value, else 128 */
	uint32_t use_graph;               /* 1: launch through a CUDA graph captured once and reused while
	                                     the batch's launch parameters stay the same */
} psy_batch_desc;

/* Renders the batch on ctx's device (ctx owns the wave buffers and the
 * graph; it may be one of the scene contexts).  Stream-ordered on `stream`;
 * stats, when given, synchronises and reports the whole batch.  There is no
 * single reference seam: it replaces running PathTraceIntegrator::integrate
 * once per scene. */
int psy_render_batch(psy_ctx* ctx, const psy_batch_desc* batch, psy_render_stats* stats, void* stream);

typedef struct psy_batch_tuning {
	uint32_t stream_paths;            /* chosen paths per wave */
	uint32_t block_size;              /* chosen threads per block */
	float ms;                         /* time of the chosen configuration on the tuning batch */
	uint32_t trials;                  /* configurations timed */
} psy_batch_tuning;

/* Autotuner: times the batch with every sample count divided by
 * spp_divisor (at least 1; scratch films, the batch's films are not
 * touched) for waves of 2^14..2^22 paths and blocks of 64, 128 and 256
 * threads, keeps the fastest in ctx for psy_render_batch calls whose
 * configuration fields are 0, and returns it.  Synchronous. */
int psy_batch_autotune(psy_ctx* ctx, const psy_batch_desc* batch, uint32_t spp_divisor, psy_batch_tuning* out);

#ifdef __cplusplus
}
#endif

#endif /* PSY_B200_H */
