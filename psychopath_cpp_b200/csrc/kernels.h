/*
 * Internal interface between the C ABI layer and the CUDA kernels.
 */
#ifndef PSY_KERNELS_H
#define PSY_KERNELS_H

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/psy_b200.h"
#include "psy_scene.h"

namespace psy {

struct RaySoA {
	const float *o, *d, *odx, *ody, *ddx, *ddy, *time;
	const uint16_t* type;
};

struct HitSoA {
	uint8_t* hit;
	uint64_t* id;
	float *t, *uv, *p, *n, *dpdu, *dpdv, *dndu, *dndv;
	uint8_t* backfacing;
	float* light_pdf;
	float* offset;
	float* space;
	uint8_t* closure;
	float* closure_color;
	int want_geometry;  // any geometry field requested
};

struct HaltonDev {
	const uint16_t* perm;
	const uint4* dims;     // base, pow_base, groups, perm_offset
	const double* cmul;
};

// Parameters of one render (PathTraceIntegrator's settings and its film).
struct RenderParams {
	uint32_t width, height, spp, seed, path_length;
	uint32_t light_count;    // root LightTree::light_count()
	float min_x, max_x, min_y, max_y;  // film extent (renderer/renderer.cpp:52-55)
	float ident_inv;         // diagonal of the reference's inverse of the identity
	uint64_t path_base;      // first global path index of the render (0 unless batched)
	uint64_t pixel_base;     // first global pixel index of the render (0 unless batched)
	float* xyz;              // film XYZ sums, width * height * 3
	uint32_t* counts;        // film sample counts (may be null)
	// differentiable rendering (all null in plain renders)
	const float* params;     // parameter vector
	const int* shader_param; // per scene shader: first of its 4 albedo weights (>= 0), -2 - q for an RGB
	                         // albedo scaled by params[q], or -1
	const int* object_param; // per scene object: its emission scale, or -1
	const float* dl_dxyz;    // adjoint: dL / d(film sums), width * height * 3
	float* grad;             // adjoint: gradient accumulator, param_count floats
	int param_count;
	int grad_in_smem;        // adjoint: accumulate per block in shared memory first
};

// Largest path_length of the adjoint (vertex records per path).
#define PSY_ADJ_MAX_VERTS 8

// The global paths one wave covers: whole pixels, in order.
struct WaveRange {
	uint64_t base;           // first global path index
	uint64_t pix_base;       // first global pixel index
	int paths;
	int pixels;
};

// Path state of one wave, structure of arrays (PTState,
// integrator/path_trace_integrator.hpp:49-63).
struct PathSoA {
	uint32_t* smp;      // sampler offset
	uint32_t* dimstep;  // next sampler dimension | step << 16
	float* wl;
	float* time;
	float* last_pdf;
	float4* col;
	float4* fcol;
	float4* lcol;       // between the shadow ray and its result: the light's contribution
	float* hit;         // stored intersection, 16 floats per path
	float* pray;        // previous ray, 16 floats per path
	float* hitx;        // GTR hits: world dpdu, dpdv, dndu, dndv, 12 floats per path
	float* sample;      // film sample XYZ, 3 floats per path
	uint16_t* rid;      // render of the path (batches)
	// adjoint pass only
	float4* adj;        // dL / d(sample spectrum) per hero wavelength
	float4* valb;       // albedo spectrum of each parameterised vertex, PSY_ADJ_MAX_VERTS per path
	int* vpid;          // its first albedo weight (-1: not parameterised), PSY_ADJ_MAX_VERTS per path
	int* nee_param;     // emission scale of the light sampled at the current vertex, or -1
	float4* vdsc;       // d(albedo)/d(scale) of each scale-parameterised vertex, PSY_ADJ_MAX_VERTS per path
	float4* fexcl;      // fcol with every parameterised albedo factor left out
	float4* nee_base;   // the pending light contribution with its parameterised factors left out
};

// Rays and hits of a wave by queue position (cap = the wave's path capacity).
struct WaveBufs {
	float4* ray[2];     // [0] camera / bounce rays, [1] shadow rays: 5 planes of cap float4
	float4* hit_f;      // t, u, v, max_dim
	int4* hit_i;        // 3 planes: obj, kind | depth << 8, shader, path[0]; path[1..4]; path[5..7]
	uint8_t* occl;      // shadow ray result: 1 = blocked (or no shadow ray)
	int cap;
};

// Traversal counters of a render, one block of TC_COUNT per ray kind
// (closest-hit rays first, then occlusion rays), summed over its launches.
enum : int {
	TC_RAYS = 0,        // rays traced
	TC_NODES = 1,       // BVH4 inner nodes visited
	TC_LEAVES = 2,      // leaves visited (assembly instance entries and object tests)
	TC_PATCH_ITERS = 3, // patch bisection loop iterations (leaf tests and splits)
	TC_WARP_STEPS = 4,  // traversal warp-loop iterations that ran work
	TC_LANE_STEPS = 5,  // lanes that ran work, summed over those iterations
	TC_COUNT = 8
};

struct WaveQueues {
	int* q0;
	int* q1;
	int* counters;      // render_counter_count(path_length) work and live counters
	unsigned long long* rays;   // 2 * TC_COUNT traversal counters: closest-hit rays, then occlusion rays
};

// Optional profiling: CUDA events recorded around each traversal launch, in
// pairs, on the launch stream (events[2 k], events[2 k + 1] for the k-th).
struct LaunchTimer {
	cudaEvent_t* events;
	int capacity;  // pairs
	int* used;     // pairs recorded so far
};

struct LightQuerySoADev {
	const float *n, *u, *v, *pos, *nor, *d, *wavelength, *time;
};
struct LightSampleSoADev {
	float *to_light, *spec, *selection_pdf, *light_pdf;
	uint64_t* id;
};

int render_counter_count(uint32_t path_length);

// One wave of a single render: scene and parameters go in kernel parameters.
cudaError_t launch_render_wave(const DevScene& sc, const HaltonDev& hd, const RenderParams& rp, const WaveRange& wr,
                               const PathSoA& ps, const WaveBufs& wb, const WaveQueues& wq, unsigned* status,
                               int block, cudaStream_t st, uint32_t* launches, const LaunchTimer* timer = nullptr);

// One wave of a batch: the render of each path is found in device arrays
// (scenes and renders, count entries each); features is the union of the
// scenes' FEAT_* bits and max_path_length the largest path_length.
cudaError_t launch_batch_wave(const DevScene* scenes, const RenderParams* renders, int count, unsigned features,
                              uint32_t max_path_length, const HaltonDev& hd, const WaveRange& wr, const PathSoA& ps,
                              const WaveBufs& wb, const WaveQueues& wq, unsigned* status, int block,
                              cudaStream_t st, uint32_t* launches);

cudaError_t launch_light_sample(const DevScene& sc, const LightQuerySoADev& q, const LightSampleSoADev& o, uint32_t n,
                                float ident_inv, unsigned* status, cudaStream_t st);

cudaError_t launch_trace(const DevScene& sc, const RaySoA& rays, const HitSoA& hits, uint32_t n, unsigned* status,
                         cudaStream_t stream);

// Device build of a BVH4 over n leaves (leaf k is local instance k): host
// arrays of every instance's time-sample boxes (6 floats each: lo xyz, hi
// xyz; instance i's are samples [h_first[i], h_first[i + 1])) and box
// centres at time 0.5 (3 floats each).  The nodes go to d_nodes[0..] (room
// for n - 1), numbered from node_base in their child references; their
// time samples after the first to d_extra (24 floats each, room for
// (n - 1) * (most samples - 1)), numbered from extra_base.  *root_ref,
// *node_count and *extra_count describe the result.  Synchronous on `st`
// (bvh_gpu.cu).
cudaError_t build_bvh4_gpu(const float* h_samples, const int* h_first, const float* h_centres, int n,
                           int node_base, DevNode* d_nodes, float* d_extra, int extra_base, int* root_ref,
                           int* node_count, int* extra_count, cudaStream_t st);

// Device build of a light tree over n lights (host arrays, see
// BuiltScene::gpu_light_elems / gpu_light_samples / gpu_light_first) into
// d_nodes[0 .. 2n - 2], numbered from node_base in their child references;
// the nodes' bounds samples after the first go to d_extra (6 floats each,
// room for (2n - 1) * (most samples - 1)), numbered from extra_base.
// *root_energy and *extra_count receive the root's energy and the records
// written.  Synchronous on `st` (light_gpu.cu).
cudaError_t build_light_tree_gpu(const float* h_elems, const float* h_samples, const int* h_first, int n,
                                 int node_base, DevLightNode* d_nodes, float* d_extra, int extra_base,
                                 float* root_energy, int* extra_count, cudaStream_t st);

}  // namespace psy

#endif
