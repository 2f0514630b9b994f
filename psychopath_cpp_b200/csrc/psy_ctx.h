/*
 * The context object behind the opaque psy_ctx handle.
 */
#ifndef PSY_CTX_H
#define PSY_CTX_H

#include <map>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "kernels.h"
#include "psy_scene.h"
#include "scene_build.h"

#define PSY_MAX_LEVELS_HOST 8

struct psy_ctx {
	struct Scratch {
		void* ptr = nullptr;
		size_t bytes = 0;
	};

	int device = 0;
	std::string last_error;
	bool has_scene = false;
	std::unique_ptr<psy::BuiltScene> host;
	std::vector<void*> scene_allocs;
	psy::DevScene dev{};
	size_t device_bytes = 0;
	unsigned* d_status = nullptr;
	unsigned* h_status = nullptr;
	std::map<std::string, Scratch> scratch;
	cudaStream_t stream_ = nullptr;
	// Halton tables (device) and the host CPU's identity-inverse diagonal
	psy::HaltonDev halton{};
	std::vector<void*> const_allocs;
	float ident_inv = 1.0f;
	psy::RcpTable rcp{};  // device copy of the host CPU's reciprocal table
	// batched rendering: the instantiated graph of the last batch and the
	// launch configuration it was captured for, and the autotuner's choice
	cudaGraphExec_t batch_graph = nullptr;
	std::vector<uint8_t> batch_graph_key;
	cudaStream_t capture_stream = nullptr;
	uint32_t tuned_stream_paths = 0;
	uint32_t tuned_block = 0;
	// optional timing of the traversal launches (psy_profile_enable)
	bool profiling = false;
	std::vector<cudaEvent_t> timer_events;
	int timer_used = 0;
	psy::LaunchTimer timer{};
	// traversal counters of the last psy_render* call (its scratch buffer)
	const unsigned long long* last_counts = nullptr;
	// BVH4 nodes the last upload built on the device (-1: built on the host)
	int gpu_bvh_nodes = -1;
	int gpu_light_nodes = -1;  // light nodes the device built for the root, -1 if none

	~psy_ctx();
	void free_scene();
	int upload(const void* src, size_t bytes, void** dst);
	// A named device buffer of at least `bytes`, reused between calls.
	void* scratch_buffer(const char* name, size_t bytes, int* rc);
	// Synchronises `stream`, reads and clears the device status word.
	int check_status(cudaStream_t stream);
	cudaStream_t host_stream() { return stream_; }
};

int ctx_fail(psy_ctx* ctx, int code, const char* fmt, ...);
int ctx_cuda(psy_ctx* ctx, cudaError_t e, const char* what);
// Makes the fixed trace array of psy_trace_host_noalloc resident on ctx's
// device (psy_noalloc.cu).
int noalloc_reserve(psy_ctx* ctx);

#endif
