/*
 * Device build of an assembly's traversal BVH4 (the root assembly's, when
 * psy_scene_upload_ex is asked for it): a linear BVH over the instances'
 * bounding boxes, then packed four-wide as BVH4::build packs a binary tree
 * (reference accel/bvh4.cpp:17-159: each node takes its binary children,
 * or their children when they are inner nodes).
 *
 *   1. morton_kernel     30-bit Morton code of each box centre in the
 *                        centres' bounds, with the instance index as the
 *                        low word: unique 64-bit keys, so the tree is
 *                        deterministic;
 *   2. CUB radix sort of the keys;
 *   3. radix_tree_kernel the binary radix tree of the sorted keys, one
 *                        thread per inner node (Karras, "Maximizing
 *                        Parallelism in the Construction of BVHs, Octrees,
 *                        and k-d Trees", HPG 2012);
 *   4. bounds_kernel     node boxes bottom-up: a leaf's thread climbs while
 *                        it is the second child to arrive at a node;
 *   5. collapse_kernel   BVH4 nodes level by level from a queue of binary
 *                        inner nodes, in the device node format.
 *
 * The reference builds its BVH with midpoint splits and the host builder
 * traverses a surface-area tree; which valid tree is walked changes only
 * the order candidates are met, not a ray's closest hit (exact ties aside).
 * Node boxes are exact unions (min / max) of the leaf boxes, which the host
 * computes as it does for its own trees.
 */
#include <vector>

#include <cub/cub.cuh>

#include "kernels.h"
#include "psy_scene.h"

namespace psy {
namespace {

__device__ __forceinline__ unsigned spread10(unsigned v) {
	v &= 0x3ffu;
	v = (v | (v << 16)) & 0x030000ffu;
	v = (v | (v << 8)) & 0x0300f00fu;
	v = (v | (v << 4)) & 0x030c30c3u;
	v = (v | (v << 2)) & 0x09249249u;
	return v;
}

__global__ void morton_kernel(const float* __restrict__ boxes, int n, float3 cmin, float3 cscale,
                              unsigned long long* __restrict__ keys) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const float* b = boxes + 6 * (size_t)i;
	const float c[3] = {(b[0] + b[3]) * 0.5f, (b[1] + b[4]) * 0.5f, (b[2] + b[5]) * 0.5f};
	const float lo[3] = {cmin.x, cmin.y, cmin.z};
	const float sc[3] = {cscale.x, cscale.y, cscale.z};
	unsigned q[3];
	for (int k = 0; k < 3; ++k) {
		float u = (c[k] - lo[k]) * sc[k];
		u = u != u ? 0.0f : fminf(fmaxf(u, 0.0f), 1023.0f);
		q[k] = (unsigned)u;
	}
	const unsigned m = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
	keys[i] = ((unsigned long long)m << 32) | (unsigned)i;
}

__device__ __forceinline__ int delta(const unsigned long long* keys, int n, int i, int j) {
	if (j < 0 || j >= n) return -1;
	return __clzll(keys[i] ^ keys[j]);
}

// Inner nodes are 0..n-2 (0 is the root), leaves n-1 .. 2n-2 (sorted order).
__global__ void radix_tree_kernel(const unsigned long long* __restrict__ keys, int n, int* __restrict__ left,
                                  int* __restrict__ right, int* __restrict__ parent) {
	const int i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n - 1) return;
	const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) > 0 ? 1 : -1;
	const int dmin = delta(keys, n, i, i - d);
	int lmax = 2;
	while (delta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
	int l = 0;
	for (int t = lmax / 2; t >= 1; t /= 2)
		if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
	const int j = i + l * d;
	const int dnode = delta(keys, n, i, j);
	int s = 0;
	for (int div = 2;; div *= 2) {
		const int t = (l + div - 1) / div;
		if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
		if (t == 1) break;
	}
	const int gamma = i + s * d + (d < 0 ? -1 : 0);
	const int lo = i < j ? i : j, hi = i < j ? j : i;
	const int lc = (lo == gamma) ? (n - 1) + gamma : gamma;
	const int rc = (hi == gamma + 1) ? (n - 1) + gamma + 1 : gamma + 1;
	left[i] = lc;
	right[i] = rc;
	parent[lc] = i;
	parent[rc] = i;
}

__global__ void bounds_kernel(const unsigned long long* __restrict__ keys, const float* __restrict__ boxes, int n,
                              const int* __restrict__ left, const int* __restrict__ right,
                              const int* __restrict__ parent, int* __restrict__ arrived, float* nbox) {
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= n) return;
	const int inst = (int)(keys[k] & 0xffffffffull);
	int node = (n - 1) + k;
	for (int c = 0; c < 6; ++c) nbox[6 * (size_t)node + c] = boxes[6 * (size_t)inst + c];
	while (node != 0) {
		__threadfence();
		const int p = parent[node];
		if (atomicAdd(&arrived[p], 1) == 0) return;  // the other child is not done yet
		__threadfence();
		const volatile float* a = nbox + 6 * (size_t)left[p];
		const volatile float* b = nbox + 6 * (size_t)right[p];
		float u[6];
		for (int c = 0; c < 3; ++c) {
			u[c] = fminf(a[c], b[c]);
			u[3 + c] = fmaxf(a[3 + c], b[3 + c]);
		}
		for (int c = 0; c < 6; ++c) nbox[6 * (size_t)p + c] = u[c];
		node = p;
	}
}

// One level of BVH4 nodes: each queued binary inner node becomes a device
// node whose children are its binary children, or their children when they
// are inner nodes; inner children are numbered and queued for the next level.
__global__ void collapse_kernel(const int* __restrict__ queue_in, int n_in, const int* __restrict__ index_in,
                                int* __restrict__ queue_out, int* __restrict__ index_out, int* __restrict__ n_out,
                                int* __restrict__ counter, const unsigned long long* __restrict__ keys, int n,
                                const int* __restrict__ left, const int* __restrict__ right,
                                const float* __restrict__ nbox, int node_base, DevNode* __restrict__ nodes) {
	const int q = blockIdx.x * blockDim.x + threadIdx.x;
	if (q >= n_in) return;
	const int bn = queue_in[q];
	int kids[4];
	int nk = 0;
	const int two[2] = {left[bn], right[bn]};
	for (int c = 0; c < 2; ++c) {
		const int x = two[c];
		if (x >= n - 1) {
			kids[nk++] = x;
		} else {
			kids[nk++] = left[x];
			kids[nk++] = right[x];
		}
	}
	DevNode dn;
	for (int c = 0; c < 4; ++c) {
		float b[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
		int ref = REF_EMPTY;
		if (c < nk) {
			const int x = kids[c];
			for (int k = 0; k < 6; ++k) b[k] = nbox[6 * (size_t)x + k];
			if (x >= n - 1) {
				ref = leaf_ref((int)(keys[x - (n - 1)] & 0xffffffffull));
			} else {
				const int idx = atomicAdd(counter, 1);
				const int slot = atomicAdd(n_out, 1);
				queue_out[slot] = x;
				index_out[slot] = idx;
				ref = node_base + idx;
			}
		}
		dn.b[0 * 4 + c] = b[0];
		dn.b[1 * 4 + c] = b[3];
		dn.b[2 * 4 + c] = b[1];
		dn.b[3 * 4 + c] = b[4];
		dn.b[4 * 4 + c] = b[2];
		dn.b[5 * 4 + c] = b[5];
		dn.child[c] = ref;
	}
	dn.nchild = nk;
	dn.ts = 1;
	dn.extra = 0;
	dn.pad = 0;
	nodes[index_in[q]] = dn;
}

struct Scratch {
	std::vector<void*> ptrs;
	~Scratch() {
		for (void* p : ptrs) cudaFree(p);
	}
	template <typename T>
	cudaError_t get(T** out, size_t count) {
		void* p = nullptr;
		const cudaError_t e = cudaMalloc(&p, (count ? count : 1) * sizeof(T));
		if (e == cudaSuccess) ptrs.push_back(p);
		*out = static_cast<T*>(p);
		return e;
	}
};

#define PSY_TRY(x)                           \
	do {                                     \
		const cudaError_t e_ = (x);          \
		if (e_ != cudaSuccess) return e_;    \
	} while (0)

}  // namespace

cudaError_t build_bvh4_gpu(const float* h_boxes, int n, int node_base, DevNode* d_nodes, int* root_ref,
                           int* node_count, cudaStream_t st) {
	*node_count = 0;
	if (n == 0) {
		*root_ref = REF_EMPTY;
		return cudaSuccess;
	}
	if (n == 1) {
		*root_ref = leaf_ref(0);
		return cudaSuccess;
	}
	// centre bounds (host: the boxes are there already)
	float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
	for (int i = 0; i < n; ++i)
		for (int k = 0; k < 3; ++k) {
			const float c = (h_boxes[6 * (size_t)i + k] + h_boxes[6 * (size_t)i + 3 + k]) * 0.5f;
			if (c == c) {
				lo[k] = fminf(lo[k], c);
				hi[k] = fmaxf(hi[k], c);
			}
		}
	float scale[3];
	for (int k = 0; k < 3; ++k) {
		const float ext = hi[k] - lo[k];
		scale[k] = (ext > 0.0f && ext == ext) ? 1023.0f / ext : 0.0f;
		if (!(lo[k] == lo[k]) || lo[k] == INFINITY) lo[k] = 0.0f;
	}
	Scratch s;
	float *d_boxes, *d_nbox;
	unsigned long long *d_keys, *d_sorted;
	int *d_left, *d_right, *d_parent, *d_arrived, *d_q[2], *d_idx[2], *d_count;
	PSY_TRY(s.get(&d_boxes, 6 * (size_t)n));
	PSY_TRY(s.get(&d_nbox, 6 * (size_t)(2 * n - 1)));
	PSY_TRY(s.get(&d_keys, n));
	PSY_TRY(s.get(&d_sorted, n));
	PSY_TRY(s.get(&d_left, n - 1));
	PSY_TRY(s.get(&d_right, n - 1));
	PSY_TRY(s.get(&d_parent, 2 * n - 1));
	PSY_TRY(s.get(&d_arrived, n - 1));
	PSY_TRY(s.get(&d_q[0], n));
	PSY_TRY(s.get(&d_q[1], n));
	PSY_TRY(s.get(&d_idx[0], n));
	PSY_TRY(s.get(&d_idx[1], n));
	PSY_TRY(s.get(&d_count, 2));
	PSY_TRY(cudaMemcpyAsync(d_boxes, h_boxes, 6 * sizeof(float) * (size_t)n, cudaMemcpyHostToDevice, st));
	PSY_TRY(cudaMemsetAsync(d_arrived, 0, sizeof(int) * (size_t)(n - 1), st));
	const int B = 256;
	morton_kernel<<<(n + B - 1) / B, B, 0, st>>>(d_boxes, n, make_float3(lo[0], lo[1], lo[2]),
	                                             make_float3(scale[0], scale[1], scale[2]), d_keys);
	PSY_TRY(cudaGetLastError());
	size_t temp_bytes = 0;
	PSY_TRY(cub::DeviceRadixSort::SortKeys(nullptr, temp_bytes, d_keys, d_sorted, n, 0, 64, st));
	unsigned char* d_temp;
	PSY_TRY(s.get(&d_temp, temp_bytes));
	PSY_TRY(cub::DeviceRadixSort::SortKeys(d_temp, temp_bytes, d_keys, d_sorted, n, 0, 64, st));
	radix_tree_kernel<<<(n - 1 + B - 1) / B, B, 0, st>>>(d_sorted, n, d_left, d_right, d_parent);
	PSY_TRY(cudaGetLastError());
	bounds_kernel<<<(n + B - 1) / B, B, 0, st>>>(d_sorted, d_boxes, n, d_left, d_right, d_parent, d_arrived, d_nbox);
	PSY_TRY(cudaGetLastError());
	// level by level from the root (binary inner node 0, device node 0)
	const int zero_one[2] = {0, 1};
	PSY_TRY(cudaMemcpyAsync(d_q[0], &zero_one[0], sizeof(int), cudaMemcpyHostToDevice, st));
	PSY_TRY(cudaMemcpyAsync(d_idx[0], &zero_one[0], sizeof(int), cudaMemcpyHostToDevice, st));
	PSY_TRY(cudaMemcpyAsync(d_count, &zero_one[1], sizeof(int), cudaMemcpyHostToDevice, st));  // nodes numbered
	int n_in = 1, cur = 0;
	while (n_in > 0) {
		PSY_TRY(cudaMemsetAsync(d_count + 1, 0, sizeof(int), st));
		collapse_kernel<<<(n_in + B - 1) / B, B, 0, st>>>(d_q[cur], n_in, d_idx[cur], d_q[1 - cur], d_idx[1 - cur],
		                                                  d_count + 1, d_count, d_sorted, n, d_left, d_right,
		                                                  d_nbox, node_base, d_nodes);
		PSY_TRY(cudaGetLastError());
		PSY_TRY(cudaMemcpyAsync(&n_in, d_count + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
		PSY_TRY(cudaStreamSynchronize(st));
		cur = 1 - cur;
	}
	int total = 0;
	PSY_TRY(cudaMemcpyAsync(&total, d_count, sizeof(int), cudaMemcpyDeviceToHost, st));
	PSY_TRY(cudaStreamSynchronize(st));
	*node_count = total;
	*root_ref = node_base;
	return cudaSuccess;
}

}  // namespace psy
