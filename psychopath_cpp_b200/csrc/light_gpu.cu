/*
 * Device build of an assembly's light tree (the root assembly's, when
 * psy_scene_upload_ex is asked for device builds): LightTree::build's
 * recursive midpoint split (reference accel/light_tree.cpp:99-238) run
 * breadth first.
 *
 * Which light a path samples depends on the tree's exact shape, so the
 * device tree must be the reference's, node for node:
 *   - a segment of lights splits at the midpoint of its centres' extent on
 *     the axis of largest extent, partitioned in place with the element
 *     order of libstdc++'s std::partition on random-access iterators (the
 *     two-ended swap loop), and a split that leaves the first part empty
 *     takes its first element alone (light_tree.cpp:161-191);
 *   - nodes are numbered in the reference's depth-first order: a segment of
 *     n lights takes 2n - 1 nodes, its first part's subtree right after it,
 *     the second part's after that;
 *   - inner bounds and energies come bottom-up as unions and sums of the
 *     two children, in child order (light_tree.cpp:223-229); bounds are
 *     time-sample sequences, merged per sample when the children have as
 *     many samples, else each of the longer sequence's samples with the
 *     shorter sequence interpolated at its time.
 * The segments of one level are independent, so each level's splits run in
 * parallel: a segment of more than 32 lights is split by one warp, a smaller
 * one by one thread.  Every node's children are on the next level, so the
 * bottom-up pass runs the levels in reverse, each level's nodes in parallel.
 * The build is one kernel of one block (the levels are separated by block
 * barriers).
 */
#include <vector>

#include "kernels.h"
#include "psy_scene.h"

namespace psy {
namespace {

struct LightElem {
	float c[3];   // centre of its bounds at time 0.5
	float e;      // energy
	int inst;     // local instance index
	int box;      // its leaf bounds in the box array
};

struct Seg {
	int start, end, node;
};

constexpr int kBlock = 1024;
constexpr int kWarps = kBlock / 32;
constexpr unsigned kFull = 0xffffffffu;

// Time samples of the bounds: the lights' (light i's are samples
// [first[i], first[i + 1])), every node's while the tree is built (max_ts
// per node), and the records of a node's samples after the first.
struct LightSamples {
	const float* samples;
	const int* first;
	float* nbuf;
	int* nts;
	int max_ts;
	float* extra;       // 6 floats per record
	int* extra_count;
	int extra_base;     // record index of extra[0]
};

struct BuildOut {
	DevLightNode* nodes;
	int base;
	Seg* segs;  // every level's segments, level after level (2n - 1 in all)
	int* total; // segments written so far (shared memory)
	LightSamples ls;
};

__device__ __forceinline__ Box node_sample(const LightSamples& ls, int node, int i) {
	const float* b = ls.nbuf + ((size_t)node * ls.max_ts + i) * 6;
	Box r;
	r.lo = V3(b[0], b[1], b[2]);
	r.hi = V3(b[3], b[4], b[5]);
	return r;
}

__device__ __forceinline__ void put_sample(const LightSamples& ls, int node, int i, const Box& x) {
	float* b = ls.nbuf + ((size_t)node * ls.max_ts + i) * 6;
	b[0] = x.lo.x; b[1] = x.lo.y; b[2] = x.lo.z;
	b[3] = x.hi.x; b[4] = x.hi.y; b[5] = x.hi.z;
}

// A node's bounds in its record: sample 0 in the node, the others in extra
// records of their own.
__device__ void store_bounds(const LightSamples& ls, DevLightNode& nd, int node, int ts) {
	const Box b0 = node_sample(ls, node, 0);
	nd.lo[0] = b0.lo.x; nd.lo[1] = b0.lo.y; nd.lo[2] = b0.lo.z;
	nd.hi[0] = b0.hi.x; nd.hi[1] = b0.hi.y; nd.hi[2] = b0.hi.z;
	nd.ts = ts;
	int ex = 0;
	if (ts > 1) {
		ex = atomicAdd(ls.extra_count, ts - 1);
		for (int i = 1; i < ts; ++i) {
			const Box x = node_sample(ls, node, i);
			float* r = ls.extra + (size_t)(ex + i - 1) * 6;
			r[0] = x.lo.x; r[1] = x.lo.y; r[2] = x.lo.z;
			r[3] = x.hi.x; r[4] = x.hi.y; r[5] = x.hi.z;
		}
	}
	nd.extra = ls.extra_base + ex;
}

__device__ __forceinline__ void write_leaf(const BuildOut& o, const Seg& s, const LightElem* el) {
	DevLightNode& nd = o.nodes[s.node];
	const LightElem l = el[s.start];
	const int f = o.ls.first[l.box], ts = o.ls.first[l.box + 1] - f;
	for (int i = 0; i < ts; ++i) {
		const float* b = o.ls.samples + 6 * (size_t)(f + i);
		Box x;
		x.lo = V3(b[0], b[1], b[2]);
		x.hi = V3(b[3], b[4], b[5]);
		put_sample(o.ls, s.node, i, x);
	}
	o.ls.nts[s.node] = ts;
	store_bounds(o.ls, nd, s.node, ts);
	nd.energy = l.e;
	nd.is_leaf = 1;
	nd.c1 = l.inst;
	nd.c2 = 0;
}

// An inner node split at `mid`: its first part's subtree follows it, the
// second part's after that (2 k - 1 nodes for a part of k lights).
__device__ __forceinline__ void write_inner(const BuildOut& o, const Seg& s, int mid) {
	DevLightNode& nd = o.nodes[s.node];
	const int c1 = s.node + 1, c2 = s.node + 2 * (mid - s.start);
	nd.is_leaf = 0;
	nd.c1 = o.base + c1;
	nd.c2 = o.base + c2;
	const int q = atomicAdd(o.total, 2);
	o.segs[q] = Seg{s.start, mid, c1};
	o.segs[q + 1] = Seg{mid, s.end, c2};
}

// The split axis and plane of LightTree::split_lights (light_tree.cpp:
// 161-191): the midpoint of the centres' extent on its largest axis.
__device__ __forceinline__ void split_plane(const float mn[3], const float mx[3], int& axis, float& pmid) {
	axis = 0;
	if ((mx[1] - mn[1]) > (mx[0] - mn[0])) axis = 1;
	if ((mx[2] - mn[2]) > (mx[1] - mn[1])) axis = 2;
	pmid = .5f * (mn[axis] + mx[axis]);
}

// A segment split by one thread: the extent, then std::partition's
// two-ended loop on random-access iterators as libstdc++ writes it.
__device__ void thread_split(const BuildOut& o, const Seg& s, LightElem* el) {
	float mn[3] = {el[s.start].c[0], el[s.start].c[1], el[s.start].c[2]};
	float mx[3] = {mn[0], mn[1], mn[2]};
	for (int k = s.start + 1; k < s.end; ++k)
		for (int d = 0; d < 3; ++d) {
			const float c = el[k].c[d];
			mn[d] = mn[d] < c ? mn[d] : c;
			mx[d] = mx[d] > c ? mx[d] : c;
		}
	int axis;
	float pmid;
	split_plane(mn, mx, axis, pmid);
	int first = s.start, last = s.end;
	while (true) {
		while (first != last && el[first].c[axis] < pmid) ++first;
		if (first == last) break;
		--last;
		while (first != last && !(el[last].c[axis] < pmid)) --last;
		if (first == last) break;
		const LightElem t = el[first];
		el[first] = el[last];
		el[last] = t;
		++first;
	}
	// (every light in front of the plane only when it overflowed to infinity:
	// both parts non-empty all the same)
	write_inner(o, s, first == s.start ? first + 1 : (first == s.end ? first - 1 : first));
}

// The same split by one warp.  The two-ended loop's outcome in closed form:
// with m lights in front of the plane, its k-th swap exchanges the k-th
// light behind the plane among the first m positions (counted from the
// front) with the k-th light in front of it among the others (counted from
// the back), for as many swaps as there are such pairs.  Ballot prefix
// counts give every light its rank; pos[] holds the back ranks' positions.
__device__ void warp_split(const BuildOut& o, const Seg& s, LightElem* el, int* pos, int lane) {
	float mn[3] = {el[s.start].c[0], el[s.start].c[1], el[s.start].c[2]};
	float mx[3] = {mn[0], mn[1], mn[2]};
	for (int k = s.start + lane; k < s.end; k += 32)
		for (int d = 0; d < 3; ++d) {
			const float c = el[k].c[d];
			mn[d] = mn[d] < c ? mn[d] : c;
			mx[d] = mx[d] > c ? mx[d] : c;
		}
	for (int off = 16; off > 0; off >>= 1)
		for (int d = 0; d < 3; ++d) {
			const float a = __shfl_xor_sync(kFull, mn[d], off);
			const float b = __shfl_xor_sync(kFull, mx[d], off);
			mn[d] = mn[d] < a ? mn[d] : a;
			mx[d] = mx[d] > b ? mx[d] : b;
		}
	for (int d = 0; d < 3; ++d) {
		mn[d] = __shfl_sync(kFull, mn[d], 0);
		mx[d] = __shfl_sync(kFull, mx[d], 0);
	}
	int axis;
	float pmid;
	split_plane(mn, mx, axis, pmid);
	int cnt = 0;
	for (int k = s.start + lane; k < s.end; k += 32) cnt += el[k].c[axis] < pmid ? 1 : 0;
	const int m = (int)__reduce_add_sync(kFull, (unsigned)cnt);
	const int midp = s.start + m;
	const unsigned lt = (1u << lane) - 1u;
	// behind the plane in [start, midp) or in front of it in [midp, end)
	int before = 0, swaps = 0;
	for (int k0 = s.start; k0 < s.end; k0 += 32) {
		const int k = k0 + lane;
		bool f = false;
		if (k < s.end) {
			const bool p = el[k].c[axis] < pmid;
			f = k < midp ? !p : p;
		}
		const unsigned b = __ballot_sync(kFull, f);
		swaps += __popc(__ballot_sync(kFull, f && k < midp));
		if (f && k >= midp) pos[s.start + swaps - 1 - (before + __popc(b & lt) - swaps)] = k;
		before += __popc(b);
	}
	__syncwarp();
	int r = 0;
	for (int k0 = s.start; k0 < midp; k0 += 32) {
		const int k = k0 + lane;
		const bool f = k < midp && !(el[k].c[axis] < pmid);
		const unsigned b = __ballot_sync(kFull, f);
		if (f) {
			const int j = pos[s.start + r + __popc(b & lt)];
			const LightElem t = el[k];
			el[k] = el[j];
			el[j] = t;
		}
		r += __popc(b);
	}
	__syncwarp();
	if (lane == 0) write_inner(o, s, midp == s.start ? midp + 1 : (midp == s.end ? midp - 1 : midp));
	__syncwarp();
}

constexpr int kWarpMin = 33;  // segments of more lights split by a warp

__global__ void __launch_bounds__(kBlock) light_build_kernel(LightElem* __restrict__ el, LightSamples ls, int n,
                                                             int base, DevLightNode* __restrict__ out,
                                                             Seg* __restrict__ segs, int* __restrict__ pos,
                                                             int* __restrict__ level_start) {
	__shared__ int total, lo, hi, levels;
	if (threadIdx.x == 0) {
		segs[0] = Seg{0, n, 0};
		level_start[0] = 0;
		total = 1;
		lo = 0;
		hi = 1;
		levels = 0;
	}
	__syncthreads();
	const BuildOut o{out, base, segs, &total, ls};
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	// every level makes every segment of two or more lights strictly smaller,
	// so there are at most n levels
	for (int level = 0; level < n; ++level) {
		const int a = lo, b = hi;
		if (a == b) break;
		for (int i = a + warp; i < b; i += kWarps) {
			const Seg s = segs[i];
			if (s.end - s.start >= kWarpMin) warp_split(o, s, el, pos, lane);
		}
		for (int i = a + (int)threadIdx.x; i < b; i += kBlock) {
			const Seg s = segs[i];
			const int size = s.end - s.start;
			if (size == 1)
				write_leaf(o, s, el);
			else if (size < kWarpMin)
				thread_split(o, s, el);
		}
		__syncthreads();
		if (threadIdx.x == 0) {
			level_start[level + 1] = b;
			lo = b;
			hi = total;
			levels = level + 1;
		}
		__syncthreads();
	}
	// bounds and energies bottom-up, a level's nodes after their children's
	// (light_tree.cpp:223-229); the bounds merged as the time-sample
	// sequences of the two children: per sample when they have as many, else
	// the longer one's samples each with the shorter one interpolated at its
	// time
	for (int level = levels - 1; level >= 0; --level) {
		const int a = level_start[level], b = level_start[level + 1];
		for (int i = a + (int)threadIdx.x; i < b; i += kBlock) {
			const int node = segs[i].node;
			DevLightNode& nd = out[node];
			if (nd.is_leaf) continue;
			const int ia = nd.c1 - base, ib = nd.c2 - base;
			const int ta = ls.nts[ia], tb = ls.nts[ib];
			const int tl = ta >= tb ? ta : tb;               // the longer sequence
			const int il = ta >= tb ? ia : ib, is = ta >= tb ? ib : ia;
			const int tsh = ta >= tb ? tb : ta;
			for (int k = 0; k < tl; ++k) {
				Box other;
				if (ta == tb) {
					other = node_sample(ls, is, k);
				} else {
					const SeqPos sp = seq_pos((float)k / (float)(tl - 1), tsh);
					other = sp.single ? node_sample(ls, is, sp.i0)
					                  : box_lerp(sp.nalpha, node_sample(ls, is, sp.i0), node_sample(ls, is, sp.i0 + 1));
				}
				// equal lengths: the first child's sample first; else the
				// longer one's
				put_sample(ls, node, k, box_union(node_sample(ls, ta == tb ? ia : il, k), other));
			}
			ls.nts[node] = tl;
			store_bounds(ls, nd, node, tl);
			nd.energy = out[ia].energy + out[ib].energy;
		}
		__syncthreads();
	}
}

}  // namespace

cudaError_t build_light_tree_gpu(const float* h_elems, const float* h_samples, const int* h_first, int n,
                                 int node_base, DevLightNode* d_nodes, float* d_extra, int extra_base,
                                 float* root_energy, int* extra_count, cudaStream_t st) {
	*extra_count = 0;
	if (n < 2) return cudaErrorInvalidValue;
	std::vector<LightElem> el((size_t)n);
	int max_ts = 1;
	for (int i = 0; i < n; ++i) {
		const float* p = h_elems + 5 * (size_t)i;
		el[i] = LightElem{{p[0], p[1], p[2]}, p[3], (int)p[4], i};
		const int ts = h_first[i + 1] - h_first[i];
		if (ts < 1) return cudaErrorInvalidValue;
		max_ts = ts > max_ts ? ts : max_ts;
	}
	const size_t n_samples = (size_t)h_first[n];
	LightElem* d_el = nullptr;
	float *d_samples = nullptr, *d_nbuf = nullptr;
	Seg* d_seg = nullptr;
	int* d_int = nullptr;
	cudaError_t e = cudaMalloc(&d_el, sizeof(LightElem) * (size_t)n);
	if (e == cudaSuccess) e = cudaMalloc(&d_samples, sizeof(float) * 6 * n_samples);
	if (e == cudaSuccess) e = cudaMalloc(&d_nbuf, sizeof(float) * 6 * (size_t)max_ts * (2 * (size_t)n - 1));
	if (e == cudaSuccess) e = cudaMalloc(&d_seg, sizeof(Seg) * (2 * (size_t)n - 1));
	// pos (n), level starts (n + 1), first (n + 1), node sample counts
	// (2n - 1), the extra-record counter (1)
	if (e == cudaSuccess) e = cudaMalloc(&d_int, sizeof(int) * (5 * (size_t)n + 2));
	int* d_pos = d_int;
	int* d_level = d_int + n;
	int* d_first = d_level + n + 1;
	int* d_nts = d_first + n + 1;
	int* d_count = d_nts + 2 * n - 1;
	if (e == cudaSuccess) e = cudaMemcpyAsync(d_el, el.data(), sizeof(LightElem) * (size_t)n, cudaMemcpyHostToDevice, st);
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(d_samples, h_samples, sizeof(float) * 6 * n_samples, cudaMemcpyHostToDevice, st);
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(d_first, h_first, sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice, st);
	if (e == cudaSuccess) e = cudaMemsetAsync(d_count, 0, sizeof(int), st);
	if (e == cudaSuccess) {
		const LightSamples ls{d_samples, d_first, d_nbuf, d_nts, max_ts, d_extra, d_count, extra_base};
		light_build_kernel<<<1, kBlock, 0, st>>>(d_el, ls, n, node_base, d_nodes, d_seg, d_pos, d_level);
		e = cudaGetLastError();
	}
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(root_energy, &d_nodes[0].energy, sizeof(float), cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess) e = cudaMemcpyAsync(extra_count, d_count, sizeof(int), cudaMemcpyDeviceToHost, st);
	if (e == cudaSuccess) e = cudaStreamSynchronize(st);
	cudaFree(d_int);
	cudaFree(d_seg);
	cudaFree(d_nbuf);
	cudaFree(d_samples);
	cudaFree(d_el);
	return e;
}

}  // namespace psy
