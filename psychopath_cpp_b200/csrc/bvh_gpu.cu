/*
 * Device build of an assembly's traversal BVH4 (the root assembly's, when
 * psy_scene_upload_ex is asked for it): the host builder's binned
 * surface-area tree, split for split, then packed four-wide as
 * BVH4::build packs a binary tree (reference accel/bvh4.cpp:17-159: each
 * node takes its binary children, or their children when they are inner
 * nodes).
 *
 *   1. sah_build_kernel  the binary tree, top down and level by level in one
 *                        block: a segment of more than 32 instances is split
 *                        by one warp (bins in shared memory), a smaller one
 *                        by one thread.  Each split is the host's: 16 bins
 *                        per axis over the centres' extent, the cheapest bin
 *                        boundary by half-area times count (in double), the
 *                        elements partitioned in libstdc++'s std::partition
 *                        order, and the reference's midpoint split
 *                        (accel/bvh.cpp:89-188) when no boundary separates
 *                        them.  An inner node is numbered by its split
 *                        position (the last index of its first part), a leaf
 *                        by n - 1 + its position;
 *   2. bounds_kernel     node boxes bottom-up: a leaf's thread climbs while
 *                        it is the second child to arrive at a node;
 *   3. collapse_kernel   BVH4 nodes level by level from a queue of binary
 *                        inner nodes, in the device node format.
 *
 * The tree is the host build's node for node (in another node numbering),
 * so a ray visits the same nodes in the same order either way.  Node boxes
 * are exact unions of the instances' boxes, which the host computes as it
 * does for its own trees.
 */
#include <vector>

#include "kernels.h"
#include "psy_scene.h"

namespace psy {
namespace {

constexpr int kNB = 16;            // bins per axis
constexpr int kBlock = 1024;
constexpr int kWarps = kBlock / 32;
constexpr int kWarpMin = 33;       // segments of more instances split by a warp
constexpr unsigned kFull = 0xffffffffu;

struct SahElem {
	float c[3];  // centre of the instance's box at time 0.5
	int inst;    // instance (and box) index
};

// A segment of the element array, the node it becomes a child of (-1 for
// the root) and on which side.
struct Seg {
	int start, end, parent, side;
};

struct Bins {
	float lo[3 * kNB][3], hi[3 * kNB][3];
	int cnt[3 * kNB];
};

__device__ __forceinline__ float half_area_dev(const float lo[3], const float hi[3]) {
	const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
	if (!(dx >= 0.0f && dy >= 0.0f && dz >= 0.0f)) return 0.0f;
	return dx * dy + dy * dz + dz * dx;
}

__device__ __forceinline__ int bin_of(float c, float mn, float ext) {
	const int k = (int)((c - mn) / ext * (float)kNB);
	return k < 0 ? 0 : (k >= kNB ? kNB - 1 : k);
}

// Float min / max through integer atomics (ordered by the sign bit: the
// bit patterns of non-negative floats order as signed integers, those of
// negative floats in reverse as unsigned ones).
__device__ __forceinline__ void atomic_min_f(float* a, float v) {
	if (!(__float_as_uint(v) >> 31))
		atomicMin(reinterpret_cast<int*>(a), __float_as_int(v));
	else
		atomicMax(reinterpret_cast<unsigned*>(a), __float_as_uint(v));
}

__device__ __forceinline__ void atomic_max_f(float* a, float v) {
	if (!(__float_as_uint(v) >> 31))
		atomicMax(reinterpret_cast<int*>(a), __float_as_int(v));
	else
		atomicMin(reinterpret_cast<unsigned*>(a), __float_as_uint(v));
}

// The sweeps of one axis's bins, as the host's sah_split runs them: the
// cost of each boundary against the best so far (strictly cheaper wins, so
// the first of equal costs stays).
__device__ void sah_sweep(const float (*blo)[3], const float (*bhi)[3], const int* bcnt, int axis, double& best,
                          int& best_axis, int& best_bin) {
	double right_area[kNB];
	int right_cnt[kNB];
	float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
	int n = 0;
	for (int k = kNB - 1; k >= 0; --k) {
		for (int d = 0; d < 3; ++d) {
			lo[d] = fminf(lo[d], blo[k][d]);
			hi[d] = fmaxf(hi[d], bhi[k][d]);
		}
		n += bcnt[k];
		right_area[k] = half_area_dev(lo, hi);
		right_cnt[k] = n;
	}
	for (int d = 0; d < 3; ++d) {
		lo[d] = INFINITY;
		hi[d] = -INFINITY;
	}
	n = 0;
	for (int k = 0; k < kNB - 1; ++k) {
		for (int d = 0; d < 3; ++d) {
			lo[d] = fminf(lo[d], blo[k][d]);
			hi[d] = fmaxf(hi[d], bhi[k][d]);
		}
		n += bcnt[k];
		if (n == 0 || right_cnt[k + 1] == 0) continue;
		const double cost = (double)half_area_dev(lo, hi) * (double)n + right_area[k + 1] * (double)right_cnt[k + 1];
		if (cost < best) {
			best = cost;
			best_axis = axis;
			best_bin = k;
		}
	}
}

// The reference's midpoint split plane (accel/bvh.cpp:89-128): the
// midpoint of the centres' extent on its largest axis.
__device__ __forceinline__ void mid_plane(const float mn[3], const float mx[3], int& axis, float& pmid) {
	axis = 0;
	if ((mx[1] - mn[1]) > (mx[0] - mn[0])) axis = 1;
	if ((mx[2] - mn[2]) > (mx[1] - mn[1])) axis = 2;
	pmid = .5f * (mn[axis] + mx[axis]);
}

// Which side of a split an element goes to: by bin (surface-area split) or
// by plane (midpoint split).
struct SplitPred {
	int axis, bin;  // bin >= 0: surface-area split
	float mn, ext, pmid;
	__device__ __forceinline__ bool operator()(const SahElem& e) const {
		return bin >= 0 ? bin_of(e.c[axis], mn, ext) <= bin : e.c[axis] < pmid;
	}
};

// std::partition's two-ended loop on random-access iterators, as libstdc++
// writes it; returns the partition point.
__device__ int thread_partition(SahElem* el, int first, int last, const SplitPred& p) {
	while (true) {
		while (first != last && p(el[first])) ++first;
		if (first == last) return first;
		--last;
		while (first != last && !p(el[last])) --last;
		if (first == last) return first;
		const SahElem t = el[first];
		el[first] = el[last];
		el[last] = t;
		++first;
	}
}

// The same partition by one warp, in closed form: with m elements
// satisfying the predicate, the loop's k-th swap exchanges the k-th element
// failing it among the first m positions (from the front) with the k-th
// element satisfying it among the others (from the back).  Ballot prefix
// counts rank them; pos[] holds the back ranks' positions.
__device__ int warp_partition(SahElem* el, int* pos, int start, int end, const SplitPred& p, int lane) {
	int cnt = 0;
	for (int k = start + lane; k < end; k += 32) cnt += p(el[k]) ? 1 : 0;
	const int m = (int)__reduce_add_sync(kFull, (unsigned)cnt);
	const int midp = start + m;
	const unsigned lt = (1u << lane) - 1u;
	int before = 0, swaps = 0;
	for (int k0 = start; k0 < end; k0 += 32) {
		const int k = k0 + lane;
		bool f = false;
		if (k < end) {
			const bool q = p(el[k]);
			f = k < midp ? !q : q;
		}
		const unsigned b = __ballot_sync(kFull, f);
		swaps += __popc(__ballot_sync(kFull, f && k < midp));
		if (f && k >= midp) pos[start + swaps - 1 - (before + __popc(b & lt) - swaps)] = k;
		before += __popc(b);
	}
	__syncwarp();
	int r = 0;
	for (int k0 = start; k0 < midp; k0 += 32) {
		const int k = k0 + lane;
		const bool f = k < midp && !p(el[k]);
		const unsigned b = __ballot_sync(kFull, f);
		if (f) {
			const int j = pos[start + r + __popc(b & lt)];
			const SahElem t = el[k];
			el[k] = el[j];
			el[j] = t;
		}
		r += __popc(b);
	}
	__syncwarp();
	return midp;
}

struct SahOut {
	int* left;                  // binary inner nodes' children
	int* right;
	int* parent;                // every node's parent
	unsigned long long* keys;   // leaf k's instance in the low word
	int* root;
	Seg* segs;                  // every level's segments, level after level
	int* total;                 // segments written so far (shared memory)
};

// A segment's node, linked to its parent.
__device__ __forceinline__ void link(const SahOut& o, const Seg& s, int id) {
	if (s.parent < 0)
		*o.root = id;
	else
		(s.side ? o.right : o.left)[s.parent] = id;
	o.parent[id] = s.parent;
}

// An inner node split at `mid` (its first part [start, mid)).
__device__ __forceinline__ void emit_inner(const SahOut& o, const Seg& s, int mid) {
	const int id = mid - 1;
	link(o, s, id);
	const int q = atomicAdd(o.total, 2);
	o.segs[q] = Seg{s.start, mid, id, 0};
	o.segs[q + 1] = Seg{mid, s.end, id, 1};
}

__device__ void thread_split(const SahOut& o, const Seg& s, SahElem* el, const float* boxes) {
	float mn[3] = {el[s.start].c[0], el[s.start].c[1], el[s.start].c[2]};
	float mx[3] = {mn[0], mn[1], mn[2]};
	for (int k = s.start + 1; k < s.end; ++k)
		for (int d = 0; d < 3; ++d) {
			const float c = el[k].c[d];
			mn[d] = c < mn[d] ? c : mn[d];
			mx[d] = mx[d] < c ? c : mx[d];
		}
	double best = INFINITY;
	int best_axis = -1, best_bin = -1;
	float blo[kNB][3], bhi[kNB][3];
	int bcnt[kNB];
	for (int axis = 0; axis < 3; ++axis) {
		const float ext = mx[axis] - mn[axis];
		if (!(ext > 0.0f)) continue;
		for (int k = 0; k < kNB; ++k) {
			for (int d = 0; d < 3; ++d) {
				blo[k][d] = INFINITY;
				bhi[k][d] = -INFINITY;
			}
			bcnt[k] = 0;
		}
		for (int i = s.start; i < s.end; ++i) {
			const int k = bin_of(el[i].c[axis], mn[axis], ext);
			const float* bb = boxes + 6 * (size_t)el[i].inst;
			for (int d = 0; d < 3; ++d) {
				blo[k][d] = fminf(blo[k][d], bb[d]);
				bhi[k][d] = fmaxf(bhi[k][d], bb[3 + d]);
			}
			++bcnt[k];
		}
		sah_sweep(blo, bhi, bcnt, axis, best, best_axis, best_bin);
	}
	int mid = -1;
	if (best_axis >= 0) {
		const SplitPred p{best_axis, best_bin, mn[best_axis], mx[best_axis] - mn[best_axis], 0.0f};
		mid = thread_partition(el, s.start, s.end, p);
		if (!(mid > s.start && mid < s.end)) mid = -1;
	}
	if (mid < 0) {
		SplitPred p{0, -1, 0.0f, 0.0f, 0.0f};
		mid_plane(mn, mx, p.axis, p.pmid);
		mid = thread_partition(el, s.start, s.end, p);
		if (mid == s.start) ++mid;
		// every element in front of the plane only when it overflowed to
		// infinity: both parts non-empty all the same
		if (mid == s.end) --mid;
	}
	emit_inner(o, s, mid);
}

__device__ void warp_split(const SahOut& o, const Seg& s, SahElem* el, const float* boxes, int* pos, Bins& b,
                           int lane) {
	float mn[3] = {el[s.start].c[0], el[s.start].c[1], el[s.start].c[2]};
	float mx[3] = {mn[0], mn[1], mn[2]};
	for (int k = s.start + lane; k < s.end; k += 32)
		for (int d = 0; d < 3; ++d) {
			const float c = el[k].c[d];
			mn[d] = c < mn[d] ? c : mn[d];
			mx[d] = mx[d] < c ? c : mx[d];
		}
	for (int off = 16; off > 0; off >>= 1)
		for (int d = 0; d < 3; ++d) {
			const float a = __shfl_xor_sync(kFull, mn[d], off);
			const float c = __shfl_xor_sync(kFull, mx[d], off);
			mn[d] = a < mn[d] ? a : mn[d];
			mx[d] = mx[d] < c ? c : mx[d];
		}
	for (int d = 0; d < 3; ++d) {
		mn[d] = __shfl_sync(kFull, mn[d], 0);
		mx[d] = __shfl_sync(kFull, mx[d], 0);
	}
	for (int j = lane; j < 3 * kNB; j += 32) {
		for (int d = 0; d < 3; ++d) {
			b.lo[j][d] = INFINITY;
			b.hi[j][d] = -INFINITY;
		}
		b.cnt[j] = 0;
	}
	__syncwarp();
	const float ext[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
	for (int i = s.start + lane; i < s.end; i += 32) {
		const SahElem e = el[i];
		const float* bb = boxes + 6 * (size_t)e.inst;
		for (int axis = 0; axis < 3; ++axis) {
			if (!(ext[axis] > 0.0f)) continue;
			const int j = axis * kNB + bin_of(e.c[axis], mn[axis], ext[axis]);
			for (int d = 0; d < 3; ++d) {
				atomic_min_f(&b.lo[j][d], bb[d]);
				atomic_max_f(&b.hi[j][d], bb[3 + d]);
			}
			atomicAdd(&b.cnt[j], 1);
		}
	}
	__syncwarp();
	int best_axis = -1, best_bin = -1;
	if (lane == 0) {
		double best = INFINITY;
		for (int axis = 0; axis < 3; ++axis)
			if (ext[axis] > 0.0f)
				sah_sweep(&b.lo[axis * kNB], &b.hi[axis * kNB], &b.cnt[axis * kNB], axis, best, best_axis, best_bin);
	}
	best_axis = __shfl_sync(kFull, best_axis, 0);
	best_bin = __shfl_sync(kFull, best_bin, 0);
	int mid = -1;
	if (best_axis >= 0) {
		const SplitPred p{best_axis, best_bin, mn[best_axis], ext[best_axis], 0.0f};
		mid = warp_partition(el, pos, s.start, s.end, p, lane);
		if (!(mid > s.start && mid < s.end)) mid = -1;
	}
	if (mid < 0) {
		SplitPred p{0, -1, 0.0f, 0.0f, 0.0f};
		mid_plane(mn, mx, p.axis, p.pmid);
		mid = warp_partition(el, pos, s.start, s.end, p, lane);
		if (mid == s.start) ++mid;
		if (mid == s.end) --mid;
	}
	if (lane == 0) emit_inner(o, s, mid);
	__syncwarp();
}

__global__ void __launch_bounds__(kBlock, 1) sah_build_kernel(SahElem* __restrict__ el, const float* __restrict__ boxes,
                                                           int n, SahOut o, int* __restrict__ pos) {
	__shared__ Bins bins[kWarps];
	__shared__ int total, lo, hi;
	if (threadIdx.x == 0) {
		o.segs[0] = Seg{0, n, -1, 0};
		total = 1;
		lo = 0;
		hi = 1;
	}
	__syncthreads();
	o.total = &total;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	// every level makes every segment of two or more elements strictly
	// smaller, so there are at most n levels
	for (int level = 0; level < n; ++level) {
		const int a = lo, b = hi;
		if (a == b) break;
		for (int i = a + warp; i < b; i += kWarps) {
			const Seg s = o.segs[i];
			if (s.end - s.start >= kWarpMin) warp_split(o, s, el, boxes, pos, bins[warp], lane);
		}
		for (int i = a + (int)threadIdx.x; i < b; i += kBlock) {
			const Seg s = o.segs[i];
			const int size = s.end - s.start;
			if (size == 1) {
				link(o, s, (n - 1) + s.start);
				o.keys[s.start] = (unsigned long long)(unsigned)el[s.start].inst;
			} else if (size < kWarpMin) {
				thread_split(o, s, el, boxes);
			}
		}
		__syncthreads();
		if (threadIdx.x == 0) {
			lo = b;
			hi = total;
		}
		__syncthreads();
	}
}

// A node's time sample i: nbox holds max_ts samples per node.
__device__ __forceinline__ Box node_box(const float* nbox, int max_ts, int node, int i) {
	const volatile float* b = nbox + ((size_t)node * max_ts + i) * 6;
	Box r;
	r.lo = V3(b[0], b[1], b[2]);
	r.hi = V3(b[3], b[4], b[5]);
	return r;
}

__device__ __forceinline__ void put_box(float* nbox, int max_ts, int node, int i, const Box& x) {
	float* b = nbox + ((size_t)node * max_ts + i) * 6;
	b[0] = x.lo.x; b[1] = x.lo.y; b[2] = x.lo.z;
	b[3] = x.hi.x; b[4] = x.hi.y; b[5] = x.hi.z;
}

// Node boxes bottom-up, with the host builder's time-sample rule: children
// with as many samples give their per-sample unions, children with
// different counts one box over all of their samples.
__global__ void bounds_kernel(const unsigned long long* __restrict__ keys, const float* __restrict__ samples,
                              const int* __restrict__ first, int n, int max_ts, int root,
                              const int* __restrict__ left, const int* __restrict__ right,
                              const int* __restrict__ parent, int* __restrict__ arrived, int* nts, float* nbox) {
	const int k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= n) return;
	const int inst = (int)(keys[k] & 0xffffffffull);
	int node = (n - 1) + k;
	const int ts = first[inst + 1] - first[inst];
	for (int i = 0; i < ts; ++i) {
		const float* s = samples + 6 * (size_t)(first[inst] + i);
		Box x;
		x.lo = V3(s[0], s[1], s[2]);
		x.hi = V3(s[3], s[4], s[5]);
		put_box(nbox, max_ts, node, i, x);
	}
	nts[node] = ts;
	while (node != root) {
		__threadfence();
		const int p = parent[node];
		if (atomicAdd(&arrived[p], 1) == 0) return;  // the other child is not done yet
		__threadfence();
		const int a = left[p], b = right[p];
		const int ta = ((const volatile int*)nts)[a], tb = ((const volatile int*)nts)[b];
		if (ta == tb) {
			for (int i = 0; i < ta; ++i)
				put_box(nbox, max_ts, p, i, box_union(node_box(nbox, max_ts, a, i), node_box(nbox, max_ts, b, i)));
			nts[p] = ta;
		} else {
			Box m = node_box(nbox, max_ts, a, 0);
			for (int i = 1; i < ta; ++i) m = box_union(m, node_box(nbox, max_ts, a, i));
			for (int i = 0; i < tb; ++i) m = box_union(m, node_box(nbox, max_ts, b, i));
			put_box(nbox, max_ts, p, 0, m);
			nts[p] = 1;
		}
		node = p;
	}
}

// One level of BVH4 nodes: each queued binary inner node becomes a device
// node whose children are its binary children, or their children when they
// are inner nodes; inner children are numbered and queued for the next level.
// A node's time samples are its children's when they have as many, else as
// many as the most of them, the others' boxes interpolated at each sample's
// time (BVH4::build, accel/bvh4.cpp:88-135); samples after the first go to
// the extra records.
__global__ void collapse_kernel(const int* __restrict__ queue_in, int n_in, const int* __restrict__ index_in,
                                int* __restrict__ queue_out, int* __restrict__ index_out, int* __restrict__ n_out,
                                int* __restrict__ counter, const unsigned long long* __restrict__ keys, int n,
                                const int* __restrict__ left, const int* __restrict__ right,
                                const int* __restrict__ nts, const float* __restrict__ nbox, int max_ts,
                                int node_base, DevNode* __restrict__ nodes, float* __restrict__ extra,
                                int* __restrict__ extra_count, int extra_base) {
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
	bool equal_ts = true;
	int most = nts[kids[0]];
	for (int c = 1; c < nk; ++c) {
		equal_ts = equal_ts && nts[kids[c - 1]] == nts[kids[c]];
		most = nts[kids[c]] > most ? nts[kids[c]] : most;
	}
	const int rts = equal_ts ? nts[kids[0]] : most;
	const int ex = rts > 1 ? atomicAdd(extra_count, rts - 1) : 0;
	for (int i = 0; i < rts; ++i) {
		float* rec = i == 0 ? dn.b : extra + (size_t)(ex + i - 1) * 24;
		for (int c = 0; c < 4; ++c) {
			Box x = box_empty();
			if (c < nk) {
				const int kc = kids[c], tc = nts[kc];
				if (equal_ts || tc == most) {
					x = node_box(nbox, max_ts, kc, i);
				} else {
					const SeqPos sp = seq_pos((float)i / (float)(most - 1), tc);
					x = sp.single ? node_box(nbox, max_ts, kc, sp.i0)
					              : box_lerp(sp.nalpha, node_box(nbox, max_ts, kc, sp.i0),
					                         node_box(nbox, max_ts, kc, sp.i0 + 1));
				}
			}
			rec[0 * 4 + c] = x.lo.x;
			rec[1 * 4 + c] = x.hi.x;
			rec[2 * 4 + c] = x.lo.y;
			rec[3 * 4 + c] = x.hi.y;
			rec[4 * 4 + c] = x.lo.z;
			rec[5 * 4 + c] = x.hi.z;
		}
	}
	for (int c = 0; c < 4; ++c) {
		int ref = REF_EMPTY;
		if (c < nk) {
			const int x = kids[c];
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
		dn.child[c] = ref;
	}
	dn.nchild = nk;
	dn.ts = rts;
	dn.extra = rts > 1 ? extra_base + ex : 0;
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

cudaError_t build_bvh4_gpu(const float* h_samples, const int* h_first, const float* h_centres, int n,
                           int node_base, DevNode* d_nodes, float* d_extra, int extra_base, int* root_ref,
                           int* node_count, int* extra_count, cudaStream_t st) {
	*node_count = 0;
	*extra_count = 0;
	if (n == 0) {
		*root_ref = REF_EMPTY;
		return cudaSuccess;
	}
	if (n == 1) {
		*root_ref = leaf_ref(0);
		return cudaSuccess;
	}
	// the surface-area split bins each instance's box over all its samples
	std::vector<SahElem> el((size_t)n);
	std::vector<float> ubox(6 * (size_t)n);
	int max_ts = 1;
	for (int i = 0; i < n; ++i) {
		el[i] = SahElem{{h_centres[3 * (size_t)i], h_centres[3 * (size_t)i + 1], h_centres[3 * (size_t)i + 2]}, i};
		const int ts = h_first[i + 1] - h_first[i];
		if (ts < 1) return cudaErrorInvalidValue;
		max_ts = ts > max_ts ? ts : max_ts;
		Box u = box_empty();
		for (int k = 0; k < ts; ++k) {
			const float* s = h_samples + 6 * (size_t)(h_first[i] + k);
			Box x;
			x.lo = V3(s[0], s[1], s[2]);
			x.hi = V3(s[3], s[4], s[5]);
			u = box_union(u, x);
		}
		const float f[6] = {u.lo.x, u.lo.y, u.lo.z, u.hi.x, u.hi.y, u.hi.z};
		for (int c = 0; c < 6; ++c) ubox[6 * (size_t)i + c] = f[c];
	}
	const size_t n_samples = (size_t)h_first[n];
	Scratch s;
	SahElem* d_el;
	Seg* d_seg;
	float *d_ubox, *d_samples, *d_nbox;
	unsigned long long* d_keys;
	int *d_first, *d_nts, *d_left, *d_right, *d_parent, *d_arrived, *d_pos, *d_q[2], *d_idx[2], *d_count;
	PSY_TRY(s.get(&d_el, n));
	PSY_TRY(s.get(&d_seg, 2 * (size_t)n - 1));
	PSY_TRY(s.get(&d_ubox, 6 * (size_t)n));
	PSY_TRY(s.get(&d_samples, 6 * n_samples));
	PSY_TRY(s.get(&d_first, (size_t)n + 1));
	PSY_TRY(s.get(&d_nbox, 6 * (size_t)max_ts * (size_t)(2 * n - 1)));
	PSY_TRY(s.get(&d_nts, 2 * (size_t)n - 1));
	PSY_TRY(s.get(&d_keys, n));
	PSY_TRY(s.get(&d_left, n - 1));
	PSY_TRY(s.get(&d_right, n - 1));
	PSY_TRY(s.get(&d_parent, 2 * n - 1));
	PSY_TRY(s.get(&d_arrived, n - 1));
	PSY_TRY(s.get(&d_pos, n));
	PSY_TRY(s.get(&d_q[0], n));
	PSY_TRY(s.get(&d_q[1], n));
	PSY_TRY(s.get(&d_idx[0], n));
	PSY_TRY(s.get(&d_idx[1], n));
	PSY_TRY(s.get(&d_count, 4));
	PSY_TRY(cudaMemcpyAsync(d_el, el.data(), sizeof(SahElem) * (size_t)n, cudaMemcpyHostToDevice, st));
	PSY_TRY(cudaMemcpyAsync(d_ubox, ubox.data(), sizeof(float) * ubox.size(), cudaMemcpyHostToDevice, st));
	PSY_TRY(cudaMemcpyAsync(d_samples, h_samples, 6 * sizeof(float) * n_samples, cudaMemcpyHostToDevice, st));
	PSY_TRY(cudaMemcpyAsync(d_first, h_first, sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice, st));
	PSY_TRY(cudaMemsetAsync(d_arrived, 0, sizeof(int) * (size_t)(n - 1), st));
	PSY_TRY(cudaMemsetAsync(d_count, 0, sizeof(int) * 4, st));
	const SahOut o{d_left, d_right, d_parent, d_keys, d_count + 2, d_seg, nullptr};
	sah_build_kernel<<<1, kBlock, 0, st>>>(d_el, d_ubox, n, o, d_pos);
	PSY_TRY(cudaGetLastError());
	int root = 0;
	PSY_TRY(cudaMemcpyAsync(&root, d_count + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
	PSY_TRY(cudaStreamSynchronize(st));
	if (root < 0 || root >= n - 1) return cudaErrorUnknown;  // n >= 2: the root is an inner node
	const int B = 256;
	bounds_kernel<<<(n + B - 1) / B, B, 0, st>>>(d_keys, d_samples, d_first, n, max_ts, root, d_left, d_right,
	                                             d_parent, d_arrived, d_nts, d_nbox);
	PSY_TRY(cudaGetLastError());
	// level by level from the root (device node 0)
	const int zero_one[2] = {0, 1};
	PSY_TRY(cudaMemcpyAsync(d_q[0], &root, sizeof(int), cudaMemcpyHostToDevice, st));
	PSY_TRY(cudaMemcpyAsync(d_idx[0], &zero_one[0], sizeof(int), cudaMemcpyHostToDevice, st));
	PSY_TRY(cudaMemcpyAsync(d_count, &zero_one[1], sizeof(int), cudaMemcpyHostToDevice, st));  // nodes numbered
	int n_in = 1, cur = 0;
	while (n_in > 0) {
		PSY_TRY(cudaMemsetAsync(d_count + 1, 0, sizeof(int), st));
		collapse_kernel<<<(n_in + B - 1) / B, B, 0, st>>>(d_q[cur], n_in, d_idx[cur], d_q[1 - cur], d_idx[1 - cur],
		                                                  d_count + 1, d_count, d_keys, n, d_left, d_right, d_nts,
		                                                  d_nbox, max_ts, node_base, d_nodes, d_extra, d_count + 3,
		                                                  extra_base);
		PSY_TRY(cudaGetLastError());
		PSY_TRY(cudaMemcpyAsync(&n_in, d_count + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
		PSY_TRY(cudaStreamSynchronize(st));
		cur = 1 - cur;
	}
	int totals[4] = {0, 0, 0, 0};
	PSY_TRY(cudaMemcpyAsync(totals, d_count, sizeof(totals), cudaMemcpyDeviceToHost, st));
	PSY_TRY(cudaStreamSynchronize(st));
	*node_count = totals[0];
	*extra_count = totals[3];
	*root_ref = node_base;
	return cudaSuccess;
}

}  // namespace psy
