/*
 * Host scene preparation (the Assembly::finalize step of the reference,
 * scene/assembly.hpp:206-238), producing the device tables of psy_scene.h.
 *
 * The acceleration structures are built with the reference's algorithms so
 * that the device traverses the same BVH4 and samples the same light tree:
 *   - object bounds per time sample (object/sphere.cpp:51-62,
 *     object/bilinear.cpp:22-34, object/bicubic.cpp:85-96,
 *     lights/sphere_light.hpp:22-55);
 *   - instance bounds (scene/assembly.hpp:261-312, basics/bbox.hpp:638-669);
 *   - BVH: midpoint split on the centroid axis of largest extent, one
 *     instance per leaf (accel/bvh.cpp:14-188);
 *   - BVH4: the reference's packing of that BVH (accel/bvh4.cpp:17-159);
 *   - light tree (accel/light_tree.cpp:99-238).
 * Where the reference partitions with std::partition, the same element order
 * is produced (the bidirectional partition of libstdc++), so degenerate
 * splits pick the same elements.
 */
#include "scene_build.h"

#include "host_cpu.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <numeric>

namespace psy {

namespace {

// libstdc++'s std::partition for bidirectional iterators.
template <typename T, typename Pred>
size_t bidir_partition(std::vector<T>& v, size_t first, size_t last, Pred pred) {
	while (true) {
		while (true) {
			if (first == last) return first;
			if (pred(v[first])) ++first;
			else break;
		}
		--last;
		while (true) {
			if (first == last) return first;
			if (!pred(v[last])) --last;
			else break;
		}
		std::swap(v[first], v[last]);
		++first;
	}
}

M44 load_m44(const float* p) {
	M44 m;
	for (int i = 0; i < 16; ++i) m.m[i / 4][i % 4] = p[i];
	return m;
}

Box lerp_seq_box(float alpha, const std::vector<Box>& seq) {
	const SeqPos sp = seq_pos(alpha, (int)seq.size());
	if (sp.single) return seq[sp.i0];
	return box_lerp(sp.nalpha, seq[sp.i0], seq[sp.i0 + 1]);
}

M44 lerp_seq_m44(float alpha, const M44* seq, int count) {
	const SeqPos sp = seq_pos(alpha, count);
	if (sp.single) return seq[sp.i0];
	return m44_lerp(sp.nalpha, seq[sp.i0], seq[sp.i0 + 1]);
}

V3 lerp_seq_v3(float alpha, const std::vector<V3>& seq) {
	const SeqPos sp = seq_pos(alpha, (int)seq.size());
	if (sp.single) return seq[sp.i0];
	return lerp3(sp.nalpha, seq[sp.i0], seq[sp.i0 + 1]);
}

float lerp_seq_f(float alpha, const std::vector<float>& seq) {
	const SeqPos sp = seq_pos(alpha, (int)seq.size());
	if (sp.single) return seq[sp.i0];
	return lerp1(sp.nalpha, seq[sp.i0], seq[sp.i0 + 1]);
}

// transform_from (basics/bbox.hpp:638-669).
std::vector<Box> transform_from(const std::vector<Box>& bbs_in, const M44* xs, int tcount) {
	std::vector<Box> bbs = bbs_in;
	if (tcount == 0) {
	} else if ((int)bbs.size() == tcount) {
		for (size_t i = 0; i < bbs.size(); ++i) bbs[i] = box_inverse_transformed(bbs[i], xs[i], host_rcp().table());
	} else if ((int)bbs.size() > tcount) {
		const float s = (float)(bbs.size() - 1);
		for (size_t i = 0; i < bbs.size(); ++i)
			bbs[i] = box_inverse_transformed(bbs[i], lerp_seq_m44((float)i / s, xs, tcount), host_rcp().table());
	} else {
		const float s = (float)(tcount - 1);
		std::vector<Box> t;
		for (int i = 0; i < tcount; ++i)
			t.push_back(box_inverse_transformed(lerp_seq_box((float)i / s, bbs), xs[i], host_rcp().table()));
		bbs = std::move(t);
	}
	return bbs;
}

// merge of bbox time sequences (basics/bbox.hpp:615-635).
std::vector<Box> merge_boxes(const std::vector<Box>& a, const std::vector<Box>& b) {
	std::vector<Box> c;
	if (a.empty()) {
		c = b;
	} else if (b.empty()) {
		c = a;
	} else if (a.size() == b.size()) {
		for (size_t i = 0; i < a.size(); ++i) c.push_back(box_union(a[i], b[i]));
	} else if (a.size() > b.size()) {
		const float s = (float)(a.size() - 1);
		for (size_t i = 0; i < a.size(); ++i) c.push_back(box_union(a[i], lerp_seq_box((float)i / s, b)));
	} else {
		const float s = (float)(b.size() - 1);
		for (size_t i = 0; i < b.size(); ++i) c.push_back(box_union(b[i], lerp_seq_box((float)i / s, a)));
	}
	return c;
}

// Colour energy (Color::energy, color/color.hpp:387-393).
float colour_energy(const float* c) {
	float acc = 0.0f;
	acc += c[0];
	acc += c[1];
	acc += c[2];
	acc /= 3.0f;
	return acc;
}

struct HObject {
	int kind = 0;
	std::vector<Box> bounds;
	float emit[3] = {0, 0, 0};  // total_emitted_color
};

struct HAssembly {
	const psy_assembly_desc* d = nullptr;
	std::vector<int> objects;     // global object index per local object
	std::vector<M44> xforms;
	std::vector<int> children;    // global assembly index per child slot
	// results
	std::vector<Box> accel_bounds{box_empty()};
	std::vector<Box> light_bounds{box_empty()};
	uint32_t light_count = 0;
	float light_energy = 0.0f;
	bool finalized = false;
};

struct Builder {
	const psy_scene_desc* desc;
	BuiltScene* out;
	std::string* err;
	bool gpu_root_bvh = false;
	std::vector<HObject> objs;
	std::vector<HAssembly> asms;
	std::vector<int> asm_inst_base;
	std::vector<int> asm_xform_base;

	bool fail(const std::string& m) {
		*err = m;
		return false;
	}

	// ---------------------------------------------------------------
	bool load_objects() {
		for (uint32_t a = 0; a < desc->assembly_count; ++a) {
			const psy_assembly_desc& ad = desc->assemblies[a];
			HAssembly& ha = asms[a];
			ha.d = &ad;
			if (ad.object_count && !ad.objects) return fail("assembly objects pointer is NULL");
			for (uint32_t i = 0; i < ad.object_count; ++i) {
				const psy_object_desc& od = ad.objects[i];
				HObject ho;
				ho.kind = (int)od.kind;
				DevObject dob{};
				dob.kind = (int)od.kind;
				dob.n0 = (int)od.n0;
				dob.n1 = (int)od.n1;
				dob.n2 = (int)od.n2;
				dob.data = (int)out->fpool.size();
				size_t nfl = 0;
				switch (od.kind) {
					case PSY_OBJ_SPHERE: nfl = (size_t)od.n0 * 4; break;
					case PSY_OBJ_BILINEAR: nfl = (size_t)od.n0 * 12; break;
					case PSY_OBJ_BICUBIC: nfl = (size_t)od.n0 * 48; break;
					case PSY_OBJ_SPHERE_LIGHT: nfl = (size_t)od.n0 * 3 + od.n1 + (size_t)od.n2 * 3; break;
					case PSY_OBJ_RECT_LIGHT: nfl = (size_t)od.n0 * 2 + (size_t)od.n1 * 3; break;
					default: return fail("unknown object kind " + std::to_string(od.kind));
				}
				if (od.n0 == 0) return fail("object with zero time samples");
				if (od.kind == PSY_OBJ_SPHERE_LIGHT && (od.n1 == 0 || od.n2 == 0))
					return fail("sphere light needs at least one radius and one colour");
				if (od.kind == PSY_OBJ_RECT_LIGHT && od.n1 == 0) return fail("rectangle light needs at least one colour");
				if (!od.data) return fail("object data pointer is NULL");
				for (size_t k = 0; k < nfl; ++k) {
					if (!std::isfinite(od.data[k])) return fail("non-finite object data");
				}
				out->fpool.insert(out->fpool.end(), od.data, od.data + nfl);
				const float* p = od.data;
				if (od.kind == PSY_OBJ_SPHERE) {
					for (uint32_t t = 0; t < od.n0; ++t) {
						const float* s = p + t * 4;
						Box b;
						b.lo = V3(s[0] - s[3], s[1] - s[3], s[2] - s[3]);
						b.hi = V3(s[0] + s[3], s[1] + s[3], s[2] + s[3]);
						ho.bounds.push_back(b);
					}
				} else if (od.kind == PSY_OBJ_BILINEAR || od.kind == PSY_OBJ_BICUBIC) {
					const int nv = od.kind == PSY_OBJ_BILINEAR ? 4 : 16;
					for (uint32_t t = 0; t < od.n0; ++t) {
						const float* v = p + t * nv * 3;
						Box b;
						b.lo = b.hi = V3(v[0], v[1], v[2]);
						for (int k = 1; k < nv; ++k) {
							const V3 q(v[k * 3], v[k * 3 + 1], v[k * 3 + 2]);
							b.lo = vmin3(b.lo, q);
							b.hi = vmax3(b.hi, q);
						}
						// Config::displace_distance (0.0) widening, kept for the arithmetic.
						for (int k = 0; k < 3; ++k) {
							b.lo.at(k) -= 0.0f;
							b.hi.at(k) += 0.0f;
						}
						ho.bounds.push_back(b);
					}
				} else if (od.kind == PSY_OBJ_RECT_LIGHT) {
					// RectangleLight's bounds (lights/rectangle_light.hpp:28-35):
					// the rectangle in its xy plane, one box per dimension sample
					for (uint32_t t = 0; t < od.n0; ++t) {
						const V3 dim3(p[t * 2] * 0.5f, p[t * 2 + 1] * 0.5f, 0.0f);
						Box b;
						b.lo = V3(0.0f) - dim3;
						b.hi = V3(0.0f) + dim3;
						ho.bounds.push_back(b);
					}
					// total_emitted_color = lerp_seq(0, colours) = the first colour
					const float* col = p + od.n0 * 2;
					for (int k = 0; k < 3; ++k) ho.emit[k] = col[k];
					if (od.n1 > 1) {
						for (int k = 0; k < 3; ++k) ho.emit[k] = (col[k] * one_minus(0.0f)) + (col[3 + k] * 0.0f);
					}
				} else {
					std::vector<V3> pos;
					std::vector<float> rad;
					for (uint32_t t = 0; t < od.n0; ++t) pos.push_back(V3(p[t * 3], p[t * 3 + 1], p[t * 3 + 2]));
					for (uint32_t t = 0; t < od.n1; ++t) rad.push_back(p[od.n0 * 3 + t]);
					const float* col = p + od.n0 * 3 + od.n1;
					if (pos.size() >= rad.size()) {
						const float s = (float)std::max<size_t>(pos.size() - 1, 1);
						for (size_t i = 0; i < pos.size(); ++i) {
							const float r = lerp_seq_f((float)i / s, rad);
							Box b;
							b.lo = pos[i] - V3(r);
							b.hi = pos[i] + V3(r);
							ho.bounds.push_back(b);
						}
					} else {
						const float s = (float)std::max<size_t>(rad.size() - 1, 1);
						for (size_t i = 0; i < rad.size(); ++i) {
							const V3 q = lerp_seq_v3((float)i / s, pos);
							Box b;
							b.lo = q - V3(rad[i]);
							b.hi = q + V3(rad[i]);
							ho.bounds.push_back(b);
						}
					}
					// total_emitted_color = lerp_seq(0, colours) = the first colour
					for (int k = 0; k < 3; ++k) ho.emit[k] = col[k];
					if (od.n2 > 1) {
						for (int k = 0; k < 3; ++k) ho.emit[k] = (col[k] * one_minus(0.0f)) + (col[3 + k] * 0.0f);
					}
				}
				ha.objects.push_back((int)objs.size());
				objs.push_back(ho);
				out->objects.push_back(dob);
			}
		}
		return true;
	}

	// ---------------------------------------------------------------
	bool load_structure() {
		// parent check: the assembly graph must be a tree rooted at 0
		std::vector<int> parent(desc->assembly_count, -1);
		for (uint32_t a = 0; a < desc->assembly_count; ++a) {
			const psy_assembly_desc& ad = desc->assemblies[a];
			if (ad.child_count && !ad.children) return fail("assembly children pointer is NULL");
			for (uint32_t c = 0; c < ad.child_count; ++c) {
				const uint32_t ch = ad.children[c];
				if (ch == 0 || ch >= desc->assembly_count) return fail("bad child assembly index");
				if (parent[ch] != -1) return fail("assembly has two parents");
				parent[ch] = (int)a;
				asms[a].children.push_back((int)ch);
			}
			if (ad.transform_count && !ad.transforms) return fail("assembly transforms pointer is NULL");
			for (uint32_t t = 0; t < ad.transform_count; ++t) {
				for (int k = 0; k < 16; ++k)
					if (!std::isfinite(ad.transforms[t * 16 + k])) return fail("non-finite transform");
				asms[a].xforms.push_back(load_m44(ad.transforms + t * 16));
			}
			if (ad.instance_count && !ad.instances) return fail("assembly instances pointer is NULL");
			for (uint32_t i = 0; i < ad.instance_count; ++i) {
				const psy_instance_desc& id = ad.instances[i];
				if (id.kind == PSY_INSTANCE_OBJECT) {
					if (id.data_index >= ad.object_count) return fail("instance object index out of range");
				} else if (id.kind == PSY_INSTANCE_ASSEMBLY) {
					if (id.data_index >= ad.child_count) return fail("instance assembly slot out of range");
				} else {
					return fail("unknown instance kind");
				}
				if ((uint64_t)id.transform_index + id.transform_count > ad.transform_count)
					return fail("instance transforms out of range");
				if (id.shader < -1 || id.shader >= (int32_t)desc->shader_count) return fail("instance shader out of range");
			}
		}
		for (uint32_t a = 1; a < desc->assembly_count; ++a)
			if (parent[a] == -1) return fail("assembly " + std::to_string(a) + " is not reachable from the root");
		return true;
	}

	// ---------------------------------------------------------------
	std::vector<Box> child_bounds_of(const HAssembly& ha, uint32_t i) {
		const psy_instance_desc& id = ha.d->instances[i];
		if (id.kind == PSY_INSTANCE_OBJECT) return objs[ha.objects[id.data_index]].bounds;
		return asms[ha.children[id.data_index]].accel_bounds;
	}

	// Assembly::instance_bounds (scene/assembly.hpp:261-281).
	std::vector<Box> instance_bounds(const HAssembly& ha, uint32_t i) {
		const psy_instance_desc& id = ha.d->instances[i];
		std::vector<Box> bbs = child_bounds_of(ha, i);
		return transform_from(bbs, ha.xforms.data() + id.transform_index, (int)id.transform_count);
	}

	// Assembly::instance_bounds_at (scene/assembly.hpp:288-312).
	Box instance_bounds_at(const HAssembly& ha, float t, uint32_t i) {
		const psy_instance_desc& id = ha.d->instances[i];
		Box bb = lerp_seq_box(t, child_bounds_of(ha, i));
		if (id.transform_count > 0)
			bb = box_inverse_transformed(bb, lerp_seq_m44(t, ha.xforms.data() + id.transform_index, (int)id.transform_count),
			                             host_rcp().table());
		return bb;
	}

	M44 instance_xform_at(const HAssembly& ha, float t, uint32_t i) {
		const psy_instance_desc& id = ha.d->instances[i];
		if (id.transform_count > 0) return lerp_seq_m44(t, ha.xforms.data() + id.transform_index, (int)id.transform_count);
		return m44_identity();
	}

	// ---------------------------------------------------------------
	// Binary BVH (accel/bvh.cpp)
	struct BNode {
		size_t bbox_index = 0;
		size_t child_or_data = 0;
		size_t parent_index = 0;
		uint16_t ts = 0;
		uint16_t flags = 0;
	};
	struct BPrim {
		size_t instance;
		V3 c;
		Box bb;  // bounds over all time samples (surface-area split only)
	};
	enum { IS_LEAF = 1 << 0, IS_SKIP = 1 << 8, IS_2ND = 1 << 9, IS_3RD = 1 << 10, IS_4TH = 1 << 11 };

	struct BVHBuild {
		std::vector<BNode> nodes;
		std::vector<Box> bboxes;
		std::vector<BPrim> bag;
		bool sah = false;  // surface-area split (device tree) instead of the reference's midpoint split
	};

	static float half_area(const Box& b) {
		const float dx = b.hi.x - b.lo.x, dy = b.hi.y - b.lo.y, dz = b.hi.z - b.lo.z;
		if (!(dx >= 0.0f && dy >= 0.0f && dz >= 0.0f)) return 0.0f;
		return dx * dy + dy * dz + dz * dx;
	}

	// Binned surface-area split (16 bins per axis over the centroid extent).
	// Returns the last index of the left part, or first - 1 when no bin
	// boundary separates the primitives (the caller then takes the midpoint
	// split).
	size_t sah_split(BVHBuild& b, size_t first, size_t last) {
		constexpr int NB = 16;
		V3 mn = b.bag[first].c, mx = b.bag[first].c;
		for (size_t i = first + 1; i <= last; ++i)
			for (int d = 0; d < 3; ++d) {
				const float c = b.bag[i].c[d];
				mn.at(d) = std::min(mn[d], c);
				mx.at(d) = std::max(mx[d], c);
			}
		auto bin_of = [&](const BPrim& p, int axis) {
			const float ext = mx[axis] - mn[axis];
			int k = (int)((p.c[axis] - mn[axis]) / ext * (float)NB);
			return k < 0 ? 0 : (k >= NB ? NB - 1 : k);
		};
		double best = INFINITY;
		int best_axis = -1, best_bin = -1;
		for (int axis = 0; axis < 3; ++axis) {
			if (!(mx[axis] - mn[axis] > 0.0f)) continue;
			Box bins[NB];
			size_t cnt[NB] = {0};
			for (int k = 0; k < NB; ++k) bins[k] = box_empty();
			for (size_t i = first; i <= last; ++i) {
				const int k = bin_of(b.bag[i], axis);
				bins[k] = box_union(bins[k], b.bag[i].bb);
				++cnt[k];
			}
			double right_area[NB];
			size_t right_cnt[NB];
			Box acc = box_empty();
			size_t n = 0;
			for (int k = NB - 1; k >= 0; --k) {
				acc = box_union(acc, bins[k]);
				n += cnt[k];
				right_area[k] = half_area(acc);
				right_cnt[k] = n;
			}
			acc = box_empty();
			n = 0;
			for (int k = 0; k < NB - 1; ++k) {
				acc = box_union(acc, bins[k]);
				n += cnt[k];
				if (n == 0 || right_cnt[k + 1] == 0) continue;
				const double cost = half_area(acc) * (double)n + right_area[k + 1] * (double)right_cnt[k + 1];
				if (cost < best) {
					best = cost;
					best_axis = axis;
					best_bin = k;
				}
			}
		}
		if (best_axis < 0) return first - 1;
		auto mid = std::partition(b.bag.begin() + first, b.bag.begin() + last + 1,
		                          [&](const BPrim& p) { return bin_of(p, best_axis) <= best_bin; });
		return (size_t)(mid - b.bag.begin()) - 1;
	}

	size_t split_primitives(BVHBuild& b, size_t first, size_t last) {
		if (b.sah) {
			const size_t s = sah_split(b, first, last);
			if (s + 1 > first && s < last) return s;
		}
		V3 mn = b.bag[first].c, mx = b.bag[first].c;
		for (size_t i = first + 1; i <= last; ++i) {
			for (int d = 0; d < 3; ++d) {
				const float c = b.bag[i].c[d];
				mn.at(d) = mn[d] < c ? mn[d] : c;
				mx.at(d) = mx[d] > c ? mx[d] : c;
			}
		}
		int axis = 0;
		if ((mx.y - mn.y) > (mx.x - mn.x)) axis = 1;
		if ((mx.z - mn.z) > (mx.y - mn.y)) axis = 2;
		const float pmid = .5f * (mn[axis] + mx[axis]);
		size_t split = bidir_partition(b.bag, first, last + 1, [axis, pmid](const BPrim& p) { return p.c[axis] < pmid; });
		if (split > 0) split--;
		if (split < first) split = first;
		return split;
	}

	size_t bvh_recursive(BVHBuild& b, const HAssembly& ha, size_t parent, size_t first, size_t last) {
		const size_t me = b.nodes.size();
		b.nodes.push_back(BNode());
		b.nodes[me].flags = 0;
		b.nodes[me].parent_index = parent;
		if (first == last) {
			b.nodes[me].flags |= IS_LEAF;
			b.nodes[me].child_or_data = b.bag[first].instance;
			const std::vector<Box> bbs = instance_bounds(ha, (uint32_t)b.bag[first].instance);
			b.nodes[me].bbox_index = b.bboxes.size();
			b.nodes[me].ts = (uint16_t)bbs.size();
			b.bboxes.insert(b.bboxes.end(), bbs.begin(), bbs.end());
		} else {
			const size_t split = split_primitives(b, first, last);
			const size_t c1 = bvh_recursive(b, ha, me, first, split);
			const size_t c2 = bvh_recursive(b, ha, me, split + 1, last);
			b.nodes[me].child_or_data = c2;
			b.nodes[me].bbox_index = b.bboxes.size();
			if (b.nodes[c1].ts == b.nodes[c2].ts) {
				b.nodes[me].ts = b.nodes[c1].ts;
				for (size_t i = 0; i < b.nodes[me].ts; ++i) {
					Box m = b.bboxes[b.nodes[c1].bbox_index + i];
					m = box_union(m, b.bboxes[b.nodes[c2].bbox_index + i]);
					b.bboxes.push_back(m);
				}
			} else {
				b.nodes[me].ts = 1;
				Box m = b.bboxes[b.nodes[c1].bbox_index];
				for (size_t i = 1; i < b.nodes[c1].ts; ++i) m = box_union(m, b.bboxes[b.nodes[c1].bbox_index + i]);
				for (size_t i = 0; i < b.nodes[c2].ts; ++i) m = box_union(m, b.bboxes[b.nodes[c2].bbox_index + i]);
				b.bboxes.push_back(m);
			}
		}
		return me;
	}

	// BBox4 record (the reference's 6 x float4 SoA).
	struct Rec4 {
		float b[24];
		uint64_t child[3] = {0, 0, 0};
		uint32_t ts = 0;
		uint64_t data = 0;
		bool leaf_data = false;
		Rec4() {
			for (int i = 0; i < 24; ++i) b[i] = ((i / 4) % 2 == 0) ? INFINITY : -INFINITY;
		}
		void set(const Box* bb, int n) {
			for (int c = 0; c < 4; ++c) {
				const Box x = c < n ? bb[c] : box_empty();
				b[0 * 4 + c] = x.lo.x;
				b[1 * 4 + c] = x.hi.x;
				b[2 * 4 + c] = x.lo.y;
				b[3 * 4 + c] = x.hi.y;
				b[4 * 4 + c] = x.lo.z;
				b[5 * 4 + c] = x.hi.z;
			}
		}
	};

	// BVH4::build packing (accel/bvh4.cpp:17-159).  With device == false the
	// reference's tree (midpoint splits) is built for the reference-form dump
	// and the assembly's bounds; with device == true a surface-area-split tree
	// of the same form is built for traversal.  Which valid tree is traversed
	// does not change a ray's closest hit, only the order candidates are met
	// (exact ties aside), and the surface-area tree visits fewer nodes.
	void build_bvh4(HAssembly& ha, int aidx, bool device) {
		BVHBuild b;
		b.sah = device;
		const uint32_t n_inst = ha.d->instance_count;
		for (uint32_t i = 0; i < n_inst; ++i) {
			const Box bb = instance_bounds_at(ha, 0.5f, i);
			BPrim p;
			p.instance = i;
			p.c = lerp3(0.5f, bb.lo, bb.hi);
			p.bb = box_empty();
			if (device)
				for (const Box& x : instance_bounds(ha, i)) p.bb = box_union(p.bb, x);
			b.bag.push_back(p);
		}
		RefBVH4& ref = out->ref_bvh4[aidx];
		DevAssembly& da = out->assemblies[aidx];
		if (device) da.root = REF_EMPTY;
		if (b.bag.empty()) {
			if (!device) ha.accel_bounds = {box_empty()};
			return;
		}
		bvh_recursive(b, ha, 0, 0, b.bag.size() - 1);

		std::vector<Rec4> recs;
		recs.push_back(Rec4());
		for (size_t bni = 0; bni < b.nodes.size(); ++bni) {
			BNode& bn = b.nodes[bni];
			const size_t ni = recs.size() - 1;
			if (bn.flags & IS_SKIP) continue;
			if (bn.flags & IS_2ND) recs[bn.parent_index].child[0] = ni;
			else if (bn.flags & IS_3RD) recs[bn.parent_index].child[1] = ni;
			else if (bn.flags & IS_4TH) recs[bn.parent_index].child[2] = ni;
			if (bn.flags & IS_LEAF) {
				recs[ni].child[0] = 0;
				recs[ni].data = bn.child_or_data;
				recs[ni].leaf_data = true;
				recs.push_back(Rec4());
			} else {
				int cc = 0;
				BNode* ch[4] = {nullptr, nullptr, nullptr, nullptr};
				const size_t ci1 = bni + 1;
				const size_t ci2 = bn.child_or_data;
				for (size_t ci : {ci1, ci2}) {
					if (b.nodes[ci].flags & IS_LEAF) {
						ch[cc++] = &b.nodes[ci];
					} else {
						b.nodes[ci].flags |= IS_SKIP;
						ch[cc++] = &b.nodes[ci + 1];
						ch[cc++] = &b.nodes[b.nodes[ci].child_or_data];
					}
				}
				if (ch[1]) ch[1]->flags |= IS_2ND;
				if (ch[2]) ch[2]->flags |= IS_3RD;
				if (ch[3]) ch[3]->flags |= IS_4TH;
				for (int i = 0; i < cc; ++i) ch[i]->parent_index = ni;
				bool equal_ts = true;
				int most = ch[0]->ts;
				for (int i = 1; i < cc; ++i) {
					equal_ts = equal_ts && (ch[i - 1]->ts == ch[i]->ts);
					if (ch[i]->ts > most) most = ch[i]->ts;
				}
				if (equal_ts) {
					recs[ni].ts = ch[0]->ts;
					for (uint16_t i = 0; i < ch[0]->ts; ++i) {
						Box bb[4];
						for (int c = 0; c < cc; ++c) bb[c] = b.bboxes[ch[c]->bbox_index + i];
						recs.back().set(bb, cc);
						recs.push_back(Rec4());
					}
				} else {
					recs[ni].ts = most;
					const float s = (float)(most - 1);
					for (uint16_t i = 0; i < most; ++i) {
						Box bb[4];
						for (int c = 0; c < cc; ++c) {
							if (ch[c]->ts == most) {
								bb[c] = b.bboxes[ch[c]->bbox_index + i];
							} else {
								std::vector<Box> seq(b.bboxes.begin() + ch[c]->bbox_index,
								                     b.bboxes.begin() + ch[c]->bbox_index + ch[c]->ts);
								bb[c] = lerp_seq_box((float)i / s, seq);
							}
						}
						recs.back().set(bb, cc);
						recs.push_back(Rec4());
					}
				}
			}
		}
		recs.pop_back();
		if (!device) {
			ha.accel_bounds.assign(b.bboxes.begin() + b.nodes[0].bbox_index,
			                       b.bboxes.begin() + b.nodes[0].bbox_index + b.nodes[0].ts);
			dump_ref(recs, ref);
			return;
		}
		emit_device(recs, da);
	}

	// The reference-form record dump (BVH4::Node, accel/bvh4.hpp:39-71).
	void dump_ref(const std::vector<Rec4>& recs, RefBVH4& ref) {
		for (const Rec4& r : recs) {
			float bb[24];
			std::memcpy(bb, r.b, sizeof(bb));
			if (r.leaf_data) std::memcpy(bb, &r.data, sizeof(uint64_t));  // the union's integer view
			ref.bounds.insert(ref.bounds.end(), bb, bb + 24);
			ref.child.insert(ref.child.end(), r.child, r.child + 3);
			ref.ts.push_back(r.ts);
			ref.data_index.push_back(r.leaf_data ? r.data : 0);
		}
	}

	// Device nodes: one DevNode per inner record group.
	void emit_device(const std::vector<Rec4>& recs, DevAssembly& da) {
		std::vector<int> dev_of(recs.size(), -1);
		for (size_t i = 0; i < recs.size();) {
			if (recs[i].leaf_data) {
				++i;
				continue;
			}
			dev_of[i] = (int)out->nodes.size();
			out->nodes.push_back(DevNode());
			i += std::max<uint32_t>(recs[i].ts, 1);
		}
		auto ref_of = [&](size_t ri) -> int {
			if (recs[ri].leaf_data) return leaf_ref((int)recs[ri].data);
			return dev_of[ri];
		};
		for (size_t i = 0; i < recs.size();) {
			if (recs[i].leaf_data) {
				++i;
				continue;
			}
			DevNode& dn = out->nodes[dev_of[i]];
			std::memset(&dn, 0, sizeof(dn));
			const Rec4& r = recs[i];
			const int nch = r.child[1] == 0 ? 2 : (r.child[2] == 0 ? 3 : 4);
			dn.nchild = nch;
			dn.ts = (int)r.ts;
			std::memcpy(dn.b, r.b, sizeof(dn.b));
			dn.child[0] = ref_of(i + r.ts);
			for (int c = 1; c < nch; ++c) dn.child[c] = ref_of(r.child[c - 1]);
			for (int c = nch; c < 4; ++c) dn.child[c] = REF_EMPTY;
			dn.extra = (int)(out->node_extra.size() / 24);
			for (uint32_t t = 1; t < r.ts; ++t) out->node_extra.insert(out->node_extra.end(), recs[i + t].b, recs[i + t].b + 24);
			i += std::max<uint32_t>(r.ts, 1);
		}
		da.root = ref_of(0);
	}

	// ---------------------------------------------------------------
	// Light tree (accel/light_tree.cpp:99-238)
	struct LBuild {
		size_t instance;
		V3 center;
		Box bbox;
		float energy;
	};
	struct LNode {
		std::vector<Box> bounds;
		float energy = 0.0f;
		size_t i1 = 0, i2 = 0;
		bool leaf = false;
		size_t instance = 0;
	};

	size_t light_split(std::vector<LBuild>& v, size_t start, size_t end) {
		V3 mn = v[start].center, mx = v[start].center;
		for (size_t i = start + 1; i < end; ++i) {
			for (int d = 0; d < 3; ++d) {
				const float c = v[i].center[d];
				mn.at(d) = mn[d] < c ? mn[d] : c;
				mx.at(d) = mx[d] > c ? mx[d] : c;
			}
		}
		int axis = 0;
		if ((mx.y - mn.y) > (mx.x - mn.x)) axis = 1;
		if ((mx.z - mn.z) > (mx.y - mn.y)) axis = 2;
		const float pmid = .5f * (mn[axis] + mx[axis]);
		size_t mid = bidir_partition(v, start, end, [axis, pmid](const LBuild& b) { return b.center[axis] < pmid; });
		if (mid == start) mid++;
		return mid;
	}

	size_t light_recursive(std::vector<LNode>& nodes, std::vector<LBuild>& v, const HAssembly& ha, size_t start,
	                       size_t end) {
		const size_t me = nodes.size();
		nodes.push_back(LNode());
		if (start + 1 == end) {
			const psy_instance_desc& id = ha.d->instances[v[start].instance];
			nodes[me].leaf = true;
			nodes[me].instance = v[start].instance;
			if (id.kind == PSY_INSTANCE_OBJECT) {
				nodes[me].bounds = instance_bounds(ha, (uint32_t)v[start].instance);
			} else {
				const HAssembly& sub = asms[ha.children[id.data_index]];
				if (id.transform_count > 0)
					nodes[me].bounds = transform_from(sub.light_bounds, ha.xforms.data() + id.transform_index,
					                                  (int)id.transform_count);
				else
					nodes[me].bounds = sub.light_bounds;
			}
			nodes[me].energy = v[start].energy;
		} else {
			const size_t split = light_split(v, start, end);
			const size_t c1 = light_recursive(nodes, v, ha, start, split);
			const size_t c2 = light_recursive(nodes, v, ha, split, end);
			nodes[me].i1 = c1;
			nodes[me].i2 = c2;
			nodes[me].bounds = merge_boxes(nodes[c1].bounds, nodes[c2].bounds);
			nodes[me].energy = nodes[c1].energy + nodes[c2].energy;
		}
		return me;
	}

	// The assembly's lights as LightTree::build lists them (light_tree.cpp:
	// 99-150): emitting object instances and assembly instances with lights.
	void collect_lights(HAssembly& ha, std::vector<LBuild>& bn, uint32_t& total_lights) {
		total_lights = 0;
		for (uint32_t i = 0; i < ha.d->instance_count; ++i) {
			const psy_instance_desc& id = ha.d->instances[i];
			if (id.kind == PSY_INSTANCE_OBJECT) {
				const HObject& ob = objs[ha.objects[id.data_index]];
				const float e = colour_energy(ob.emit);
				if (e > 0.0f) {
					LBuild l;
					l.instance = i;
					l.bbox = instance_bounds_at(ha, 0.5f, i);
					l.center = box_center(l.bbox);
					const V3 s = inv_scale(instance_xform_at(ha, 0.5f, i));
					const float surface_scale = ((s.x * s.y) + (s.x * s.z) + (s.y * s.z)) * 0.33333333f;
					l.energy = e / surface_scale;
					bn.push_back(l);
					++total_lights;
				}
			} else {
				const HAssembly& sub = asms[ha.children[id.data_index]];
				const uint32_t count = sub.light_count;
				const float tot[3] = {sub.light_energy, sub.light_energy, sub.light_energy};
				const float e = colour_energy(tot);
				if (count > 0 && e > 0.0f) {
					LBuild l;
					l.instance = i;
					if (id.transform_count > 0)
						l.bbox = box_inverse_transformed(lerp_seq_box(0.5f, sub.light_bounds),
						                                 lerp_seq_m44(0.5f, ha.xforms.data() + id.transform_index,
						                                              (int)id.transform_count),
						                                 host_rcp().table());
					else
						l.bbox = lerp_seq_box(0.5f, sub.light_bounds);
					l.center = box_center(l.bbox);
					const V3 s = inv_scale(instance_xform_at(ha, 0.5f, i));
					const float surface_scale = ((s.x * s.y) + (s.x * s.z) + (s.y * s.z)) * 0.33333333f;
					l.energy = e / surface_scale;
					bn.push_back(l);
					total_lights += count;
				}
			}
		}
	}

	void build_light_tree(HAssembly& ha, int aidx) {
		std::vector<LBuild> bn;
		uint32_t total_lights = 0;
		collect_lights(ha, bn, total_lights);
		DevAssembly& da = out->assemblies[aidx];
		da.light_root = -1;
		da.light_count = (int)total_lights;
		ha.light_count = total_lights;
		if (bn.empty()) {
			ha.light_bounds = {box_empty()};
			ha.light_energy = 0.0f;
			da.light_energy = 0.0f;
			return;
		}
		std::vector<LNode> nodes;
		light_recursive(nodes, bn, ha, 0, bn.size());
		ha.light_bounds = nodes[0].bounds;
		ha.light_energy = nodes[0].energy;
		da.light_energy = nodes[0].energy;
		const int base = (int)out->light_nodes.size();
		da.light_root = base;
		for (const LNode& ln : nodes) {
			DevLightNode dl{};
			const Box b0 = ln.bounds.empty() ? box_empty() : ln.bounds[0];
			dl.lo[0] = b0.lo.x; dl.lo[1] = b0.lo.y; dl.lo[2] = b0.lo.z;
			dl.hi[0] = b0.hi.x; dl.hi[1] = b0.hi.y; dl.hi[2] = b0.hi.z;
			dl.energy = ln.energy;
			dl.ts = (int)ln.bounds.size();
			dl.extra = (int)(out->light_extra.size() / 6);
			for (size_t t = 1; t < ln.bounds.size(); ++t) {
				const Box& b = ln.bounds[t];
				const float f[6] = {b.lo.x, b.lo.y, b.lo.z, b.hi.x, b.hi.y, b.hi.z};
				out->light_extra.insert(out->light_extra.end(), f, f + 6);
			}
			dl.is_leaf = ln.leaf ? 1 : 0;
			dl.c1 = ln.leaf ? (int)ln.instance : base + (int)ln.i1;
			dl.c2 = ln.leaf ? 0 : base + (int)ln.i2;
			out->light_nodes.push_back(dl);
		}
	}

	// The lights of the root for the device build of its light tree, when
	// it has two or more and each light has bounds; false otherwise.
	bool light_tree_for_gpu(HAssembly& ha, int aidx) {
		std::vector<LBuild> bn;
		uint32_t total_lights = 0;
		collect_lights(ha, bn, total_lights);
		if (bn.size() < 2) return false;
		std::vector<float> el, samples;
		std::vector<int> first{0};
		el.reserve(bn.size() * 5);
		for (const LBuild& l : bn) {
			const psy_instance_desc& id = ha.d->instances[l.instance];
			std::vector<Box> bb;
			if (id.kind == PSY_INSTANCE_OBJECT) {
				bb = instance_bounds(ha, (uint32_t)l.instance);
			} else {
				const HAssembly& sub = asms[ha.children[id.data_index]];
				bb = id.transform_count > 0 ? transform_from(sub.light_bounds, ha.xforms.data() + id.transform_index,
				                                             (int)id.transform_count)
				                            : sub.light_bounds;
			}
			if (bb.empty() || bb.size() > 64 || l.instance >= (1u << 24)) return false;
			el.insert(el.end(), {l.center.x, l.center.y, l.center.z, l.energy, (float)l.instance});
			for (const Box& b : bb) samples.insert(samples.end(), {b.lo.x, b.lo.y, b.lo.z, b.hi.x, b.hi.y, b.hi.z});
			first.push_back(first.back() + (int)bb.size());
		}
		out->gpu_light_elems.swap(el);
		out->gpu_light_samples.swap(samples);
		out->gpu_light_first.swap(first);
		out->gpu_light_pending = true;
		DevAssembly& da = out->assemblies[aidx];
		da.light_root = -1;  // set by the device build
		da.light_count = (int)total_lights;
		ha.light_count = total_lights;
		return true;
	}

	// ---------------------------------------------------------------
	// The root's leaf bounds for the device build (every time sample), when
	// every root instance has bounds; false otherwise.
	bool root_leaves_for_gpu(HAssembly& ha) {
		std::vector<float> boxes, centres;
		std::vector<int> first{0};
		for (uint32_t i = 0; i < ha.d->instance_count; ++i) {
			const std::vector<Box> bbs = instance_bounds(ha, i);
			if (bbs.empty() || bbs.size() > 64) return false;
			for (const Box& b : bbs) boxes.insert(boxes.end(), {b.lo.x, b.lo.y, b.lo.z, b.hi.x, b.hi.y, b.hi.z});
			first.push_back(first.back() + (int)bbs.size());
			// the centre build_bvh4 splits on
			const Box bh = instance_bounds_at(ha, 0.5f, i);
			const V3 c = lerp3(0.5f, bh.lo, bh.hi);
			centres.insert(centres.end(), {c.x, c.y, c.z});
		}
		out->gpu_leaf_boxes.swap(boxes);
		out->gpu_leaf_first.swap(first);
		out->gpu_leaf_centres.swap(centres);
		out->gpu_root_pending = true;
		out->assemblies[0].root = REF_EMPTY;
		return true;
	}

	int finalize(int a, int depth) {
		HAssembly& ha = asms[a];
		int maxd = depth;
		for (int c : ha.children) maxd = std::max(maxd, finalize(c, depth + 1));
		// the root is never instanced, so its reference-form tree (which gives
		// an assembly its bounds) is not needed when the device builds its
		// traversal tree
		// the root's light tree is left to the device build when asked for
		// and possible (the root is never instanced: nothing above it needs
		// its light bounds)
		const bool gpu_lights = a == 0 && gpu_root_bvh && light_tree_for_gpu(ha, a);
		if (a == 0 && gpu_root_bvh && root_leaves_for_gpu(ha)) {
			if (!gpu_lights) build_light_tree(ha, a);
			ha.finalized = true;
			return maxd;
		}
		build_bvh4(ha, a, false);
		build_bvh4(ha, a, true);
		if (!gpu_lights) build_light_tree(ha, a);
		ha.finalized = true;
		return maxd;
	}

	bool run() {
		if (!desc) return fail("scene description is NULL");
		if (desc->assembly_count == 0 || !desc->assemblies) return fail("scene has no root assembly");
		if (desc->cam_transform_count == 0 || !desc->cam_transforms) return fail("camera has no transform");
		if (desc->cam_fov_count == 0 || !desc->cam_fovs) return fail("camera has no fov");
		if (desc->shader_count && !desc->shaders) return fail("shaders pointer is NULL");
		asms.resize(desc->assembly_count);
		out->assemblies.assign(desc->assembly_count, DevAssembly());
		out->ref_bvh4.assign(desc->assembly_count, RefBVH4());
		if (!load_structure()) return false;
		if (!load_objects()) return false;
		// instance and transform tables
		for (uint32_t a = 0; a < desc->assembly_count; ++a) {
			const psy_assembly_desc& ad = desc->assemblies[a];
			DevAssembly& da = out->assemblies[a];
			std::memset(&da, 0, sizeof(da));
			da.inst_base = (int)out->instances.size();
			da.inst_count = (int)ad.instance_count;
			da.id_bits = (int)intlog2(upper_power_of_two(ad.instance_count));
			const int xbase = (int)(out->xforms.size() / 16);
			out->xforms.insert(out->xforms.end(), ad.transforms, ad.transforms + (size_t)ad.transform_count * 16);
			for (uint32_t i = 0; i < ad.instance_count; ++i) {
				const psy_instance_desc& id = ad.instances[i];
				DevInstance di{};
				di.kind = (int)id.kind;
				di.data = id.kind == PSY_INSTANCE_OBJECT ? asms[a].objects[id.data_index] : asms[a].children[id.data_index];
				di.xform = xbase + (int)id.transform_index;
				di.xform_count = (int)id.transform_count;
				di.shader = id.shader;
				out->instances.push_back(di);
			}
		}
		out->max_depth = finalize(0, 1);
		// kernel variant selection
		for (const DevInstance& di : out->instances) {
			if (di.kind == INST_ASSEMBLY) out->features |= FEAT_NESTED;
			if (di.xform_count > 0) out->features |= FEAT_XFORM;
		}
		for (const DevObject& ob : out->objects) {
			if (ob.kind == OBJ_BICUBIC) out->features |= FEAT_BICUBIC;
			if (ob.kind == OBJ_BILINEAR) out->features |= FEAT_BILINEAR;
			if ((ob.kind == OBJ_BILINEAR || ob.kind == OBJ_BICUBIC) && ob.n0 > 1) out->features |= FEAT_PATCH_MOTION;
			if ((ob.kind == OBJ_BILINEAR || ob.kind == OBJ_BICUBIC) && ob.n0 > 2) return fail("patches support at most two time samples");
		}
		out->total_lights = asms[0].light_count;
		for (uint32_t s = 0; s < desc->shader_count; ++s) {
			DevShader ds{};
			ds.kind = (int)desc->shaders[s].kind;
			for (int k = 0; k < 3; ++k) ds.col[k] = desc->shaders[s].color[k];
			ds.roughness = desc->shaders[s].roughness;
			ds.tail_shape = desc->shaders[s].tail_shape;
			ds.fresnel = desc->shaders[s].fresnel;
			if (ds.kind < 0 || ds.kind > 2) return fail("unknown shader kind");
			if (ds.kind == SHADER_GTR) {
				// GTRClosure::validate (shading/surface_closure.hpp:352-372)
				float r = std::max(0.0f, std::min(0.9999f, ds.roughness));
				float t = std::max(0.0001f, ds.tail_shape);
				if (r < 0.000244140625f) r = 0.0f;
				if (std::abs(t - 1.0f) < 0.0001f) t = 1.0f + 0.0001f;
				ds.roughness = r;
				ds.tail_shape = t;
				// GTRClosure::normalization (:374-380)
				const float r2 = r * r;
				const float top = (t - 1.0f) * (r2 - 1);
				const double bottom = M_PI * (double)(1.0f - std::pow(r2, 1.0f - t));
				ds.norm = (float)((double)top / bottom);
				ds.pow_r2_1mt = std::pow(r2, 1.0f - t);
			}
			out->shaders.push_back(ds);
		}
		// camera (basics/camera.hpp:28-64)
		out->cam_xforms.assign(desc->cam_transforms, desc->cam_transforms + (size_t)desc->cam_transform_count * 16);
		for (uint32_t i = 0; i < desc->cam_fov_count; ++i) {
			const float f = desc->cam_fovs[i];
			// float sinf/cosf, as the reference's unqualified sin/cos resolve to for a float
			out->cam_tfovs.push_back(std::sin(f / 2.0f) / std::cos(f / 2.0f));
		}
		bool focal = desc->cam_aperture_count > 0 && desc->cam_focus_count > 0;
		if (focal) {
			for (uint32_t i = 0; i < desc->cam_focus_count; ++i)
				if (desc->cam_focus_distances[i] <= 0.0f) focal = false;
		}
		if (focal) {
			out->cam_apertures.assign(desc->cam_aperture_radii, desc->cam_aperture_radii + desc->cam_aperture_count);
			out->cam_focus.assign(desc->cam_focus_distances, desc->cam_focus_distances + desc->cam_focus_count);
		} else {
			out->cam_apertures = {0.0f};
			out->cam_focus = {1.0f};
		}
		for (int k = 0; k < 3; ++k) out->background[k] = desc->background[k];
		out->dice_rate = desc->dice_rate;
		out->min_upoly_size = desc->min_upoly_size;
		return true;
	}
};

}  // namespace

int build_scene(const psy_scene_desc* desc, BuiltScene* out, std::string* err, bool gpu_root_bvh) {
	Builder b;
	b.desc = desc;
	b.out = out;
	b.err = err;
	b.gpu_root_bvh = gpu_root_bvh;
	return b.run() ? PSY_OK : PSY_ERR_ARG;
}

}  // namespace psy
