/*
 * Device scene layout (host + device).
 *
 * One flat set of arrays per uploaded scene, resident in HBM:
 *   assemblies[]   per-assembly roots and table bases
 *   instances[]    global instance table (all assemblies, contiguous per assembly)
 *   objects[]      global object table; geometry in the float pool
 *   nodes[]        BVH4 inner nodes, 128-byte records: the 4 child boxes of
 *                  time sample 0 as BBox4 SoA (xmin[4] xmax[4] ymin[4] ymax[4]
 *                  zmin[4] zmax[4], the reference's BBox4 layout,
 *                  basics/bbox.hpp:432-448) + child refs; further time
 *                  samples in node_extra[]
 *   xforms[]       16-float matrices, per assembly
 *   light_nodes[]  light-tree nodes
 *   shaders[]      surface shaders
 */
#ifndef PSY_SCENE_H
#define PSY_SCENE_H

#include <cstdint>

#include "psy_math.h"

namespace psy {

enum : int { OBJ_SPHERE = 0, OBJ_BILINEAR = 1, OBJ_BICUBIC = 2, OBJ_SPHERE_LIGHT = 3, OBJ_RECT_LIGHT = 4 };
enum : int { INST_OBJECT = 0, INST_ASSEMBLY = 1 };
enum : int { SHADER_LAMBERT = 0, SHADER_EMIT = 1, SHADER_GTR = 2 };
enum : int { CLOSURE_NONE = 0, CLOSURE_LAMBERT = 1, CLOSURE_EMIT = 2, CLOSURE_GTR = 3 };

// Device error flags, OR-ed into the context's status word by kernels.
enum : unsigned { ERRF_STACK = 1u, ERRF_LEVELS = 2u, ERRF_MOTION = 4u, ERRF_TIMEOUT = 8u, ERRF_NOLIGHT = 16u,
                  ERRF_BISECT = 32u /* a patch bisection exceeded its step bound */ };

// Scene features that select a compiled variant of the traversal kernels.
enum : unsigned {
	FEAT_NESTED = 1u,        // assembly instances (levels)
	FEAT_XFORM = 2u,         // instance transforms
	FEAT_BICUBIC = 4u,       // bicubic patches
	FEAT_PATCH_MOTION = 8u,  // patches with two time samples
	FEAT_BILINEAR = 16u,     // bilinear patches
	FEAT_FLAT = 16u,         // spheres, lights and bilinear patches in one level
	FEAT_STILL_BICUBIC = 7u, // levels, transforms, bicubic patches (no bilinear, no patch motion)
	FEAT_STILL = 23u,        // everything but patch motion
	FEAT_ALL = 31u
};

// The compiled variant that covers a scene's features (the smallest of
// FEAT_FLAT, FEAT_STILL_BICUBIC, FEAT_STILL, FEAT_ALL: smaller variants
// leave out the code of absent features).
inline unsigned feature_variant(unsigned f) {
	if ((f & ~FEAT_FLAT) == 0u) return FEAT_FLAT;
	if ((f & ~FEAT_STILL_BICUBIC) == 0u) return FEAT_STILL_BICUBIC;
	if ((f & ~FEAT_STILL) == 0u) return FEAT_STILL;
	return FEAT_ALL;
}

// A child reference in a BVH4 node or an assembly root:
//   >= 0          inner node index (global)
//   < 0, != EMPTY leaf: local instance index = -(ref + 1)
static constexpr int REF_EMPTY = (int)0x80000000;
PSY_HD int leaf_ref(int local_instance) { return -(local_instance + 1); }
PSY_HD int leaf_instance(int ref) { return -(ref + 1); }

struct alignas(16) DevNode {
	float b[24];      // time sample 0 child bounds, BBox4 SoA
	int child[4];     // child refs
	int nchild;       // 2..4
	int ts;           // time samples
	int extra;        // index of time sample 1 in node_extra (24 floats per sample)
	int pad;
};
static_assert(sizeof(DevNode) == 128, "DevNode must be 128 bytes");

struct alignas(16) DevInstance {
	int kind;         // INST_OBJECT / INST_ASSEMBLY
	int data;         // global object index or global assembly index
	int xform;        // global transform index of the first motion sample
	int xform_count;  // 0 = none
	int shader;       // -1 = none
	int pad[3];
};

struct alignas(16) DevObject {
	int kind;
	int n0, n1, n2;   // time-sample counts (sphere/patch: n0; light: positions, radii, colours)
	int data;         // float pool offset
	int pad[3];
};

struct alignas(16) DevAssembly {
	int root;         // BVH4 root ref
	int inst_base;    // first global instance
	int inst_count;
	int id_bits;      // Assembly::element_id_bits()
	int light_root;   // light-tree root node (global), -1 = no lights
	int light_count;  // LightTree::light_count()
	float light_energy;
	int pad;
};

struct alignas(16) DevLightNode {
	float lo[3], hi[3];  // bounds, time sample 0
	float energy;
	int ts;              // bounds time samples
	int extra;           // index of time sample 1 in light_extra (6 floats per sample)
	int is_leaf;
	int c1, c2;          // children (global) or, for leaves, c1 = local instance index
};

struct alignas(16) DevShader {
	int kind;
	float col[3];
	// GTR: the parameters as GTRClosure::validate leaves them
	// (shading/surface_closure.hpp:352-372), its normalisation factor, and
	// pow(roughness^2, 1 - tail_shape); both computed on the host with the
	// host's powf, as the reference computes them
	float roughness, tail_shape, fresnel, norm;
	float pow_r2_1mt;
	int pad[3];
};

// Device pointers of an uploaded scene, passed to kernels by value.
struct DevScene {
	const DevAssembly* assemblies;
	const DevInstance* instances;
	const DevObject* objects;
	const DevNode* nodes;
	const float* node_extra;
	const float* xforms;
	const float* fpool;
	const DevLightNode* light_nodes;
	const float* light_extra;
	const DevShader* shaders;
	int assembly_count;
	int max_depth;        // deepest assembly nesting (root = 1)
	unsigned features;    // FEAT_* present in the scene
	float dice_rate;
	float min_upoly_size;
	// camera
	const float* cam_xforms;
	const float* cam_tfovs;
	const float* cam_apertures;
	const float* cam_focus;
	int cam_xform_count, cam_tfov_count, cam_aperture_count, cam_focus_count;
	float background[3];
	int light_node_count;  // all assemblies' light nodes (bounds a tree walk)
	// the host CPU's approximate reciprocal (psy_math.h), for matrix inverses
	RcpTable rcp;
};

}  // namespace psy

#endif
