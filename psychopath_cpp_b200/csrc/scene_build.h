/*
 * Host-side scene preparation: the equivalent of Assembly::finalize
 * (reference scene/assembly.hpp:206-238) for a flattened scene description.
 */
#ifndef PSY_SCENE_BUILD_H
#define PSY_SCENE_BUILD_H

#include <string>
#include <vector>

#include "../../include/psy_b200.h"
#include "psy_scene.h"

namespace psy {

// BVH4 node records in the reference's own form (BVH4::Node, accel/bvh4.hpp:39-71),
// kept for inspection and parity tests of the builder.
struct RefBVH4 {
	std::vector<float> bounds;        // 24 per record
	std::vector<uint64_t> child;      // 3 per record
	std::vector<uint32_t> ts;
	std::vector<uint64_t> data_index;
};

struct BuiltScene {
	std::vector<DevAssembly> assemblies;
	std::vector<DevInstance> instances;
	std::vector<DevObject> objects;
	std::vector<DevNode> nodes;
	std::vector<float> node_extra;
	std::vector<float> xforms;
	std::vector<float> fpool;
	std::vector<DevLightNode> light_nodes;
	std::vector<float> light_extra;
	std::vector<DevShader> shaders;
	std::vector<float> cam_xforms, cam_tfovs, cam_apertures, cam_focus;
	float background[3] = {0, 0, 0};
	float dice_rate = 0.25f;
	float min_upoly_size = 0.00001f;
	int max_depth = 1;
	unsigned features = 0;  // FEAT_* present
	uint32_t total_lights = 0;
	std::vector<RefBVH4> ref_bvh4;    // per assembly
	// With gpu_root_bvh requested, the root's traversal BVH4 is left to the
	// device build: its instances' bounds (every time sample) are here, in
	// instance order, and assemblies[0].root stays REF_EMPTY until that
	// build sets it.
	bool gpu_root_pending = false;
	std::vector<float> gpu_leaf_boxes;    // every root instance's time samples: lo xyz, hi xyz
	std::vector<int> gpu_leaf_first;      // instance i's samples: [first[i], first[i + 1])
	std::vector<float> gpu_leaf_centres;  // per root instance: its box's centre at time 0.5
	// With gpu_root_bvh requested and a root with two or more lights, the
	// root's light tree is left to the device build: its lights in
	// LightTree::build's order, 5 floats each (centre xyz, energy, local
	// instance index), their bounds' time samples (6 floats each, light i's
	// are [first[i], first[i + 1])), and assemblies[0].light_root stays -1
	// until that build sets it.
	bool gpu_light_pending = false;
	std::vector<float> gpu_light_elems;
	std::vector<float> gpu_light_samples;
	std::vector<int> gpu_light_first;
};

// Validates the description and builds every assembly (children first).
// gpu_root_bvh: leave the root assembly's traversal tree and light tree to
// the device builds (see gpu_root_pending and gpu_light_pending).  Returns PSY_OK or
// PSY_ERR_ARG with *err set.
int build_scene(const psy_scene_desc* desc, BuiltScene* out, std::string* err, bool gpu_root_bvh = false);

}  // namespace psy

#endif
