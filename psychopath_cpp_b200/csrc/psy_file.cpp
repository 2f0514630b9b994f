/*
 * The .psy scene file reader: the reference's DataTree format (reference
 * parser/data_tree.cpp:177-400) and the reading of its Scene node into a
 * scene (parser/parser.cpp:37-662), flattened to the psy_scene_desc that
 * psy_scene_upload takes.
 *
 *   - tokens: TYPE identifiers, $names (backslash escapes), { } around a
 *     node's children, [ ] around a leaf's contents (backslash escapes,
 *     surrounding white space trimmed), # comments to the end of the line;
 *   - numbers are read from a leaf's contents as the reference reads them:
 *     every match of -?[0-9]+[.]?[0-9]* (integers: -?[0-9]+), converted by
 *     std::stof / std::stoi;
 *   - names as the reference's Assembly keeps them (scene/assembly.hpp:
 *     104-157): every definition is kept in order, and a name finds its
 *     first definition; names match as written, $ included;
 *   - an instance's shader is bound when the instance is read, to the
 *     shader of that name defined so far in its assembly or else in the
 *     enclosing ones (parser/parser.cpp:298-323, assembly.hpp:113-121);
 *   - where the reference prints an error and goes on (an instance of
 *     unknown data is dropped, an unknown shader binds none), the file is
 *     rejected instead;
 *   - the flattening: assemblies depth first in declaration order (the root
 *     first), objects and sub-assemblies in declaration order, shaders
 *     numbered in the order instances first bind them.
 */
#include <cctype>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <string>
#include <vector>

#include "../../include/psy_b200.h"

namespace {

struct Node {
	std::string type, name, leaf;
	bool is_leaf = false;
	std::vector<Node> children;
};

struct ParseError {
	std::string msg;
};

enum TokKind { T_OPEN, T_CLOSE, T_LEAF, T_NAME, T_TYPE };
struct Tok {
	TokKind kind;
	std::string text;
};

bool is_space(char c) { return std::isspace((unsigned char)c) != 0; }
bool is_break(char c) { return is_space(c) || std::strchr("{}[]#$", c) != nullptr; }

std::string trim(const std::string& s) {
	size_t a = 0, b = s.size();
	while (a < b && is_space(s[a])) ++a;
	while (b > a && is_space(s[b - 1])) --b;
	return s.substr(a, b - a);
}

std::vector<Tok> tokenize(const char* text, size_t n) {
	std::vector<Tok> toks;
	size_t i = 0;
	while (i < n) {
		const char c = text[i];
		if (is_space(c)) {
			++i;
		} else if (c == '#') {
			while (i < n && text[i] != '\n') ++i;
		} else if (c == '{' || c == '}') {
			toks.push_back({c == '{' ? T_OPEN : T_CLOSE, std::string(1, c)});
			++i;
		} else if (c == '[') {
			++i;
			std::string buf;
			while (i < n && text[i] != ']') {
				if (text[i] == '\\' && i + 1 < n) {
					buf += text[i + 1];
					i += 2;
				} else {
					buf += text[i++];
				}
			}
			if (i >= n) throw ParseError{"unterminated leaf contents"};
			++i;
			toks.push_back({T_LEAF, trim(buf)});
		} else if (c == '$') {
			std::string buf = "$";
			++i;
			while (i < n) {
				if (text[i] == '\\' && i + 1 < n) {
					buf += text[i + 1];
					i += 2;
				} else if (is_break(text[i])) {
					break;
				} else {
					buf += text[i++];
				}
			}
			toks.push_back({T_NAME, buf});
		} else {
			size_t j = i;
			while (j < n && !is_break(text[j])) ++j;
			if (j == i) throw ParseError{std::string("unexpected character '") + c + "'"};
			toks.push_back({T_TYPE, std::string(text + i, j - i)});
			i = j;
		}
	}
	return toks;
}

Node build_tree(const std::vector<Tok>& toks) {
	Node root;
	root.type = "ROOT";
	std::vector<Node*> stack{&root};
	size_t i = 0;
	while (i < toks.size()) {
		if (toks[i].kind == T_CLOSE) {
			if (stack.size() == 1) throw ParseError{"unbalanced '}'"};
			stack.pop_back();
			++i;
			continue;
		}
		if (toks[i].kind != T_TYPE) throw ParseError{"expected a type name, got '" + toks[i].text + "'"};
		Node node;
		node.type = toks[i].text;
		++i;
		if (i < toks.size() && toks[i].kind == T_NAME) node.name = toks[i++].text;
		if (i >= toks.size()) throw ParseError{"unexpected end of file after '" + node.type + "'"};
		if (toks[i].kind == T_LEAF) {
			node.is_leaf = true;
			node.leaf = toks[i++].text;
			stack.back()->children.push_back(std::move(node));
		} else if (toks[i].kind == T_OPEN) {
			++i;
			stack.back()->children.push_back(std::move(node));
			stack.push_back(&stack.back()->children.back());
		} else {
			throw ParseError{"expected '{' or '[' after '" + node.type + "'"};
		}
	}
	if (stack.size() != 1) throw ParseError{"unbalanced '{'"};
	return root;
}

// The matches of -?[0-9]+[.]?[0-9]* (with_fraction) or -?[0-9]+ in s, in
// order, as strings.
std::vector<std::string> number_matches(const std::string& s, bool with_fraction) {
	std::vector<std::string> out;
	size_t i = 0;
	const size_t n = s.size();
	while (i < n) {
		size_t j = i;
		if (s[j] == '-') ++j;
		if (j < n && std::isdigit((unsigned char)s[j])) {
			size_t k = j;
			while (k < n && std::isdigit((unsigned char)s[k])) ++k;
			if (with_fraction) {
				if (k < n && s[k] == '.') ++k;
				while (k < n && std::isdigit((unsigned char)s[k])) ++k;
			}
			out.push_back(s.substr(i, k - i));
			i = k;
		} else {
			++i;
		}
	}
	return out;
}

std::vector<float> floats(const std::string& s, size_t limit = (size_t)-1) {
	std::vector<float> v;
	for (const std::string& m : number_matches(s, true)) {
		if (v.size() >= limit) break;
		v.push_back(std::stof(m));
	}
	return v;
}

std::vector<long> ints(const std::string& s) {
	std::vector<long> v;
	for (const std::string& m : number_matches(s, false)) v.push_back(std::stol(m));
	return v;
}

// First `count` floats of s, the rest from `def`.
void fill(const std::string& s, float* out, size_t count, const float* def) {
	const std::vector<float> v = floats(s, count);
	for (size_t i = 0; i < count; ++i) out[i] = i < v.size() ? v[i] : def[i];
}

const float kIdentity[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
const float kZero3[3] = {0, 0, 0};


struct Shader {
	uint32_t kind;
	float color[3];
	float roughness = 0.1f, tail_shape = 2.0f, fresnel = 0.25f;
};

struct Object {
	uint32_t kind, n0, n1, n2;
	std::vector<float> data;
};

struct Instance {
	std::string data;
	std::vector<float> transforms;  // 16 per motion sample
	const Shader* shader = nullptr;  // bound when the instance is read
};

struct Asm {
	const Asm* parent = nullptr;
	std::deque<std::pair<std::string, Shader>> shaders;  // (stable addresses)
	std::vector<std::pair<std::string, Object>> objects;
	std::vector<std::pair<std::string, std::unique_ptr<Asm>>> subs;
	std::vector<Instance> instances;

	// the first definition of the name
	template <typename V>
	static int find(const V& v, const std::string& name) {
		for (size_t i = 0; i < v.size(); ++i)
			if (v[i].first == name) return (int)i;
		return -1;
	}
	// every definition is kept; lookups find the first
	template <typename V, typename T>
	static void put(V& v, const std::string& name, T value) {
		v.emplace_back(name, std::move(value));
	}
	// scene/assembly.hpp:113-121: the shader of that name here or in an
	// enclosing assembly
	const Shader* find_shader(const std::string& name) const {
		for (const Asm* a = this; a; a = a->parent)
			for (const auto& e : a->shaders)
				if (e.first == name) return &e.second;
		return nullptr;
	}
};

std::unique_ptr<Asm> parse_assembly(const Node& node, const Asm* parent) {
	std::unique_ptr<Asm> a(new Asm());
	a->parent = parent;
	for (const Node& ch : node.children) {
		const std::string& t = ch.type;
		const std::string& name = ch.name;
		if (t == "Assembly") {
			std::unique_ptr<Asm> sub = parse_assembly(ch, a.get());
			Asm::put(a->subs, name, std::move(sub));
		} else if (t == "BilinearPatch" || t == "BicubicPatch") {
			const bool bic = t == "BicubicPatch";
			const size_t per = bic ? 48 : 12;
			Object o{bic ? (uint32_t)PSY_OBJ_BICUBIC : (uint32_t)PSY_OBJ_BILINEAR, 0, 0, 0, {}};
			for (const Node& c : ch.children)
				if (c.type == "Vertices") {
					const std::vector<float> v = floats(c.leaf, per);
					for (size_t i = 0; i < per; ++i) o.data.push_back(i < v.size() ? v[i] : 0.0f);
					++o.n0;
				}
			Asm::put(a->objects, name, std::move(o));
		} else if (t == "Sphere") {
			float loc[3] = {0, 0, 0}, rad = 0.5f;
			for (const Node& c : ch.children) {
				if (c.type == "Radius") {
					const std::vector<float> v = floats(c.leaf, 1);
					if (!v.empty()) rad = v[0];
				} else if (c.type == "Location") {
					fill(c.leaf, loc, 3, kZero3);
				}
			}
			Asm::put(a->objects, name, Object{PSY_OBJ_SPHERE, 1, 0, 0, {loc[0], loc[1], loc[2], rad}});
		} else if (t == "SurfaceShader") {
			const Node* kind = nullptr;
			for (const Node& c : ch.children)
				if (c.type == "Type" && !kind) kind = &c;
			if (!kind) throw ParseError{"surface shader without a type"};
			Shader s{};
			if (kind->leaf == "Lambert") s.kind = PSY_SHADER_LAMBERT;
			else if (kind->leaf == "Emit") s.kind = PSY_SHADER_EMIT;
			else if (kind->leaf == "GTR") s.kind = PSY_SHADER_GTR;
			else throw ParseError{"unknown surface shader type '" + kind->leaf + "'"};
			const float grey[3] = {0.9f, 0.9f, 0.9f};
			for (int k = 0; k < 3; ++k) s.color[k] = grey[k];
			s.roughness = 0.1f;
			s.tail_shape = 2.0f;
			s.fresnel = 0.25f;
			for (const Node& c : ch.children) {
				const std::vector<float> v = c.type == "Color" ? std::vector<float>() : floats(c.leaf, 1);
				if (c.type == "Color") fill(c.leaf, s.color, 3, grey);
				else if (c.type == "Roughness" && !v.empty()) s.roughness = v[0];
				else if (c.type == "TailShape" && !v.empty()) s.tail_shape = v[0];
				else if (c.type == "Fresnel" && !v.empty()) s.fresnel = v[0];
			}
			Asm::put(a->shaders, name, s);
		} else if (t == "SphereLight") {
			std::vector<float> locs, rads, cols;
			for (const Node& c : ch.children) {
				float v3[3];
				if (c.type == "Color") {
					fill(c.leaf, v3, 3, kZero3);
					cols.insert(cols.end(), v3, v3 + 3);
				} else if (c.type == "Radius") {
					const std::vector<float> v = floats(c.leaf, 1);
					if (!v.empty()) rads.push_back(v[0]);
				} else if (c.type == "Location") {
					fill(c.leaf, v3, 3, kZero3);
					locs.insert(locs.end(), v3, v3 + 3);
				}
			}
			if (locs.empty()) locs = {0.0f, 0.0f, 0.0f};
			Object o{PSY_OBJ_SPHERE_LIGHT, (uint32_t)(locs.size() / 3), (uint32_t)rads.size(),
			         (uint32_t)(cols.size() / 3), locs};
			o.data.insert(o.data.end(), rads.begin(), rads.end());
			o.data.insert(o.data.end(), cols.begin(), cols.end());
			Asm::put(a->objects, name, std::move(o));
		} else if (t == "RectangleLight") {
			std::vector<float> dims, cols;
			for (const Node& c : ch.children) {
				if (c.type == "Color") {
					float v3[3];
					fill(c.leaf, v3, 3, kZero3);
					cols.insert(cols.end(), v3, v3 + 3);
				} else if (c.type == "Dimensions") {
					const float one[2] = {1.0f, 1.0f};
					float d[2];
					fill(c.leaf, d, 2, one);
					dims.insert(dims.end(), d, d + 2);
				}
			}
			Object o{PSY_OBJ_RECT_LIGHT, (uint32_t)(dims.size() / 2), (uint32_t)(cols.size() / 3), 0, dims};
			o.data.insert(o.data.end(), cols.begin(), cols.end());
			Asm::put(a->objects, name, std::move(o));
		} else if (t == "Instance") {
			Instance in;
			for (const Node& c : ch.children) {
				if (c.type == "Transform") {
					float m[16];
					fill(c.leaf, m, 16, kIdentity);
					in.transforms.insert(in.transforms.end(), m, m + 16);
				} else if (c.type == "Data") {
					in.data = c.leaf;
				} else if (c.type == "SurfaceShaderBind") {
					in.shader = a->find_shader(c.leaf);
					if (!in.shader) throw ParseError{"instance binds unknown shader '" + c.leaf + "'"};
				}
			}
			if (Asm::find(a->objects, in.data) < 0 && Asm::find(a->subs, in.data) < 0)
				throw ParseError{"instance of unknown data '" + in.data + "'"};
			a->instances.push_back(std::move(in));
		} else if (t == "SubdivisionSurface") {
			throw ParseError{"SubdivisionSurface is not supported"};
		}
	}
	return a;
}

}  // namespace

// Everything the description points at, owned by the handle.
struct psy_file_scene {
	std::shared_ptr<void> scene;  // the parsed assemblies, which own the object data
	struct AsmStore {
		std::vector<psy_object_desc> objects;
		std::vector<psy_instance_desc> instances;
		std::vector<float> transforms;
		std::vector<uint32_t> children;
	};
	std::deque<AsmStore> stores;
	std::vector<psy_assembly_desc> assemblies;
	std::vector<psy_shader_desc> shaders;
	std::vector<float> cam_transforms, cam_fovs, cam_apertures, cam_focus;
	psy_scene_desc desc{};
	psy_render_settings settings{1, 1, 1, 1, ""};
	std::string output_path;
};

namespace {

struct SceneRead {
	std::unique_ptr<Asm> root{new Asm()};
	std::vector<float> cam_transforms{kIdentity, kIdentity + 16};
	std::vector<float> cam_fovs_deg{45.0f}, cam_apertures, cam_focus;
	float background[3] = {0, 0, 0};
	bool has_dice_rate = false;
	float dice_rate = 0.25f;
	psy_render_settings settings{1, 1, 1, 1, ""};  // parser/parser.cpp:61-64
	std::string output_path;
};

struct NoFrame {};

// The frame-th Scene node (parser/parser.cpp:37-184; parse_next_frame reads
// them in file order).
SceneRead read_scene(const Node& tree, uint32_t frame) {
	const Node* sn = nullptr;
	uint32_t k = 0;
	for (const Node& c : tree.children)
		if (c.type == "Scene" && k++ == frame) {
			sn = &c;
			break;
		}
	if (!sn && frame == 0) throw ParseError{"no Scene node"};
	if (!sn) throw NoFrame{};
	SceneRead s;
	for (const Node& node : sn->children) {
		if (node.type == "Output") {
			// Path: the text from the first to the last double quote, the
			// quotes taken out (parser/parser.cpp:66-76)
			for (const Node& c : node.children) {
				if (c.type != "Path") continue;
				const size_t a = c.leaf.find('"'), b = c.leaf.rfind('"');
				if (a == std::string::npos || b == a) continue;
				s.output_path.clear();
				for (size_t i = a; i <= b; ++i)
					if (c.leaf[i] != '"') s.output_path += c.leaf[i];
			}
		} else if (node.type == "RenderSettings") {
			for (const Node& c : node.children) {
				if (c.type == "Resolution") {
					const std::vector<long> v = ints(c.leaf);
					if (v.size() >= 1) s.settings.width = (uint32_t)v[0];
					if (v.size() >= 2) s.settings.height = (uint32_t)v[1];
				} else if (c.type == "SamplesPerPixel") {
					const std::vector<long> v = ints(c.leaf);
					if (!v.empty()) s.settings.spp = (uint32_t)v[0];
				} else if (c.type == "DicingRate") {
					const std::vector<float> v = floats(c.leaf, 1);
					if (!v.empty()) {
						s.dice_rate = v[0];
						s.has_dice_rate = true;
					}
				} else if (c.type == "Seed") {
					const std::vector<long> v = ints(c.leaf);
					if (!v.empty()) s.settings.seed = (uint32_t)v[0];
				}
			}
		} else if (node.type == "Camera") {
			s.cam_transforms.clear();
			s.cam_fovs_deg.clear();
			for (const Node& c : node.children) {
				const std::vector<float> v = c.type == "Transform" ? std::vector<float>() : floats(c.leaf, 1);
				if (c.type == "Fov" && !v.empty()) s.cam_fovs_deg.push_back(v[0]);
				else if (c.type == "FocalDistance" && !v.empty()) s.cam_focus.push_back(v[0]);
				else if (c.type == "ApertureRadius" && !v.empty()) s.cam_apertures.push_back(v[0]);
				else if (c.type == "Transform") {
					float m[16];
					fill(c.leaf, m, 16, kIdentity);
					s.cam_transforms.insert(s.cam_transforms.end(), m, m + 16);
				}
			}
		} else if (node.type == "World") {
			for (const Node& c : node.children) {
				if (c.type != "BackgroundShader") continue;
				const Node* kind = nullptr;
				for (const Node& d : c.children)
					if (d.type == "Type" && !kind) kind = &d;
				if (!kind) throw ParseError{"background shader without a type"};
				if (kind->leaf == "Color")
					for (const Node& d : c.children)
						if (d.type == "Color") fill(d.leaf, s.background, 3, kZero3);
			}
		} else if (node.type == "Assembly") {
			s.root = parse_assembly(node, nullptr);
		}
	}
	return s;
}

void collect(Asm* a, std::vector<Asm*>& order) {
	order.push_back(a);
	for (auto& sub : a->subs) collect(sub.second.get(), order);
}

void flatten(SceneRead& s, psy_file_scene* f) {
	std::vector<Asm*> order;
	collect(s.root.get(), order);
	std::vector<const Shader*> shader_list;
	auto shader_id = [&](const Shader* sh) -> int32_t {
		if (!sh) return -1;
		for (size_t i = 0; i < shader_list.size(); ++i)
			if (shader_list[i] == sh) return (int32_t)i;
		shader_list.push_back(sh);
		return (int32_t)shader_list.size() - 1;
	};
	for (Asm* a : order) {
		f->stores.emplace_back();
		psy_file_scene::AsmStore& st = f->stores.back();
		st.objects.resize(a->objects.size() ? a->objects.size() : 1);
		for (size_t i = 0; i < a->objects.size(); ++i) {
			const Object& o = a->objects[i].second;
			st.objects[i] = psy_object_desc{o.kind, o.n0, o.n1, o.n2, o.data.data()};
		}
		st.instances.resize(a->instances.size() ? a->instances.size() : 1);
		for (size_t i = 0; i < a->instances.size(); ++i) {
			const Instance& in = a->instances[i];
			// the object of that name first, as create_object_instance /
			// create_assembly_instance are tried in the reference
			uint32_t kind = PSY_INSTANCE_OBJECT;
			int didx = Asm::find(a->objects, in.data);
			if (didx < 0) {
				kind = PSY_INSTANCE_ASSEMBLY;
				didx = Asm::find(a->subs, in.data);
			}
			const int32_t sh = shader_id(in.shader);
			st.instances[i] = psy_instance_desc{kind, (uint32_t)didx, (uint32_t)(st.transforms.size() / 16),
			                                    (uint32_t)(in.transforms.size() / 16), sh};
			st.transforms.insert(st.transforms.end(), in.transforms.begin(), in.transforms.end());
		}
		const uint32_t n_xf = (uint32_t)(st.transforms.size() / 16);
		if (st.transforms.empty()) st.transforms.assign(16, 0.0f);
		for (auto& sub : a->subs)
			for (size_t k = 0; k < order.size(); ++k)
				if (order[k] == sub.second.get()) st.children.push_back((uint32_t)k);
		const uint32_t n_ch = (uint32_t)st.children.size();
		if (st.children.empty()) st.children.push_back(0);
		f->assemblies.push_back(psy_assembly_desc{(uint32_t)a->objects.size(), st.objects.data(),
		                                          (uint32_t)a->instances.size(), st.instances.data(), n_xf,
		                                          st.transforms.data(), n_ch, st.children.data()});
	}
	for (const Shader* sh : shader_list) {
		psy_shader_desc d{};
		d.kind = sh->kind;
		for (int k = 0; k < 3; ++k) d.color[k] = sh->color[k];
		d.roughness = sh->roughness;
		d.tail_shape = sh->tail_shape;
		d.fresnel = sh->fresnel;
		f->shaders.push_back(d);
	}
	if (f->shaders.empty()) f->shaders.push_back(psy_shader_desc{});
	// parser/parser.cpp:218: field of view in radians, in float
	const float k = 3.1415926536f / 180.0f;
	for (float deg : s.cam_fovs_deg) f->cam_fovs.push_back(k * deg);
	f->cam_transforms = s.cam_transforms;
	f->cam_apertures = s.cam_apertures.empty() ? std::vector<float>{0.0f} : s.cam_apertures;
	f->cam_focus = s.cam_focus.empty() ? std::vector<float>{1.0f} : s.cam_focus;
	if (f->cam_transforms.empty()) f->cam_transforms.assign(16, 0.0f);
	if (f->cam_fovs.empty()) f->cam_fovs.push_back(0.0f);
	psy_scene_desc& d = f->desc;
	d.cam_transform_count = (uint32_t)(s.cam_transforms.size() / 16);
	d.cam_transforms = f->cam_transforms.data();
	d.cam_fov_count = (uint32_t)s.cam_fovs_deg.size();
	d.cam_fovs = f->cam_fovs.data();
	d.cam_aperture_count = (uint32_t)s.cam_apertures.size();
	d.cam_aperture_radii = f->cam_apertures.data();
	d.cam_focus_count = (uint32_t)s.cam_focus.size();
	d.cam_focus_distances = f->cam_focus.data();
	for (int c = 0; c < 3; ++c) d.background[c] = s.background[c];
	d.dice_rate = s.has_dice_rate ? s.dice_rate : 0.25f;
	d.min_upoly_size = 0.00001f;
	d.assembly_count = (uint32_t)f->assemblies.size();
	d.assemblies = f->assemblies.data();
	d.shader_count = (uint32_t)shader_list.size();
	d.shaders = f->shaders.data();
	f->settings = s.settings;
	f->output_path = s.output_path;
	f->settings.output_path = f->output_path.c_str();
	f->scene = std::shared_ptr<void>(s.root.release(), [](void* p) { delete static_cast<Asm*>(p); });
}

}  // namespace

extern "C" int psy_file_parse(const char* text, size_t len, uint32_t frame, psy_file_scene** out, char* err,
                              size_t err_len) {
	if (!out || (len && !text)) return PSY_ERR_ARG;
	*out = nullptr;
	try {
		const Node tree = build_tree(tokenize(text, len));
		SceneRead s = read_scene(tree, frame);
		std::unique_ptr<psy_file_scene> f(new psy_file_scene());
		flatten(s, f.get());
		*out = f.release();
		return PSY_OK;
	} catch (const NoFrame&) {
		if (err && err_len) std::snprintf(err, err_len, "no Scene node %u", frame);
		return PSY_ERR_NO_SCENE;
	} catch (const ParseError& e) {
		if (err && err_len) std::snprintf(err, err_len, "%s", e.msg.c_str());
	} catch (const std::exception& e) {
		if (err && err_len) std::snprintf(err, err_len, "%s", e.what());
	}
	return PSY_ERR_ARG;
}

extern "C" const psy_scene_desc* psy_file_scene_desc(const psy_file_scene* s) { return s ? &s->desc : nullptr; }

extern "C" int psy_file_render_settings(const psy_file_scene* s, psy_render_settings* out) {
	if (!s || !out) return PSY_ERR_ARG;
	*out = s->settings;
	return PSY_OK;
}

extern "C" void psy_file_free(psy_file_scene* s) { delete s; }
