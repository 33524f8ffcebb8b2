// Scene model: owning host description (Scene) and the non-owning flat view (SceneView).
//
// The struct layouts are the reference's public API (WVM/include/wf/scene.hpp:12-100) and are
// kept byte-identical so that code written against the reference links against this engine:
// Material 48 B, Sphere 32 B, Triangle 16 B, Light 16 B, BvhNode 48 B, HitRecord 16 B.
// The device never reads these structs directly during traversal; the engine repacks them into
// its own layout at upload (see csrc/dev_scene.cuh).
#pragma once
#include <string>
#include <vector>
#include "wf/math.hpp"

namespace wf {

enum MaterialType : int { kLambert = 0, kMetal = 1, kDielectric = 2, kEmissive = 3 };
constexpr int kNumMaterialTypes = 4;

struct Material {
    int type;
    float ior;   // dielectric index of refraction
    float pad0;  // this engine stores the metal roughness of generated scenes here (shading ignores it)
    float pad1;
    Vec3 albedo;
    float pad2;
    Vec3 emission;  // radiance; any material type may emit
    float pad3;
};

struct Sphere {
    Vec3 center;
    float radius;
    int material;
    int pad[3];
};

struct Triangle {  // indexed triangle
    int i0, i1, i2;
    int material;
};

struct Camera {
    Vec3 position;
    Vec3 look_at;
    Vec3 up;
    float vfov_deg;
};

struct CameraRig {
    Vec3 origin;
    Vec3 lower_left;
    Vec3 horizontal;
    Vec3 vertical;
};

struct Light {
    int prim;  // primitive id: spheres first, then triangles
    float area;
    float pad[2];
};

// Preorder BVH node: the left child of an internal node N is N+1; `skip` is the node to visit
// after N's subtree (miss or finished leaf), -1 ends the traversal.
struct BvhNode {
    Vec3 lo;
    int skip;
    Vec3 hi;
    int prim_start;  // leaf: first entry in prim_order; internal: -1
    int prim_count;  // leaf: > 0; internal: 0
    int pad[3];
};

struct HitRecord {
    float t;
    int prim;  // -1 for a miss
    float u, v;
};

struct SceneView {
    const Sphere* spheres;
    const Vec3* vertices;
    const Triangle* triangles;
    const Material* materials;
    const BvhNode* nodes;
    const int* prim_order;
    const Light* lights;
    int n_spheres, n_triangles, n_materials, n_nodes, n_lights;
    Vec3 env;
    CameraRig camera;
    int width, height;
};

struct Scene {
    std::string name;
    std::vector<Sphere> spheres;
    std::vector<Vec3> vertices;
    std::vector<Triangle> triangles;
    std::vector<Material> materials;
    std::vector<BvhNode> nodes;
    std::vector<int> prim_order;
    std::vector<Light> lights;
    Vec3 env{0.0f, 0.0f, 0.0f};
    Camera camera{};
    int width = 1280, height = 720;

    int n_prims() const { return (int)spheres.size() + (int)triangles.size(); }
    SceneView view() const;
};

// Light list from emissive primitives + BVH + validation. Throws std::runtime_error.
void finalize_scene(Scene& scene);
// Finalize with an explicit SAH bin count (the reference uses 8; the benchmark scenes use 16).
void finalize_scene_bins(Scene& scene, int sah_bins);
std::string validate_scene(const Scene& scene);
void build_bvh(Scene& scene);
void build_bvh_bins(Scene& scene, int sah_bins);
// SAH builder knobs (bins == 8 selects the reference-compatible policy and ignores the others):
// leaves hold at most max_leaf primitives (1..15); a node of <= max_leaf primitives becomes a
// leaf unless a split is cheaper with traversal cost `traversal_cost` (intersection cost 1).
// Subtrees are built on `threads` threads (0: all cores); the tree does not depend on it.
void build_bvh_options(Scene& scene, int sah_bins, int max_leaf, float traversal_cost, int threads = 0);
std::string validate_bvh(const Scene& scene);
Scene make_scene(const std::string& name, int width, int height);
Scene load_obj(const std::string& path, int width, int height);
uint64_t scene_hash(const Scene& scene);

static_assert(sizeof(Material) == 48, "Material layout");
static_assert(sizeof(Sphere) == 32, "Sphere layout");
static_assert(sizeof(Triangle) == 16, "Triangle layout");
static_assert(sizeof(Light) == 16, "Light layout");
static_assert(sizeof(BvhNode) == 48, "BvhNode layout");
static_assert(sizeof(HitRecord) == 16, "HitRecord layout");

// Pinhole camera rig (WVM/include/wf/scene.hpp:129-141): w points from the target to the eye,
// u = normalize(up x w), v = w x u, half-height h = tan(vfov/2). Always evaluated on the HOST
// (glibc tanf), also for the GPU arms, exactly as the reference does.
WF_HD CameraRig make_camera_rig(const Camera& cam, int width, int height) {
    const float aspect = (float)width / (float)height;
    const float h = tanf(cam.vfov_deg * 0.5f * kPi / 180.0f);
    const Vec3 w = normalize(cam.position - cam.look_at);
    const Vec3 u = normalize(cross(cam.up, w));
    const Vec3 v = cross(w, u);
    CameraRig rig;
    rig.origin = cam.position;
    rig.horizontal = u * (2.0f * h * aspect);
    rig.vertical = v * (2.0f * h);
    rig.lower_left = rig.origin - rig.horizontal * 0.5f - rig.vertical * 0.5f - w;
    return rig;
}

}  // namespace wf
