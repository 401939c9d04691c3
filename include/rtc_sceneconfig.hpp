// rtc_sceneconfig.hpp - C++ adapter from the reference's sceneConfig to rtc_scene_desc.
//
// Header-only and templated on the config type, so it compiles wherever the reference's
// scenes/scene_config.h (flarive/CortexRaytracerCuda core/src/scenes/scene_config.h:452-459) is
// included, without this repository depending on glm.  It reproduces how the reference's load_scene
// turns a sceneConfig into objects (core/src/gpu.cu:481-751):
//   * object order: directional lights, spheres, quads (gpu.cu:504-547);
//   * materials and textures resolved by name, first match wins, in the order fetchMaterial /
//     fetchTexture search them (gpu.cu:193-470): lambertian (texture if named, else rgb), metal (rgb,
//     fuzziness), dielectric (refraction); solid colour, checker (textures if both resolve, else
//     colours; odd lands in m_even as scene_factory does, scene_factory.cuh:619-629), image;
//   * an object whose material does not resolve is skipped, as `if (mat)` skips it (gpu.cu:531).
// OBJ meshes are read through an optional loader callback (with this library: rtc_load_obj).
// Lights map to omni, directional and spot lights in the light list's order.  Spheres, quads and boxes
// keep their rt::transform as scene_factory::applyTransform applies it; OBJ meshes take their
// `position` as a vertex offset and their transform too, where the reference's createObjMesh drops both
// (scene_factory.cuh createObjMesh) and renders meshes[0] for every entry (gpu.cu:628); the flag
// REFERENCE_MESHES reproduces the reference there, including its texture-coordinate read with a stride
// of 3 (mesh_loader.cuh:370-371).  Primitives the
// B200 path does not cover (planes, cones, cylinders, disks, tori, volumes) are reported in `skipped`.
// Image textures need decoded RGB8 pixels: pass `load_image(filepath, &w, &h)` returning a pointer
// that stays valid while the description is used (the reference decodes with stbi_load, gpu.cu:1743).
#pragma once

#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "rtc.h"

namespace rtc_adapter {

struct SceneHolder {
    std::vector<rtc_texture> textures;
    std::vector<rtc_image> images;
    std::vector<rtc_material> materials;
    std::vector<rtc_dir_light> dir_lights;
    std::vector<rtc_omni_light> omni_lights;
    std::vector<rtc_spot_light> spot_lights;
    std::vector<rtc_sphere> spheres;
    std::vector<rtc_quad> quads;
    std::vector<rtc_mesh> meshes;
    std::vector<rtc_box> boxes;
    std::vector<rtc_transform> transforms;
    std::vector<uint32_t> sphere_transforms, quad_transforms, mesh_transforms;   // 1-based, 0 = none
    // geometry of the OBJ meshes (owned here; rtc_mesh points into it)
    std::vector<std::vector<float>> mesh_vertices, mesh_normals, mesh_uvs;
    std::vector<std::vector<uint32_t>> mesh_indices;
    std::vector<std::string> skipped;
    rtc_scene_desc desc{};

    const rtc_scene_desc* finish() {
        desc.textures = textures.data();
        desc.num_textures = (uint32_t)textures.size();
        desc.images = images.data();
        desc.num_images = (uint32_t)images.size();
        desc.materials = materials.data();
        desc.num_materials = (uint32_t)materials.size();
        desc.dir_lights = dir_lights.data();
        desc.num_dir_lights = (uint32_t)dir_lights.size();
        desc.omni_lights = omni_lights.data();
        desc.num_omni_lights = (uint32_t)omni_lights.size();
        desc.spot_lights = spot_lights.data();
        desc.num_spot_lights = (uint32_t)spot_lights.size();
        desc.spheres = spheres.data();
        desc.num_spheres = (uint32_t)spheres.size();
        desc.quads = quads.data();
        desc.num_quads = (uint32_t)quads.size();
        for (size_t i = 0; i < meshes.size(); ++i) {   // vectors may have moved since push_back
            meshes[i].vertices = mesh_vertices[i].data();
            meshes[i].indices = mesh_indices[i].data();
            meshes[i].normals = mesh_normals[i].empty() ? nullptr : mesh_normals[i].data();
            meshes[i].uvs = mesh_uvs[i].empty() ? nullptr : mesh_uvs[i].data();
        }
        desc.meshes = meshes.data();
        desc.num_meshes = (uint32_t)meshes.size();
        desc.boxes = boxes.data();
        desc.num_boxes = (uint32_t)boxes.size();
        desc.transforms = transforms.data();
        desc.num_transforms = (uint32_t)transforms.size();
        desc.sphere_transforms = transforms.empty() ? nullptr : sphere_transforms.data();
        desc.quad_transforms = transforms.empty() ? nullptr : quad_transforms.data();
        desc.mesh_transforms = transforms.empty() ? nullptr : mesh_transforms.data();
        return &desc;
    }
};

using ImageLoader = std::function<const uint8_t*(const char* filepath, int* width, int* height)>;
// Reads an OBJ file's triangles: positions (3 per vertex), indices (3 per triangle), per-vertex
// normals (3 per vertex, or left empty) and per-vertex texture coordinates (2 per vertex, or left
// empty); returns false when the file cannot be read.  With this library, a wrapper around
// rtc_load_obj / rtc_free_obj.
using ObjLoader = std::function<bool(const char* filepath, std::vector<float>& vertices, std::vector<uint32_t>& indices,
                                     std::vector<float>& normals, std::vector<float>& uvs)>;

namespace detail {
inline bool same(const char* a, const char* b) { return a && b && std::strcmp(a, b) == 0; }
inline bool named(const char* a) { return a && a[0] != '\0'; }
template <class V> void put3(float* dst, const V& v) { dst[0] = v.x; dst[1] = v.y; dst[2] = v.z; }
template <class C> void putc3(float* dst, const C& c) { dst[0] = c.r(); dst[1] = c.g(); dst[2] = c.b(); }
// An rt::transform (misc/transform.cuh) as a 1-based reference into out.transforms; 0 when it has no part.
template <class T> uint32_t add_transform(const T& trs, SceneHolder& out) {
    rtc_transform x{};
    x.flags = (trs.hasTranslate() ? RTC_XF_TRANSLATE : 0u) | (trs.hasRotate() ? RTC_XF_ROTATE : 0u) |
              (trs.hasScale() ? RTC_XF_SCALE : 0u);
    if (!x.flags) return 0;
    put3(x.translate, trs.getTranslate());
    put3(x.rotate, trs.getRotate());
    put3(x.scale, trs.getScale());
    out.transforms.push_back(x);
    return (uint32_t)out.transforms.size();
}
}  // namespace detail

// from_sceneconfig flag: OBJ meshes as the reference's load_scene adds them.  Every objMeshes entry
// renders the first entry's file, meshes[0] (gpu.cu:626-631), with its own material and smoothing, and
// without its position or transform, which createObjMesh drops (scene_factory.cuh:373-385).  By default
// each entry renders its own file, offset by its position and transformed.
constexpr uint32_t REFERENCE_MESHES = 1u;

// Converts `cfg` (a reference sceneConfig) into `out`; returns out.finish().
template <class SceneConfig>
const rtc_scene_desc* from_sceneconfig(const SceneConfig& cfg, SceneHolder& out, const ImageLoader& load_image = nullptr,
                                       const ObjLoader& load_obj = nullptr, uint32_t flags = 0) {
    using namespace detail;
    const auto& T = cfg.texturesCfg;
    const auto& M = cfg.materialsCfg;

    auto solid = [&](const auto& c) {
        rtc_texture t{};
        t.kind = RTC_TEX_SOLID;
        putc3(t.color, c);
        t.even = t.odd = t.image = -1;
        out.textures.push_back(t);
        return (int)out.textures.size() - 1;
    };

    std::function<int(const char*, int)> fetch_texture = [&](const char* name, int depth) -> int {
        if (!named(name) || depth > 4) return -1;
        for (int i = 0; i < T.solidColorTextureCount; ++i)
            if (same(T.solidColorTextures[i].name, name)) return solid(T.solidColorTextures[i].rgb);
        for (int i = 0; i < T.imageTextureCount; ++i) {
            if (!same(T.imageTextures[i].name, name)) continue;
            if (!load_image) { out.skipped.push_back(std::string("image texture without loader: ") + name); return -1; }
            int w = 0, h = 0;
            const uint8_t* px = load_image(T.imageTextures[i].filepath, &w, &h);
            if (!px || w <= 0 || h <= 0) { out.skipped.push_back(std::string("image not loaded: ") + name); return -1; }
            out.images.push_back(rtc_image{px, w, h});
            rtc_texture t{};
            t.kind = RTC_TEX_IMAGE;
            t.even = t.odd = -1;
            t.image = (int)out.images.size() - 1;
            out.textures.push_back(t);
            return (int)out.textures.size() - 1;
        }
        for (int i = 0; i < T.checkerTextureCount; ++i) {
            const auto& c = T.checkerTextures[i];
            if (!same(c.name, name)) continue;
            int odd = fetch_texture(c.oddTextureName, depth + 1);
            int even = fetch_texture(c.evenTextureName, depth + 1);
            if (odd < 0 || even < 0) { odd = solid(c.oddColor); even = solid(c.evenColor); }
            rtc_texture t{};
            t.kind = RTC_TEX_CHECKER;
            t.scale = c.scale;
            t.even = odd;    // checker_texture(scale, odd, even): m_even <- odd (checker_texture.cuh:28-31)
            t.odd = even;
            t.image = -1;
            out.textures.push_back(t);
            return (int)out.textures.size() - 1;
        }
        out.skipped.push_back(std::string("texture kind not covered: ") + name);
        return -1;
    };

    auto fetch_material = [&](const char* name) -> int {
        if (!named(name)) return -1;
        for (int i = 0; i < M.lambertianMaterialCount; ++i) {
            const auto& m = M.lambertianMaterials[i];
            if (!same(m.name, name)) continue;
            int tex = named(m.textureName) ? fetch_texture(m.textureName, 0) : solid(m.rgb);
            if (tex < 0) return -1;
            out.materials.push_back(rtc_material{RTC_MAT_LAMBERTIAN, tex, 0.f, 0.f, 0.f, 0});
            return (int)out.materials.size() - 1;
        }
        for (int i = 0; i < M.metalMaterialCount; ++i) {
            const auto& m = M.metalMaterials[i];
            if (!same(m.name, name)) continue;
            out.materials.push_back(rtc_material{RTC_MAT_METAL, solid(m.rgb), m.fuzziness < 1 ? m.fuzziness : 1.f, 0.f, 0.f, 0});
            return (int)out.materials.size() - 1;
        }
        for (int i = 0; i < M.dielectricMaterialCount; ++i) {
            const auto& m = M.dielectricMaterials[i];
            if (!same(m.name, name)) continue;
            out.materials.push_back(rtc_material{RTC_MAT_DIELECTRIC, -1, 0.f, m.refraction, 0.f, 0});
            return (int)out.materials.size() - 1;
        }
        out.skipped.push_back(std::string("material not covered or missing: ") + name);
        return -1;
    };

    const auto& L = cfg.lightsCfg;
    // lightsCfg -> light list: omni, directional, spot (load_scene, gpu.cu:504-523)
    for (int i = 0; i < L.omniLightCount; ++i) {
        const auto& o = L.omniLights[i];
        rtc_omni_light l{};
        put3(l.position, o.position);
        l.radius = o.radius;
        putc3(l.color, o.rgb);
        l.intensity = o.intensity;
        l.invisible = o.invisible ? 1 : 0;
        out.omni_lights.push_back(l);
    }
    for (int i = 0; i < L.dirLightCount; ++i) {
        const auto& d = L.dirLights[i];
        rtc_dir_light l{};
        put3(l.position, d.position);
        put3(l.u, d.u);
        put3(l.v, d.v);
        putc3(l.color, d.rgb);
        l.intensity = d.intensity;
        l.invisible = d.invisible ? 1 : 0;
        out.dir_lights.push_back(l);
    }
    for (int i = 0; i < L.spotLightCount; ++i) {
        const auto& sp = L.spotLights[i];
        rtc_spot_light l{};
        put3(l.position, sp.position);
        put3(l.direction, sp.direction);
        l.cutoff = sp.cutoff;
        l.falloff = sp.falloff;
        l.intensity = sp.intensity;
        l.radius = sp.radius;
        putc3(l.color, sp.rgb);
        l.invisible = sp.invisible ? 1 : 0;
        out.spot_lights.push_back(l);
    }

    const auto& P = cfg.primitivesCfg;
    for (int i = 0; i < P.spherePrimitiveCount; ++i) {
        const auto& s = P.spherePrimitives[i];
        int m = fetch_material(s.materialName);
        if (m < 0) continue;
        rtc_sphere o{};
        put3(o.center, s.position);
        o.radius = s.radius;
        o.material = m;
        out.spheres.push_back(o);
        out.sphere_transforms.push_back(add_transform(s.transform, out));   // scene_factory::createSphere
    }
    if (P.planePrimitiveCount) out.skipped.push_back("planes");
    for (int i = 0; i < P.quadPrimitiveCount; ++i) {
        const auto& q = P.quadPrimitives[i];
        int m = fetch_material(q.materialName);
        if (m < 0) continue;
        rtc_quad o{};
        put3(o.q, q.position);
        put3(o.u, q.u);
        put3(o.v, q.v);
        o.material = m;
        out.quads.push_back(o);
        out.quad_transforms.push_back(add_transform(q.transform, out));
    }
    // boxes after the quads (gpu.cu:556-565; scene_factory::createBox, box.cuh)
    for (int i = 0; i < P.boxPrimitiveCount; ++i) {
        const auto& b = P.boxPrimitives[i];
        int m = fetch_material(b.materialName);
        if (m < 0) continue;
        rtc_box o{};
        put3(o.center, b.position);
        put3(o.size, b.size);
        o.material = m;
        o.transform = add_transform(b.transform, out);
        out.boxes.push_back(o);
    }
    if (P.conePrimitiveCount || P.cylinderPrimitiveCount || P.diskPrimitiveCount || P.torusPrimitiveCount ||
        P.volumePrimitiveCount)
        out.skipped.push_back("cones/cylinders/disks/tori/volumes");
    // OBJ meshes (load_scene adds them after the boxes, gpu.cu:612-635): geometry offset by `position`,
    // then the mesh's transform; one material for the whole mesh (use_mtl materials are reported)
    const auto& MS = cfg.meshesCfg;
    const bool ref_meshes = (flags & REFERENCE_MESHES) != 0;
    for (int i = 0; i < MS.objMeshCount; ++i) {
        const auto& m = MS.objMeshes[i];
        // with REFERENCE_MESHES the geometry is always meshes[0]'s file, placed as it is in the file
        const auto& g = ref_meshes ? MS.objMeshes[0] : m;
        if (!load_obj) { out.skipped.push_back(std::string("OBJ mesh without loader: ") + (g.filepath ? g.filepath : "")); continue; }
        const int mat = fetch_material(m.materialName);
        if (mat < 0) continue;
        std::vector<float> v, n, t;
        std::vector<uint32_t> idx;
        if (!g.filepath || !load_obj(g.filepath, v, idx, n, t) || idx.empty()) {
            out.skipped.push_back(std::string("OBJ mesh not loaded: ") + (g.filepath ? g.filepath : ""));
            continue;
        }
        float off[3] = {0.f, 0.f, 0.f};
        if (!ref_meshes) put3(off, m.position);
        for (size_t k = 0; k < v.size(); k += 3) {
            v[k] += off[0];
            v[k + 1] += off[1];
            v[k + 2] += off[2];
        }
        if (m.use_mtl) out.skipped.push_back(std::string("OBJ materials (use_mtl) of ") + m.filepath);
        rtc_mesh r{};
        r.num_vertices = (uint32_t)(v.size() / 3);
        r.num_triangles = (uint32_t)(idx.size() / 3);
        r.material = mat;
        r.smooth = (m.use_smoothing && n.size() == v.size()) ? 1 : 0;
        out.mesh_vertices.push_back(std::move(v));
        out.mesh_indices.push_back(std::move(idx));
        out.mesh_normals.push_back(r.smooth ? std::move(n) : std::vector<float>());
        if (t.size() != 2 * (size_t)r.num_vertices) t.clear();
        if (ref_meshes && !t.empty()) {
            // mesh_loader reads texcoords[3 * idx + 0], [3 * idx + 1] from an array of 2 per vertex
            // (mesh_loader.cuh:370-371); reads past its end - undefined memory there - give 0 here
            std::vector<float> r3(t.size(), 0.0f);
            for (size_t k = 0; k < r.num_vertices; ++k)
                for (size_t c = 0; c < 2; ++c)
                    if (3 * k + c < t.size()) r3[2 * k + c] = t[3 * k + c];
            t.swap(r3);
        }
        out.mesh_uvs.push_back(std::move(t));
        out.meshes.push_back(r);
        out.mesh_transforms.push_back(ref_meshes ? 0u : add_transform(m.transform, out));
    }

    const auto& C = cfg.cameraCfg;
    put3(out.desc.camera.look_from, C.lookFrom);
    put3(out.desc.camera.look_at, C.lookAt);
    put3(out.desc.camera.up, C.upAxis);
    out.desc.camera.vfov = C.fov;
    out.desc.camera.aspect = C.aspectRatio;
    out.desc.camera.aperture = C.aperture;
    out.desc.camera.focus = C.focus;
    out.desc.background.kind = RTC_BG_CONSTANT;   // the GPU path uses background.rgb only (gpu.cu:729-742)
    putc3(out.desc.background.color, cfg.imageCfg.background.rgb);
    return out.finish();
}

}  // namespace rtc_adapter
