// scenefile_check.cpp - TEST INFRASTRUCTURE ONLY.  Reads a `.scene` file with the reference's own loader
// (flarive/CortexRaytracerCuda core/src/scenes/scene_loader.cpp and scene_builder.cpp over its vendored
// libconfig, compiled from the reference tree in place), converts the resulting sceneConfig with
// include/rtc_sceneconfig.hpp, and prints the rtc_scene_desc as one JSON line, for
// tests/test_scene_file.py to compare with the library's own reader (rtc_scene_file_load).
//
// OBJ meshes are read here with a minimal reader of `v`, `vn` and triangular `f` lines (enough for the
// test's files); the reference itself reads them later, in load_scene, with tinyobjloader.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "scenes/scene_loader.h"
#include "rtc_sceneconfig.hpp"

static void arr(const char* k, const float* v, int n, bool comma = true) {
    std::printf("\"%s\": [", k);
    for (int i = 0; i < n; ++i) std::printf("%s%.9g", i ? ", " : "", v[i]);
    std::printf("]%s", comma ? ", " : "");
}

static bool read_obj(const char* path, std::vector<float>& v, std::vector<uint32_t>& idx, std::vector<float>& n,
                     std::vector<float>&) {
    std::ifstream f(path);
    if (!f) return false;
    std::vector<float> vn;
    std::vector<int> fn;
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream s(line);
        std::string k;
        s >> k;
        if (k == "v") { float x, y, z; s >> x >> y >> z; v.insert(v.end(), {x, y, z}); }
        else if (k == "vn") { float x, y, z; s >> x >> y >> z; vn.insert(vn.end(), {x, y, z}); }
        else if (k == "f") {
            for (int c = 0; c < 3; ++c) {
                std::string t;
                s >> t;
                idx.push_back((uint32_t)(std::atoi(t.c_str()) - 1));
                const size_t p = t.rfind('/');
                fn.push_back(p == std::string::npos ? -1 : std::atoi(t.c_str() + p + 1) - 1);
            }
        }
    }
    if (!vn.empty()) {   // one normal per vertex, from the faces' corners
        n.assign(v.size(), 0.0f);
        for (size_t c = 0; c < idx.size(); ++c)
            if (fn[c] >= 0)
                for (int k = 0; k < 3; ++k) n[3 * idx[c] + k] = vn[3 * fn[c] + k];
    }
    return true;
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    scene_loader loader(argv[1]);
    scene_builder b = loader.loadSceneFromFile();
    sceneConfig cfg{b.getImageConfig(), b.getCameraConfig(), b.getLightsConfig(), b.getTexturesConfig(),
                    b.getMaterialsConfig(), b.getPrimitivesConfig(), b.getMeshesConfig()};
    rtc_adapter::SceneHolder h;
    const rtc_scene_desc* d = rtc_adapter::from_sceneconfig(cfg, h, nullptr, read_obj);
    std::fflush(stdout);
    std::printf("\n{\"textures\": [");
    for (uint32_t i = 0; i < d->num_textures; ++i) {
        const rtc_texture& t = d->textures[i];
        std::printf("%s{\"kind\": %d, ", i ? ", " : "", t.kind);
        arr("color", t.color, 3);
        std::printf("\"scale\": %.9g, \"even\": %d, \"odd\": %d, \"image\": %d}", t.scale, t.even, t.odd, t.image);
    }
    std::printf("], \"materials\": [");
    for (uint32_t i = 0; i < d->num_materials; ++i) {
        const rtc_material& m = d->materials[i];
        std::printf("%s{\"kind\": %d, \"texture\": %d, \"fuzz\": %.9g, \"ior\": %.9g}", i ? ", " : "", m.kind, m.texture,
                    m.fuzz, m.ior);
    }
    std::printf("], \"dir_lights\": [");
    for (uint32_t i = 0; i < d->num_dir_lights; ++i) {
        const rtc_dir_light& l = d->dir_lights[i];
        std::printf("%s{", i ? ", " : "");
        arr("position", l.position, 3);
        arr("u", l.u, 3);
        arr("v", l.v, 3);
        arr("color", l.color, 3);
        std::printf("\"intensity\": %.9g, \"invisible\": %d}", l.intensity, l.invisible);
    }
    std::printf("], \"omni_lights\": [");
    for (uint32_t i = 0; i < d->num_omni_lights; ++i) {
        const rtc_omni_light& l = d->omni_lights[i];
        std::printf("%s{", i ? ", " : "");
        arr("position", l.position, 3);
        arr("color", l.color, 3);
        std::printf("\"radius\": %.9g, \"intensity\": %.9g, \"invisible\": %d}", l.radius, l.intensity, l.invisible);
    }
    std::printf("], \"spot_lights\": [");
    for (uint32_t i = 0; i < d->num_spot_lights; ++i) {
        const rtc_spot_light& l = d->spot_lights[i];
        std::printf("%s{", i ? ", " : "");
        arr("position", l.position, 3);
        arr("direction", l.direction, 3);
        arr("color", l.color, 3);
        std::printf("\"cutoff\": %.9g, \"falloff\": %.9g, \"radius\": %.9g, \"intensity\": %.9g, \"invisible\": %d}",
                    l.cutoff, l.falloff, l.radius, l.intensity, l.invisible);
    }
    std::printf("], \"spheres\": [");
    for (uint32_t i = 0; i < d->num_spheres; ++i) {
        const rtc_sphere& s = d->spheres[i];
        std::printf("%s{", i ? ", " : "");
        arr("center", s.center, 3);
        std::printf("\"radius\": %.9g, \"material\": %d}", s.radius, s.material);
    }
    std::printf("], \"quads\": [");
    for (uint32_t i = 0; i < d->num_quads; ++i) {
        const rtc_quad& q = d->quads[i];
        std::printf("%s{", i ? ", " : "");
        arr("q", q.q, 3);
        arr("u", q.u, 3);
        arr("v", q.v, 3);
        std::printf("\"material\": %d}", q.material);
    }
    std::printf("], \"boxes\": [");
    for (uint32_t i = 0; i < d->num_boxes; ++i) {
        const rtc_box& b = d->boxes[i];
        std::printf("%s{", i ? ", " : "");
        arr("center", b.center, 3);
        arr("size", b.size, 3);
        std::printf("\"material\": %d, \"transform\": %u}", b.material, b.transform);
    }
    std::printf("], \"transforms\": [");
    for (uint32_t i = 0; i < d->num_transforms; ++i) {
        const rtc_transform& x = d->transforms[i];
        std::printf("%s{", i ? ", " : "");
        arr("translate", x.translate, 3);
        arr("rotate", x.rotate, 3);
        arr("scale", x.scale, 3);
        std::printf("\"flags\": %u}", x.flags);
    }
    auto refs = [&](const char* k, const uint32_t* r, uint32_t n) {
        std::printf("], \"%s\": [", k);
        for (uint32_t i = 0; r && i < n; ++i) std::printf("%s%u", i ? ", " : "", r[i]);
    };
    refs("sphere_transforms", d->sphere_transforms, d->num_spheres);
    refs("quad_transforms", d->quad_transforms, d->num_quads);
    refs("mesh_transforms", d->mesh_transforms, d->num_meshes);
    std::printf("], \"meshes\": [");
    for (uint32_t i = 0; i < d->num_meshes; ++i) {
        const rtc_mesh& m = d->meshes[i];
        std::printf("%s{", i ? ", " : "");
        arr("vertices", m.vertices, (int)(3 * m.num_vertices));
        std::printf("\"num_triangles\": %u, \"material\": %d, \"smooth\": %d}", m.num_triangles, m.material, m.smooth);
    }
    std::printf("], \"camera\": {");
    arr("look_from", d->camera.look_from, 3);
    arr("look_at", d->camera.look_at, 3);
    arr("up", d->camera.up, 3);
    std::printf("\"vfov\": %.9g, \"aspect\": %.9g, \"aperture\": %.9g, \"focus\": %.9g}, ", d->camera.vfov,
                d->camera.aspect, d->camera.aperture, d->camera.focus);
    arr("background", d->background.color, 3, false);
    std::printf(", \"image\": {\"width\": %d, \"height\": %d, \"spp\": %d, \"max_depth\": %d}}\n", cfg.imageCfg.width,
                cfg.imageCfg.height, cfg.imageCfg.spp, cfg.imageCfg.depth);
    return 0;
}
