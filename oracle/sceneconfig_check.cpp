// sceneconfig_check.cpp - TEST INFRASTRUCTURE ONLY.  Compiles include/rtc_sceneconfig.hpp against the
// reference's own scene description types (flarive/CortexRaytracerCuda core/src/scenes/scene_config.h,
// read in place) and prints the rtc_scene_desc the adapter makes from one sceneConfig, as JSON, for
// tests/test_sceneconfig_adapter.py.
//
// The sceneConfig below is a Cornell box written the way the reference's scene loader fills it for
// data/scenes/cornell_box.scene (named lambertian materials with rgb, one directional light, five wall
// quads), plus the cases the adapter must resolve the way load_scene does (core/src/gpu.cu:481-751):
// a checker texture made from colours (odd/even swap, scene_factory.cuh:619-629), a checker whose
// child textures are named, a metal with fuzz above 1 (clamped), a dielectric, a sphere whose
// material does not exist (skipped, gpu.cu:531) and a box (not covered, reported).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "scenes/scene_config.h"
#include "rtc_sceneconfig.hpp"

static void arr3(const char* k, const float* v, bool comma = true) {
    std::printf("\"%s\": [%.9g, %.9g, %.9g]%s", k, v[0], v[1], v[2], comma ? ", " : "");
}

int main() {
    sceneConfig cfg;
    std::memset((void*)&cfg, 0, sizeof cfg);
    cfg.imageCfg.background.rgb = color(0.1f, 0.2f, 0.3f);
    cfg.cameraCfg.aspectRatio = 1.0f;
    cfg.cameraCfg.lookFrom = point3(278.0f, 278.0f, -800.0f);
    cfg.cameraCfg.lookAt = point3(278.0f, 278.0f, 0.0f);
    cfg.cameraCfg.upAxis = vector3(0.0f, 1.0f, 0.0f);
    cfg.cameraCfg.aperture = 0.0f;
    cfg.cameraCfg.focus = 10.0f;
    cfg.cameraCfg.fov = 40.0f;

    static solidColorTextureConfig solids[2];
    solids[0].name = "tex_white";
    solids[0].rgb = color(0.9f, 0.9f, 0.9f);
    solids[1].name = "tex_blue";
    solids[1].rgb = color(0.1f, 0.2f, 0.8f);
    static checkerTextureConfig checkers[2];
    checkers[0].name = "chk_colors";
    checkers[0].oddTextureName = nullptr;
    checkers[0].evenTextureName = nullptr;
    checkers[0].oddColor = color(1.0f, 0.0f, 0.0f);
    checkers[0].evenColor = color(0.0f, 1.0f, 0.0f);
    checkers[0].scale = 0.5f;
    checkers[1].name = "chk_named";
    checkers[1].oddTextureName = "tex_white";
    checkers[1].evenTextureName = "tex_blue";
    checkers[1].scale = 2.0f;
    cfg.texturesCfg.solidColorTextures = solids;
    cfg.texturesCfg.solidColorTextureCount = 2;
    cfg.texturesCfg.checkerTextures = checkers;
    cfg.texturesCfg.checkerTextureCount = 2;

    static lambertianMaterialConfig lam[5];
    lam[0].name = "red";    lam[0].textureName = nullptr; lam[0].rgb = color(0.65f, 0.05f, 0.05f);
    lam[1].name = "white";  lam[1].textureName = nullptr; lam[1].rgb = color(0.73f, 0.73f, 0.73f);
    lam[2].name = "green";  lam[2].textureName = nullptr; lam[2].rgb = color(0.12f, 0.45f, 0.15f);
    lam[3].name = "floor";  lam[3].textureName = "chk_colors";
    lam[4].name = "ball";   lam[4].textureName = "chk_named";
    static metalMaterialConfig met[1];
    met[0].name = "mirror"; met[0].rgb = color(0.8f, 0.85f, 0.9f); met[0].fuzziness = 1.7f;
    static dielectricMaterialConfig die[1];
    die[0].name = "glass"; die[0].refraction = 1.5f;
    cfg.materialsCfg.lambertianMaterials = lam;
    cfg.materialsCfg.lambertianMaterialCount = 5;
    cfg.materialsCfg.metalMaterials = met;
    cfg.materialsCfg.metalMaterialCount = 1;
    cfg.materialsCfg.dielectricMaterials = die;
    cfg.materialsCfg.dielectricMaterialCount = 1;

    static directionalLightConfig lights[1];
    lights[0].position = point3(278.0f, 554.0f, 332.0f);
    lights[0].u = vector3(-130.0f, 0.0f, 0.0f);
    lights[0].v = vector3(0.0f, 0.0f, -105.0f);
    lights[0].intensity = 1.5f;
    lights[0].rgb = color(15.0f, 15.0f, 15.0f);
    lights[0].name = "QuadLight1";
    lights[0].invisible = true;
    cfg.lightsCfg.dirLights = lights;
    cfg.lightsCfg.dirLightCount = 1;

    static omniLightConfig omnis[1];
    omnis[0].position = point3(100.0f, 500.0f, 200.0f);
    omnis[0].radius = 20.0f;
    omnis[0].intensity = 2.0f;
    omnis[0].rgb = color(4.0f, 3.0f, 2.0f);
    omnis[0].name = "SphereLight1";
    omnis[0].invisible = false;
    cfg.lightsCfg.omniLights = omnis;
    cfg.lightsCfg.omniLightCount = 1;

    static spotLightConfig spots[1];
    spots[0].position = point3(400.0f, 500.0f, 300.0f);
    spots[0].direction = vector3(0.0f, -1.0f, 0.2f);
    spots[0].cutoff = 30.0f;
    spots[0].falloff = 3.0f;
    spots[0].intensity = 5.0f;
    spots[0].radius = 10.0f;
    spots[0].rgb = color(6.0f, 6.0f, 5.0f);
    spots[0].name = "SpotLight1";
    spots[0].invisible = true;
    cfg.lightsCfg.spotLights = spots;
    cfg.lightsCfg.spotLightCount = 1;

    static quadPrimitiveConfig quads[6];
    const float qv[6][9] = {{555, 0, 0, 0, 555, 0, 0, 0, 555},     {0, 0, 0, 0, 555, 0, 0, 0, 555},
                            {0, 0, 0, 555, 0, 0, 0, 0, 555},       {555, 555, 555, -555, 0, 0, 0, 0, -555},
                            {0, 0, 555, 555, 0, 0, 0, 555, 0},     {1, 2, 3, 4, 0, 0, 0, 5, 0}};
    const char* qm[6] = {"green", "red", "floor", "white", "white", "nosuchmaterial"};
    for (int i = 0; i < 6; ++i) {
        quads[i].name = "q";
        quads[i].position = point3(qv[i][0], qv[i][1], qv[i][2]);
        quads[i].u = vector3(qv[i][3], qv[i][4], qv[i][5]);
        quads[i].v = vector3(qv[i][6], qv[i][7], qv[i][8]);
        quads[i].materialName = qm[i];
    }
    static spherePrimitiveConfig spheres[4];
    const char* sm[4] = {"glass", "mirror", "missing", "ball"};
    for (int i = 0; i < 4; ++i) {
        spheres[i].name = "s";
        spheres[i].position = point3(100.0f + 100.0f * i, 90.0f, 190.0f);
        spheres[i].radius = 90.0f - 10.0f * i;
        spheres[i].materialName = sm[i];
    }
    static boxPrimitiveConfig boxes[1];
    boxes[0].name = "box";
    boxes[0].materialName = "white";
    boxes[0].position = point3(212.5f, 82.5f, 147.5f);
    boxes[0].size = vector3(165.0f, 165.0f, 165.0f);
    boxes[0].transform.setTranslate(vector3(10.0f, 0.0f, -5.0f));
    boxes[0].transform.setRotate(vector3(0.0f, 18.0f, 0.0f));
    spheres[0].transform.setScale(vector3(2.0f, 1.0f, 1.0f));
    cfg.primitivesCfg.quadPrimitives = quads;
    cfg.primitivesCfg.quadPrimitiveCount = 6;
    cfg.primitivesCfg.spherePrimitives = spheres;
    cfg.primitivesCfg.spherePrimitiveCount = 4;
    cfg.primitivesCfg.boxPrimitives = boxes;
    cfg.primitivesCfg.boxPrimitiveCount = 1;

    static objMeshConfig objs[2];
    objs[0].name = "tetra";
    objs[0].position = point3(10.0f, 20.0f, 30.0f);
    objs[0].filepath = "tetra.obj";
    objs[0].materialName = "mirror";
    objs[0].use_mtl = false;
    objs[0].use_smoothing = true;
    objs[1].name = "unreadable";
    objs[1].filepath = "missing.obj";
    objs[1].materialName = "white";
    cfg.meshesCfg.objMeshes = objs;
    cfg.meshesCfg.objMeshCount = 2;
    // a stand-in for rtc_load_obj: one tetrahedron with normals for "tetra.obj", nothing else
    auto load_obj = [](const char* path, std::vector<float>& v, std::vector<uint32_t>& idx, std::vector<float>& n,
                       std::vector<float>&) {
        if (std::strcmp(path, "tetra.obj") != 0) return false;
        v = {0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1};
        idx = {0, 2, 1, 0, 1, 3, 0, 3, 2, 1, 2, 3};
        n = {-1, -1, -1, 1, 0, 0, 0, 1, 0, 0, 0, 1};
        return true;
    };

    rtc_adapter::SceneHolder h;
    const rtc_scene_desc* d = rtc_adapter::from_sceneconfig(cfg, h, nullptr, load_obj);

    std::printf("{\"textures\": [");
    for (uint32_t i = 0; i < d->num_textures; ++i) {
        const rtc_texture& t = d->textures[i];
        std::printf("%s{\"kind\": %d, ", i ? ", " : "", t.kind);
        arr3("color", t.color);
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
        arr3("position", l.position);
        arr3("u", l.u);
        arr3("v", l.v);
        arr3("color", l.color);
        std::printf("\"intensity\": %.9g, \"invisible\": %d}", l.intensity, l.invisible);
    }
    std::printf("], \"omni_lights\": [");
    for (uint32_t i = 0; i < d->num_omni_lights; ++i) {
        const rtc_omni_light& l = d->omni_lights[i];
        std::printf("%s{", i ? ", " : "");
        arr3("position", l.position);
        arr3("color", l.color);
        std::printf("\"radius\": %.9g, \"intensity\": %.9g, \"invisible\": %d}", l.radius, l.intensity, l.invisible);
    }
    std::printf("], \"spot_lights\": [");
    for (uint32_t i = 0; i < d->num_spot_lights; ++i) {
        const rtc_spot_light& l = d->spot_lights[i];
        std::printf("%s{", i ? ", " : "");
        arr3("position", l.position);
        arr3("direction", l.direction);
        arr3("color", l.color);
        std::printf("\"cutoff\": %.9g, \"falloff\": %.9g, \"radius\": %.9g, \"intensity\": %.9g, \"invisible\": %d}",
                    l.cutoff, l.falloff, l.radius, l.intensity, l.invisible);
    }
    std::printf("], \"spheres\": [");
    for (uint32_t i = 0; i < d->num_spheres; ++i) {
        const rtc_sphere& s = d->spheres[i];
        std::printf("%s{", i ? ", " : "");
        arr3("center", s.center);
        std::printf("\"radius\": %.9g, \"material\": %d}", s.radius, s.material);
    }
    std::printf("], \"quads\": [");
    for (uint32_t i = 0; i < d->num_quads; ++i) {
        const rtc_quad& q = d->quads[i];
        std::printf("%s{", i ? ", " : "");
        arr3("q", q.q);
        arr3("u", q.u);
        arr3("v", q.v);
        std::printf("\"material\": %d}", q.material);
    }
    std::printf("], \"boxes\": [");
    for (uint32_t i = 0; i < d->num_boxes; ++i) {
        const rtc_box& b = d->boxes[i];
        std::printf("%s{", i ? ", " : "");
        arr3("center", b.center);
        arr3("size", b.size);
        std::printf("\"material\": %d, \"transform\": %u}", b.material, b.transform);
    }
    std::printf("], \"transforms\": [");
    for (uint32_t i = 0; i < d->num_transforms; ++i) {
        const rtc_transform& x = d->transforms[i];
        std::printf("%s{", i ? ", " : "");
        arr3("translate", x.translate);
        arr3("rotate", x.rotate);
        arr3("scale", x.scale);
        std::printf("\"flags\": %u}", x.flags);
    }
    std::printf("], \"sphere_transforms\": [");
    for (uint32_t i = 0; d->sphere_transforms && i < d->num_spheres; ++i)
        std::printf("%s%u", i ? ", " : "", d->sphere_transforms[i]);
    std::printf("], \"meshes\": [");
    for (uint32_t i = 0; i < d->num_meshes; ++i) {
        const rtc_mesh& m = d->meshes[i];
        std::printf("%s{\"num_vertices\": %u, \"num_triangles\": %u, \"material\": %d, \"smooth\": %d, ", i ? ", " : "",
                    m.num_vertices, m.num_triangles, m.material, m.smooth);
        arr3("v0", m.vertices);
        arr3("v3", m.vertices + 9);
        std::printf("\"has_normals\": %d, \"i1\": %u}", m.normals ? 1 : 0, m.indices[1]);
    }
    std::printf("], \"camera\": {");
    arr3("look_from", d->camera.look_from);
    arr3("look_at", d->camera.look_at);
    arr3("up", d->camera.up);
    std::printf("\"vfov\": %.9g, \"aspect\": %.9g, \"aperture\": %.9g, \"focus\": %.9g}, ", d->camera.vfov,
                d->camera.aspect, d->camera.aperture, d->camera.focus);
    std::printf("\"background\": {\"kind\": %d, ", d->background.kind);
    arr3("color", d->background.color, false);
    std::printf("}, \"skipped\": [");
    for (size_t i = 0; i < h.skipped.size(); ++i) std::printf("%s\"%s\"", i ? ", " : "", h.skipped[i].c_str());
    std::printf("]}\n");
    return 0;
}
