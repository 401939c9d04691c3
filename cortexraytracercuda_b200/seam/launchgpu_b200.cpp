// launchgpu_b200.cpp - the reference's render call, served by the B200 library.
//
// This translation unit replaces flarive/CortexRaytracerCuda's core/src/gpu.cu in the reference's own
// build.  It defines the one function the rest of the reference calls into gpu.cu for,
//
//     void launchGPU(const sceneConfig&, int width, int height, int spp, int max_depth,
//                    int tx, int ty, const char* filepath, bool quietMode);
//
// declared by core/src/renderers/gpu_cuda_renderer.h:17 and defined at core/src/gpu.cu:2127, so the
// reference's main.cpp, srenderer, gpu_cuda_renderer and its scene loading compile and run unchanged:
// the sceneConfig is flattened by include/rtc_sceneconfig.hpp into an rtc_scene_desc and rendered by
// rtc_launchGPU (compat mode, seed 2580, the nvcc build's draw order, PNG with flipped rows).
//
// Differences from gpu.cu's launchGPU, by design:
//   * errors are printed to stderr and the call returns; gpu.cu calls cudaDeviceReset and exit(99)
//     (gpu.cu:119-129);
//   * tx, ty (the render kernel's 16x16 block shape) are not used: the library picks its own launch
//     shapes;
//   * nothing is printed per pixel (gpu.cu:801 prints "p x y r g b" for the desktop UI).
//
// Build (in the reference tree, in place of gpu.cu): compile this file with the reference's include
// paths plus this repository's include/, define RTC_SEAM_STB_IMPLEMENTATION in exactly one translation
// unit (gpu.cu, which held stb's implementation, is gone), and link librtc_b200.so.  oracle/Makefile's
// `cli` target does exactly that for the reference's command-line program.
#include <cstdio>
#include <vector>

#ifdef RTC_SEAM_STB_IMPLEMENTATION
#define STB_IMAGE_IMPLEMENTATION
#endif
#include "stb/stb_image.h"

#include "scenes/scene_config.h"
#include "rtc_sceneconfig.hpp"

void launchGPU(const sceneConfig& cfg, int width, int height, int spp, int max_depth, int tx, int ty,
               const char* filepath, bool quietMode) {
    // image textures: decoded RGB8, as load_images does (gpu.cu:1728-1770); kept alive until the render ends
    std::vector<unsigned char*> decoded;
    auto load_image = [&decoded](const char* path, int* w, int* h) -> const uint8_t* {
        int n = 0;
        unsigned char* px = stbi_load(path, w, h, &n, 3);
        if (px) decoded.push_back(px);
        return px;
    };
    // OBJ meshes: the library's reader (rtc_load_obj), in place of tinyobjloader (mesh_loader.cuh)
    auto load_obj = [](const char* path, std::vector<float>& v, std::vector<uint32_t>& idx, std::vector<float>& n,
                       std::vector<float>& uv) {
        rtc_obj_mesh m;
        if (rtc_load_obj(path, &m) != RTC_OK) return false;
        v.assign(m.vertices, m.vertices + 3 * (size_t)m.num_vertices);
        idx.assign(m.indices, m.indices + 3 * (size_t)m.num_triangles);
        if (m.normals) n.assign(m.normals, m.normals + 3 * (size_t)m.num_vertices);
        if (m.uvs) uv.assign(m.uvs, m.uvs + 2 * (size_t)m.num_vertices);
        rtc_free_obj(&m);
        return true;
    };
    rtc_adapter::SceneHolder holder;
    // the reference renders meshes[0] for every objMeshes entry, without position or transform (gpu.cu:626-631)
    const rtc_scene_desc* desc = rtc_adapter::from_sceneconfig(cfg, holder, load_image, load_obj,
                                                               rtc_adapter::REFERENCE_MESHES);
    if (!quietMode)
        for (const std::string& s : holder.skipped) std::fprintf(stderr, "[WARN] not rendered: %s\n", s.c_str());
    const rtc_status st = rtc_launchGPU(desc, width, height, spp, max_depth, tx, ty, filepath, quietMode ? 1 : 0);
    if (st != RTC_OK) std::fprintf(stderr, "[ERROR] launchGPU: %s\n", rtc_last_error_string());
    for (unsigned char* px : decoded) stbi_image_free(px);
}
