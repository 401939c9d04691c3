// rtc_obj.cpp - Wavefront OBJ geometry reader for rtc_mesh (rtc_load_obj / rtc_free_obj).
//
// The reference reads meshes with tinyobjloader inside its mesh loader (core/src/utilities/
// mesh_loader.cuh) and builds per-face triangle objects from shape 0 only (core/src/gpu.cu:628).  This
// reader takes the geometry statements of the format - `v x y z [w]`, `vt u [v [w]]`, `vn x y z` and
// `f` with `v`, `v/vt`, `v//vn` or `v/vt/vn` corners, negative (relative) indices allowed - merges every
// object and group, fan-triangulates polygons, and de-indexes the (v, vt, vn) corner triples into one
// vertex stream with 32-bit indices, the layout rtc_mesh takes.  Other statements (o, g, s, usemtl,
// mtllib, l, p, ...) are skipped.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/rtc.h"
#include "rtc_internal.h"

namespace {

struct Corner {
    int64_t v, t, n;   // 0-based, -1 = absent
    bool operator==(const Corner& o) const { return v == o.v && t == o.t && n == o.n; }
};
struct CornerHash {
    size_t operator()(const Corner& c) const {
        uint64_t h = (uint64_t)c.v * 0x9E3779B97F4A7C15ull;
        h ^= (uint64_t)(c.t + 1) * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
        h ^= (uint64_t)(c.n + 1) * 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};

rtc_status bad(int line, const std::string& what) {
    return rtc_set_error(RTC_ERR_BAD_SCENE, ("OBJ line " + std::to_string(line) + ": " + what).c_str());
}

// Resolves one index of a face corner: 1-based, or negative relative to the `count` elements so far.
bool resolve(const char* s, const char* e, int64_t count, int64_t& out) {
    if (s == e) return false;
    char* end = nullptr;
    const long long x = std::strtoll(s, &end, 10);
    if (end != e || x == 0) return false;
    out = x > 0 ? x - 1 : count + x;
    return out >= 0 && out < count;
}

}  // namespace

extern "C" rtc_status rtc_load_obj(const char* path, rtc_obj_mesh* out) {
    if (!path || !out) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "null argument");
    std::memset(out, 0, sizeof *out);
    FILE* f = std::fopen(path, "rb");
    if (!f) return rtc_set_error(RTC_ERR_IO, (std::string("cannot open ") + path + ": " + std::strerror(errno)).c_str());
    std::vector<float> V, T, N;   // as read: 3 per v, 2 per vt, 3 per vn
    std::vector<float> ov, on, ot;
    std::vector<uint32_t> idx;
    std::unordered_map<Corner, uint32_t, CornerHash> seen;
    bool any_t = false, any_n = false;
    std::vector<Corner> poly;
    std::string line;
    char buf[1 << 16];
    int lineno = 0;
    rtc_status st = RTC_OK;
    while (st == RTC_OK && std::fgets(buf, sizeof buf, f)) {
        line.assign(buf);
        while (!line.empty() && line.back() != '\n' && !std::feof(f)) {   // long line: read the rest
            if (!std::fgets(buf, sizeof buf, f)) break;
            line += buf;
        }
        ++lineno;
        const char* p = line.c_str();
        while (*p == ' ' || *p == '\t') ++p;
        if (p[0] == 'v' && (p[1] == ' ' || p[1] == '\t')) {
            float x = 0, y = 0, z = 0;
            if (std::sscanf(p + 2, "%f %f %f", &x, &y, &z) != 3) { st = bad(lineno, "vertex needs three coordinates"); break; }
            V.insert(V.end(), {x, y, z});
        } else if (p[0] == 'v' && p[1] == 't' && (p[2] == ' ' || p[2] == '\t')) {
            float u = 0, v = 0;
            const int k = std::sscanf(p + 3, "%f %f", &u, &v);
            if (k < 1) { st = bad(lineno, "texture coordinate needs u"); break; }
            T.insert(T.end(), {u, k >= 2 ? v : 0.0f});
        } else if (p[0] == 'v' && p[1] == 'n' && (p[2] == ' ' || p[2] == '\t')) {
            float x = 0, y = 0, z = 0;
            if (std::sscanf(p + 3, "%f %f %f", &x, &y, &z) != 3) { st = bad(lineno, "normal needs three components"); break; }
            N.insert(N.end(), {x, y, z});
        } else if (p[0] == 'f' && (p[1] == ' ' || p[1] == '\t')) {
            poly.clear();
            const char* q = p + 2;
            for (;;) {
                while (*q == ' ' || *q == '\t') ++q;
                if (*q == '\0' || *q == '\n' || *q == '\r' || *q == '#') break;
                const char* tok = q;
                while (*q && *q != ' ' && *q != '\t' && *q != '\n' && *q != '\r') ++q;
                const char* s1 = std::find(tok, q, '/');
                const char* s2 = s1 < q ? std::find(s1 + 1, q, '/') : q;
                Corner c{-1, -1, -1};
                if (!resolve(tok, s1, (int64_t)V.size() / 3, c.v)) { st = bad(lineno, "bad vertex index"); break; }
                if (s1 < q && s1 + 1 < s2 && !resolve(s1 + 1, s2, (int64_t)T.size() / 2, c.t)) {
                    st = bad(lineno, "bad texture-coordinate index");
                    break;
                }
                if (s2 < q && s2 + 1 < q && !resolve(s2 + 1, q, (int64_t)N.size() / 3, c.n)) {
                    st = bad(lineno, "bad normal index");
                    break;
                }
                poly.push_back(c);
            }
            if (st != RTC_OK) break;
            if (poly.size() < 3) { st = bad(lineno, "face with fewer than three corners"); break; }
            uint32_t ids[3];
            auto vid = [&](const Corner& c) -> uint32_t {
                auto it = seen.find(c);
                if (it != seen.end()) return it->second;
                const uint32_t id = (uint32_t)(ov.size() / 3);
                ov.insert(ov.end(), {V[3 * c.v], V[3 * c.v + 1], V[3 * c.v + 2]});
                if (c.t >= 0) { any_t = true; ot.insert(ot.end(), {T[2 * c.t], T[2 * c.t + 1]}); }
                else ot.insert(ot.end(), {0.0f, 0.0f});
                if (c.n >= 0) { any_n = true; on.insert(on.end(), {N[3 * c.n], N[3 * c.n + 1], N[3 * c.n + 2]}); }
                else on.insert(on.end(), {0.0f, 0.0f, 0.0f});
                seen.emplace(c, id);
                return id;
            };
            ids[0] = vid(poly[0]);
            for (size_t k = 1; k + 1 < poly.size(); ++k) {   // fan: (0, k, k+1)
                ids[1] = vid(poly[k]);
                ids[2] = vid(poly[k + 1]);
                idx.insert(idx.end(), {ids[0], ids[1], ids[2]});
            }
        }
        if (ov.size() / 3 > 0xfffffff0ull) { st = bad(lineno, "more than 2^32 vertices"); break; }
    }
    std::fclose(f);
    if (st != RTC_OK) return st;
    if (idx.empty()) return rtc_set_error(RTC_ERR_BAD_SCENE, (std::string("no faces in ") + path).c_str());
    auto dup = [](const std::vector<float>& v) {
        float* p = (float*)std::malloc(v.size() * sizeof(float));
        if (p) std::memcpy(p, v.data(), v.size() * sizeof(float));
        return p;
    };
    out->vertices = dup(ov);
    out->normals = any_n ? dup(on) : nullptr;
    out->uvs = any_t ? dup(ot) : nullptr;
    out->indices = (uint32_t*)std::malloc(idx.size() * sizeof(uint32_t));
    if (!out->vertices || !out->indices || (any_n && !out->normals) || (any_t && !out->uvs)) {
        rtc_free_obj(out);
        return rtc_set_error(RTC_ERR_OOM, "host allocation failed");
    }
    std::memcpy(out->indices, idx.data(), idx.size() * sizeof(uint32_t));
    out->num_vertices = (uint32_t)(ov.size() / 3);
    out->num_triangles = (uint32_t)(idx.size() / 3);
    return RTC_OK;
}

extern "C" void rtc_free_obj(rtc_obj_mesh* m) {
    if (!m) return;
    std::free(m->vertices);
    std::free(m->normals);
    std::free(m->uvs);
    std::free(m->indices);
    std::memset(m, 0, sizeof *m);
}
