// rtc_scene_file.cpp - reads the reference's `.scene` files (libconfig syntax) into an rtc_scene_desc
// (rtc_scene_file_load and friends).
//
// The reference parses them with libconfig++ (core/src/scenes/scene_loader.cpp:21-120) into a
// scene_builder, whose sceneConfig load_scene turns into objects (core/src/gpu.cu:481-751).  Here:
//   1. a parser for the libconfig grammar - settings `name = value` or `name : value` ended by `;` or
//      `,`, groups `{...}`, lists `(...)`, arrays `[...]`, integers (decimal, hex, L suffix), floats,
//      booleans, strings (escapes, adjacent literals joined), comments `#`, `//` and `/* */`;
//   2. the scene_loader's reading of it, section by section in its order (image, camera, lights,
//      textures, materials, primitives, meshes) into structures with sceneConfig's field names;
//   3. rtc_adapter::from_sceneconfig (include/rtc_sceneconfig.hpp), the same conversion a reference
//      caller uses, so a file read here and the reference's own sceneConfig of it give one description.
// Values follow libconfig's typing as scene_loader reads them (it never sets AutoConvert): a lookupValue
// of the wrong type keeps the loader's initial value, a setting handed straight to the builder with the
// wrong type throws, and so does a texture or material without a name or a primitive without a material;
// those throws become RTC_ERR_BAD_SCENE.  Defaults are scene_loader's and scene_builder's.
// Differences from scene_loader, all deliberate:
//   * every entry is kept.  scene_loader counts each list into a uint8_t and sizes the dielectric table
//     from a `dielectric` key while filling it from `glass` (scene_loader.cpp:191 and 1092), so the
//     reference keeps (length mod 256) entries of a kind and drops glass materials with the objects
//     using them; RTC_SCENE_FILE_REFERENCE_CAPACITY reproduces both;
//   * groups, transforms, and primitive, texture and material kinds the render path does not cover are
//     listed in the skipped notes (and not validated);
//   * relative file paths resolve against the scene file's directory, then the working directory (the
//     reference uses the working directory only);
//   * `@include` is refused.
#include <algorithm>
#include <cctype>
#include <climits>
#include <cstdint>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/rtc.h"
#include "../../include/rtc_sceneconfig.hpp"
#include "rtc_internal.h"

namespace {

// ---- libconfig document ---------------------------------------------------------------------------
struct Node {
    enum Kind { GROUP, LIST, ARRAY, INT, INT64, FLOAT, BOOL, STRING } kind = GROUP;
    int line = 0;
    long long i = 0;   // INT, INT64
    double f = 0.0;    // FLOAT
    bool b = false;    // BOOL
    std::string s;     // STRING
    std::vector<std::pair<std::string, std::unique_ptr<Node>>> members;   // GROUP
    std::vector<std::unique_ptr<Node>> items;                              // LIST / ARRAY

    // Setting::exists + operator[](name): members of a group only
    const Node* get(const char* name) const {
        for (const auto& m : members)
            if (m.first == name) return m.second.get();
        return nullptr;
    }
    bool scalar() const { return kind >= INT; }
    // Setting::getLength and operator[](index): the elements of a list or array, the members of a group
    size_t length() const {
        return kind == GROUP ? members.size() : (kind == LIST || kind == ARRAY) ? items.size() : 0;
    }
    const Node* elem(size_t k) const { return kind == GROUP ? members[k].second.get() : items[k].get(); }
};

// The libconfig grammar (libs/libconfig/lib/grammar.y, scanner.l) without @include: a setting is
// `name = value` or `name : value` with an optional `;` or `,` after it; names are
// [A-Za-z*][-A-Za-z0-9_*]*; a name repeated in one group is an error; lists and arrays take a trailing
// comma; an array holds scalars of the type of its first element.
struct Parser {
    const char* p;
    const char* end;
    int line = 1;
    std::string err;

    void skip() {
        for (;;) {
            while (p < end && std::isspace((unsigned char)*p)) { if (*p == '\n') ++line; ++p; }
            if (p < end && (*p == '#' || (*p == '/' && p + 1 < end && p[1] == '/'))) {
                while (p < end && *p != '\n') ++p;
                continue;
            }
            if (p + 1 < end && p[0] == '/' && p[1] == '*') {
                p += 2;
                while (p + 1 < end && !(p[0] == '*' && p[1] == '/')) { if (*p == '\n') ++line; ++p; }
                p = std::min(end, p + 2);
                continue;
            }
            return;
        }
    }
    bool fail(const std::string& m) {
        if (err.empty()) err = "line " + std::to_string(line) + ": " + m;
        return false;
    }
    static bool name_start(char c) { return std::isalpha((unsigned char)c) || c == '*'; }
    static bool name_char(char c) { return std::isalnum((unsigned char)c) || c == '_' || c == '-' || c == '*'; }

    bool settings(Node& g, char close) {
        for (;;) {
            skip();
            if (p >= end) return close == 0 ? true : fail("unexpected end of file");
            if (*p == close) { ++p; return true; }
            if (*p == '@') return fail("@include is not supported");
            if (!name_start(*p)) return fail(std::string("expected a setting name, found '") + *p + "'");
            const char* s0 = p;
            while (p < end && name_char(*p)) ++p;
            std::string name(s0, p);
            if (g.get(name.c_str())) return fail("duplicate setting name " + name);
            skip();
            if (p >= end || (*p != '=' && *p != ':')) return fail("expected '=' or ':' after " + name);
            ++p;
            auto v = std::make_unique<Node>();
            if (!value(*v)) return false;
            g.members.emplace_back(std::move(name), std::move(v));
            skip();
            if (p < end && (*p == ';' || *p == ',')) ++p;
        }
    }
    bool values(Node& n, char close, bool array) {
        skip();
        if (p < end && *p == close) { ++p; return true; }
        for (;;) {
            auto v = std::make_unique<Node>();
            if (!value(*v)) return false;
            if (array && !v->scalar()) return fail("an array holds scalar values only");
            if (array && !n.items.empty() && n.items[0]->kind != v->kind) return fail("mismatched element type in array");
            n.items.push_back(std::move(v));
            skip();
            if (p < end && *p == ',') {
                ++p;
                skip();
                if (p < end && *p == close) { ++p; return true; }
                continue;
            }
            if (p < end && *p == close) { ++p; return true; }
            return fail("expected ',' or a closing bracket");
        }
    }
    bool string(Node& n) {
        n.kind = Node::STRING;
        for (;;) {   // adjacent string literals are joined
            ++p;
            while (p < end && *p != '"') {
                if (*p == '\\' && p + 1 < end) {
                    static const char from[] = "abnrtvf\\\"";
                    static const char to[] = "\a\b\n\r\t\v\f\\\"";
                    const char e = p[1];
                    const char* esc = e != '\0' ? std::strchr(from, e) : nullptr;
                    if (esc) {
                        n.s += to[esc - from];
                        p += 2;
                        continue;
                    }
                    if ((e == 'x' || e == 'X') && p + 3 < end && std::isxdigit((unsigned char)p[2]) &&
                        std::isxdigit((unsigned char)p[3])) {
                        n.s += (char)std::strtol(std::string(p + 2, p + 4).c_str(), nullptr, 16);
                        p += 4;
                        continue;
                    }
                    n.s += '\\';   // any other backslash stays
                    ++p;
                    continue;
                }
                if (*p == '\n') ++line;
                n.s += *p++;
            }
            if (p >= end) return fail("unterminated string");
            ++p;
            const char* save = p;
            const int save_line = line;
            skip();
            if (p < end && *p == '"') continue;
            p = save;
            line = save_line;
            return true;
        }
    }
    // scanner.l's integer, integer64, hex, hex64 and float tokens
    static bool number(const std::string& t, Node& n) {
        auto digits = [&](size_t& j, bool hex) {
            const size_t j0 = j;
            while (j < t.size() && (hex ? std::isxdigit((unsigned char)t[j]) : std::isdigit((unsigned char)t[j]))) ++j;
            return j - j0;
        };
        auto suffix64 = [](const std::string& x) { return x == "L" || x == "LL"; };
        if (t.size() > 2 && t[0] == '0' && (t[1] == 'x' || t[1] == 'X')) {
            size_t j = 2;
            if (!digits(j, true)) return false;
            const std::string suf = t.substr(j);
            const unsigned long long v = std::strtoull(t.c_str() + 2, nullptr, 16);
            if (suf.empty()) { n.kind = Node::INT; n.i = (int32_t)(uint32_t)v; return true; }   // strtoul into an int
            if (!suffix64(suf)) return false;
            n.kind = Node::INT64;
            n.i = (long long)v;
            return true;
        }
        size_t j = (!t.empty() && (t[0] == '+' || t[0] == '-')) ? 1 : 0;
        const size_t int_digits = digits(j, false);
        bool dot = false, exp = false;
        if (j < t.size() && t[j] == '.') { dot = true; ++j; digits(j, false); }
        if (j < t.size() && (t[j] == 'e' || t[j] == 'E')) {
            ++j;
            if (j < t.size() && (t[j] == '+' || t[j] == '-')) ++j;
            if (!digits(j, false)) return false;
            exp = true;
        }
        const std::string suf = t.substr(j);
        if (!dot && !exp) {
            if (!int_digits) return false;
            if (suffix64(suf)) { n.kind = Node::INT64; n.i = std::atoll(t.c_str()); return true; }
            if (!suf.empty()) return false;
            char* e = nullptr;
            errno = 0;
            const long long v = std::strtoll(t.c_str(), &e, 0);   // base 0: a leading 0 reads octal
            if (*e || errno) return false;
            n.kind = (v < INT_MIN || v > INT_MAX) ? Node::INT64 : Node::INT;
            n.i = v;
            return true;
        }
        if (!suf.empty() || (!dot && !int_digits)) return false;
        n.kind = Node::FLOAT;
        n.f = std::atof(t.c_str());
        return true;
    }
    bool value(Node& n) {
        skip();
        if (p >= end) return fail("expected a value");
        n.line = line;
        const char c = *p;
        if (c == '{') { ++p; n.kind = Node::GROUP; return settings(n, '}'); }
        if (c == '(') { ++p; n.kind = Node::LIST; return values(n, ')', false); }
        if (c == '[') { ++p; n.kind = Node::ARRAY; return values(n, ']', true); }
        if (c == '"') return string(n);
        const char* s0 = p;
        while (p < end && (std::isalnum((unsigned char)*p) || *p == '.' || *p == '-' || *p == '+' || *p == '_')) ++p;
        std::string tok(s0, p);
        if (tok.empty()) return fail(std::string("unexpected '") + c + "'");
        std::string low = tok;
        for (char& ch : low) ch = (char)std::tolower((unsigned char)ch);
        if (low == "true" || low == "false") { n.kind = Node::BOOL; n.b = low == "true"; return true; }
        if (number(tok, n)) return true;
        return fail("bad value '" + tok + "'");
    }
};

// ---- sceneConfig-shaped structures (the field names rtc_adapter::from_sceneconfig reads) -----------
struct V3 { float x = 0, y = 0, z = 0; };
struct Col {
    float c[3] = {0, 0, 0};
    float r() const { return c[0]; }
    float g() const { return c[1]; }
    float b() const { return c[2]; }
};
struct SolidTex { const char* name; Col rgb; };
struct ImageTex { const char* name; const char* filepath; };
struct CheckerTex { const char* name; const char* oddTextureName; const char* evenTextureName; Col oddColor, evenColor; float scale; };
struct Lambertian { const char* name; const char* textureName; Col rgb; };
struct Metal { const char* name; Col rgb; float fuzziness; };
struct Dielectric { const char* name; float refraction; };
struct DirLight { V3 position, u, v; float intensity; Col rgb; bool invisible; };
struct OmniLight { V3 position; float radius, intensity; Col rgb; bool invisible; };
struct SpotLight { V3 position, direction; float cutoff, falloff, intensity, radius; Col rgb; bool invisible; };
// rt::transform (misc/transform.cuh): the parts a `transform` group sets
struct Xf {
    bool t = false, r = false, s = false;
    V3 tv, rv, sv;
    bool hasTranslate() const { return t; }
    bool hasRotate() const { return r; }
    bool hasScale() const { return s; }
    V3 getTranslate() const { return tv; }
    V3 getRotate() const { return rv; }
    V3 getScale() const { return sv; }
};
struct SpherePrim { const char* materialName; V3 position; float radius; Xf transform; };
struct QuadPrim { const char* materialName; V3 position, u, v; Xf transform; };
struct BoxPrim { const char* materialName; V3 position, size; Xf transform; };
struct ObjMesh { const char* filepath; const char* materialName; V3 position; bool use_mtl, use_smoothing; Xf transform; };

struct Config {
    struct { std::vector<SolidTex> s; std::vector<ImageTex> im; std::vector<CheckerTex> ch;
             int solidColorTextureCount = 0, imageTextureCount = 0, checkerTextureCount = 0;
             const SolidTex* solidColorTextures = nullptr; const ImageTex* imageTextures = nullptr;
             const CheckerTex* checkerTextures = nullptr; } texturesCfg;
    struct { std::vector<Lambertian> l; std::vector<Metal> m; std::vector<Dielectric> d;
             int lambertianMaterialCount = 0, metalMaterialCount = 0, dielectricMaterialCount = 0;
             const Lambertian* lambertianMaterials = nullptr; const Metal* metalMaterials = nullptr;
             const Dielectric* dielectricMaterials = nullptr; } materialsCfg;
    struct { std::vector<DirLight> d; std::vector<OmniLight> o; std::vector<SpotLight> s;
             int dirLightCount = 0, omniLightCount = 0, spotLightCount = 0;
             const DirLight* dirLights = nullptr; const OmniLight* omniLights = nullptr;
             const SpotLight* spotLights = nullptr; } lightsCfg;
    struct { std::vector<SpherePrim> s; std::vector<QuadPrim> q; std::vector<BoxPrim> b;
             int spherePrimitiveCount = 0, quadPrimitiveCount = 0, planePrimitiveCount = 0, boxPrimitiveCount = 0,
                 conePrimitiveCount = 0, cylinderPrimitiveCount = 0, diskPrimitiveCount = 0, torusPrimitiveCount = 0,
                 volumePrimitiveCount = 0;
             const SpherePrim* spherePrimitives = nullptr; const QuadPrim* quadPrimitives = nullptr;
             const BoxPrim* boxPrimitives = nullptr; } primitivesCfg;
    struct { std::vector<ObjMesh> o; int objMeshCount = 0; const ObjMesh* objMeshes = nullptr; } meshesCfg;
    struct { V3 lookFrom{0, 0, 10}, lookAt, upAxis{0, 1, 0}; float fov = 70, aspectRatio = 16.0f / 9.0f, aperture = 0,
             focus = 100; } cameraCfg;   // scene_builder's defaults (scene_builder.cpp:49)
    struct { struct { Col rgb; } background; int width = 0, height = 0, depth = 0, spp = 0; } imageCfg;
    std::vector<std::unique_ptr<std::string>> strings;   // storage behind the const char* fields

    void link() {
        auto& T = texturesCfg;
        T.solidColorTextures = T.s.data(); T.solidColorTextureCount = (int)T.s.size();
        T.imageTextures = T.im.data(); T.imageTextureCount = (int)T.im.size();
        T.checkerTextures = T.ch.data(); T.checkerTextureCount = (int)T.ch.size();
        auto& M = materialsCfg;
        M.lambertianMaterials = M.l.data(); M.lambertianMaterialCount = (int)M.l.size();
        M.metalMaterials = M.m.data(); M.metalMaterialCount = (int)M.m.size();
        M.dielectricMaterials = M.d.data(); M.dielectricMaterialCount = (int)M.d.size();
        auto& L = lightsCfg;
        L.dirLights = L.d.data(); L.dirLightCount = (int)L.d.size();
        L.omniLights = L.o.data(); L.omniLightCount = (int)L.o.size();
        L.spotLights = L.s.data(); L.spotLightCount = (int)L.s.size();
        auto& P = primitivesCfg;
        P.spherePrimitives = P.s.data(); P.spherePrimitiveCount = (int)P.s.size();
        P.quadPrimitives = P.q.data(); P.quadPrimitiveCount = (int)P.q.size();
        P.boxPrimitives = P.b.data(); P.boxPrimitiveCount = (int)P.b.size();
        meshesCfg.objMeshes = meshesCfg.o.data();
        meshesCfg.objMeshCount = (int)meshesCfg.o.size();
    }
    const char* keep(const std::string& s) {
        strings.push_back(std::make_unique<std::string>(s));
        return strings.back()->c_str();
    }
};

// Raised where scene_loader's reading throws (a setting passed straight to the builder with the wrong
// type, a texture or material without a name); rtc_scene_file_load returns it as RTC_ERR_BAD_SCENE.
struct SceneError {
    std::string msg;
};

const Node* member(const Node* g, const char* key) { return g ? g->get(key) : nullptr; }

// Setting::lookupValue: true only when the member exists with the requested type.  scene_loader never
// sets libconfig's AutoConvert option, so an integer where a float is read (or the reverse) fails and the
// caller's initial value stays.
bool look(const Node* g, const char* key, float& v) {
    const Node* n = member(g, key);
    if (!n || n->kind != Node::FLOAT) return false;
    v = (float)n->f;
    return true;
}
bool look(const Node* g, const char* key, int& v) {
    const Node* n = member(g, key);
    if (!n || (n->kind != Node::INT && n->kind != Node::INT64) || n->i < INT_MIN || n->i > INT_MAX) return false;
    v = (int)n->i;
    return true;
}
bool look(const Node* g, const char* key, bool& v) {
    const Node* n = member(g, key);
    if (!n || n->kind != Node::BOOL) return false;
    v = n->b;
    return true;
}
bool look(const Node* g, const char* key, std::string& v) {
    const Node* n = member(g, key);
    if (!n || n->kind != Node::STRING) return false;
    v = n->s;
    return true;
}

// Setting's conversion operators, where scene_loader hands setting["key"] to the builder: the wrong type
// throws (libconfig's SettingTypeException / SettingRangeException).
[[noreturn]] void wrong(const Node& n, const char* key, const char* what) {
    throw SceneError{"line " + std::to_string(n.line) + ": setting '" + key + "' " + what};
}
int as_int(const Node* g, const char* key) {
    const Node& n = *member(g, key);
    if (n.kind != Node::INT && n.kind != Node::INT64) wrong(n, key, "is not an integer");
    if (n.i < INT_MIN || n.i > INT_MAX) wrong(n, key, "is out of range");
    return (int)n.i;
}
float as_float(const Node* g, const char* key) {
    const Node& n = *member(g, key);
    if (n.kind != Node::FLOAT) wrong(n, key, "is not a float");
    return (float)n.f;
}
bool as_bool(const Node* g, const char* key) {
    const Node& n = *member(g, key);
    if (n.kind != Node::BOOL) wrong(n, key, "is not a boolean");
    return n.b;
}
std::string as_string(const Node* g, const char* key) {
    const Node& n = *member(g, key);
    if (n.kind != Node::STRING) wrong(n, key, "is not a string");
    return n.s;
}

// scene_loader::getPoint / getVector (scene_loader.cpp:1530-1620): a float, else an integer, per axis
V3 point(const Node* n) {
    V3 v;
    float* a[3] = {&v.x, &v.y, &v.z};
    const char* k[3] = {"x", "y", "z"};
    for (int i = 0; i < 3; ++i) {
        if (look(n, k[i], *a[i])) continue;
        int w = 0;
        if (look(n, k[i], w)) *a[i] = (float)w;
    }
    return v;
}
// scene_loader::getTransform (scene_loader.cpp:1692-1704): translate, rotate and scale read as vectors
// (so `scale = 4.0;`, not a group, sets a zero scale, as in the reference)
Xf transform_of(const Node& n) {
    Xf x;
    const Node* g = n.get("transform");
    if (!g) return x;
    if (g->get("translate")) { x.t = true; x.tv = point(g->get("translate")); }
    if (g->get("rotate")) { x.r = true; x.rv = point(g->get("rotate")); }
    if (g->get("scale")) { x.s = true; x.sv = point(g->get("scale")); }
    return x;
}
// scene_loader::getColor (scene_loader.cpp:1622-1656): three non-negative integers are 0-255 values;
// otherwise the float components (an integer component reads as 0)
Col color(const Node* n) {
    int r1 = -1, g1 = -1, b1 = -1;
    look(n, "r", r1);
    look(n, "g", g1);
    look(n, "b", b1);
    Col c;
    if (r1 >= 0 && g1 >= 0 && b1 >= 0) {
        c.c[0] = r1 / 255.0f;
        c.c[1] = g1 / 255.0f;
        c.c[2] = b1 / 255.0f;
        return c;
    }
    look(n, "r", c.c[0]);
    look(n, "g", c.c[1]);
    look(n, "b", c.c[2]);
    return c;
}
// getRatio (utilities/math_utils.cuh:135-162): "W:H" split at ':', std::stof on the first two pieces,
// W/H when both are positive, else 0
float ratio(const Node* cam, const char* key) {
    const std::string s = as_string(cam, key);
    std::vector<std::string> piece;   // as std::getline(..., ':') reads them: no empty piece after a final ':'
    for (size_t at = 0; at < s.size();) {
        const size_t c = s.find(':', at);
        piece.push_back(s.substr(at, c == std::string::npos ? std::string::npos : c - at));
        if (c == std::string::npos) break;
        at = c + 1;
    }
    float part[2] = {0.0f, 0.0f};
    for (size_t k = 0; k < piece.size() && k < 2; ++k) {
        char* e = nullptr;
        errno = 0;
        part[k] = std::strtof(piece[k].c_str(), &e);
        if (e == piece[k].c_str() || errno == ERANGE) wrong(*member(cam, key), key, "is not a ratio W:H");
    }
    return (part[0] > 0 && part[1] > 0) ? part[0] / part[1] : 0.0f;
}
// each element of setting `key` of group g (Setting::getLength / operator[])
template <class F> void each(const Node* g, const char* key, F f) {
    const Node* n = member(g, key);
    if (!n) return;
    for (size_t k = 0; k < n->length(); ++k) f(*n->elem(k));
}
size_t count(const Node* g, const char* key) {
    const Node* n = member(g, key);
    return n ? n->length() : 0;
}

}  // namespace

struct rtc_scene_file {
    Config cfg;
    rtc_adapter::SceneHolder holder;
    std::vector<std::unique_ptr<uint8_t, void (*)(void*)>> pixels;   // decoded images (loader-allocated)
    std::vector<std::string> skipped;
    rtc_scene_file_info info{};
    const rtc_scene_desc* desc = nullptr;
};

namespace {

std::string resolve(const std::string& dir, const std::string& path) {
    if (path.empty() || path[0] == '/') return path;
    const std::string near = dir.empty() ? path : dir + "/" + path;
    if (FILE* f = std::fopen(near.c_str(), "rb")) { std::fclose(f); return near; }
    return path;
}

rtc_status read_file(rtc_scene_file& F, const char* path, uint32_t flags, rtc_image_loader load_image, void* user) {
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return rtc_set_error(RTC_ERR_IO, (std::string("cannot open ") + path + ": " + std::strerror(errno)).c_str());
    std::string text;
    char buf[1 << 15];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof buf, fp)) > 0) text.append(buf, k);
    std::fclose(fp);
    Node root;
    Parser P{text.data(), text.data() + text.size(), 1, {}};
    if (!P.settings(root, 0)) return rtc_set_error(RTC_ERR_BAD_SCENE, (std::string(path) + ": " + P.err).c_str());
    std::string dir = path;
    const size_t slash = dir.find_last_of('/');
    dir = slash == std::string::npos ? std::string() : dir.substr(0, slash);

    Config& C = F.cfg;
    auto skip = [&](const std::string& what) { F.skipped.push_back(what); };
    const bool limits = (flags & RTC_SCENE_FILE_REFERENCE_CAPACITY) != 0;
    // a kind's table capacity: scene_loader counts each list into a uint8_t (scene_loader.cpp:124-204)
    auto cap = [&](const Node* g, const char* key) { return limits ? (count(g, key) & 255u) : SIZE_MAX; };
    auto full = [&](size_t n, size_t c, const char* what) {
        if (n < c) return false;
        skip(std::string("beyond the table capacity: ") + what);
        return true;
    };
    auto exists = [](const std::string& fp) {
        FILE* f = std::fopen(fp.c_str(), "rb");
        if (f) std::fclose(f);
        return f != nullptr;
    };
    // image (scene_loader.cpp:300-333); scene_builder's defaults (scene_builder.cpp:46)
    F.info.width = 400;
    F.info.height = 225;
    F.info.max_depth = 100;
    F.info.spp = 50;
    if (const Node* im = root.get("image")) {
        if (im->get("width")) F.info.width = as_int(im, "width");
        if (im->get("height")) F.info.height = as_int(im, "height");
        if (im->get("maxDepth")) F.info.max_depth = as_int(im, "maxDepth");
        if (im->get("samplesPerPixel")) F.info.spp = as_int(im, "samplesPerPixel");
        if (const Node* bg = im->get("background")) {
            if (bg->get("color")) C.imageCfg.background.rgb = color(bg->get("color"));
            std::string fp;
            if (look(bg, "filepath", fp) && !fp.empty()) skip("background image (the render path uses the background colour)");
        }
        if (im->get("outputFilePath")) as_string(im, "outputFilePath");
    }
    // camera (scene_loader.cpp:335-367)
    if (const Node* cam = root.get("camera")) {
        auto& K = C.cameraCfg;
        if (cam->get("aspectRatio")) K.aspectRatio = ratio(cam, "aspectRatio");
        if (cam->get("openingTime")) as_float(cam, "openingTime");
        if (cam->get("lookFrom")) K.lookFrom = point(cam->get("lookFrom"));
        if (cam->get("lookAt")) K.lookAt = point(cam->get("lookAt"));
        if (cam->get("upAxis")) K.upAxis = point(cam->get("upAxis"));
        if (cam->get("aperture")) K.aperture = as_float(cam, "aperture");
        if (cam->get("focus")) K.focus = as_float(cam, "focus");
        if (cam->get("fov")) K.fov = as_float(cam, "fov");
        if (cam->get("orthographic") && as_bool(cam, "orthographic")) skip("orthographic camera (rendered as perspective)");
        if (cam->get("orthoHeight")) as_float(cam, "orthoHeight");
    }
    // lights (scene_loader.cpp:278-298, 782-915)
    if (const Node* L = root.get("lights")) {
        const size_t cd = cap(L, "directionals"), co = cap(L, "omnis"), cs = cap(L, "spots");
        each(L, "directionals", [&](const Node& n) {
            DirLight d{point(n.get("position")), point(n.get("u")), point(n.get("v")), 0.0f, color(n.get("color")), true};
            bool active = true;
            look(&n, "intensity", d.intensity);
            look(&n, "invisible", d.invisible);
            look(&n, "active", active);
            if (active && !full(C.lightsCfg.d.size(), cd, "directional light")) C.lightsCfg.d.push_back(d);
        });
        each(L, "omnis", [&](const Node& n) {
            OmniLight o{point(n.get("position")), 0.0f, 0.0f, color(n.get("color")), true};
            bool active = true;
            look(&n, "radius", o.radius);
            look(&n, "intensity", o.intensity);
            look(&n, "invisible", o.invisible);
            look(&n, "active", active);
            if (active && !full(C.lightsCfg.o.size(), co, "omni light")) C.lightsCfg.o.push_back(o);
        });
        each(L, "spots", [&](const Node& n) {
            SpotLight t{point(n.get("position")), point(n.get("direction")), 0.0f, 0.0f, 0.0f, 0.0f, color(n.get("color")), true};
            bool active = true;
            look(&n, "cutoff", t.cutoff);
            look(&n, "falloff", t.falloff);
            look(&n, "intensity", t.intensity);
            look(&n, "radius", t.radius);
            look(&n, "invisible", t.invisible);
            look(&n, "active", active);
            if (active && !full(C.lightsCfg.s.size(), cs, "spot light")) C.lightsCfg.s.push_back(t);
        });
    }
    // textures (scene_loader.cpp:218-277, 466-592); a texture or material without a name throws there
    auto named = [&](const Node& n, const char* what) {
        std::string name;
        look(&n, "name", name);
        if (name.empty()) throw SceneError{"line " + std::to_string(n.line) + ": " + what + " name is empty"};
        return name;
    };
    if (const Node* T = root.get("textures")) {
        const size_t cs = cap(T, "solidColor"), ci = cap(T, "image"), cc = cap(T, "checker");
        each(T, "solidColor", [&](const Node& n) {
            const std::string name = named(n, "Solid color texture");
            if (!full(C.texturesCfg.s.size(), cs, "solid colour texture"))
                C.texturesCfg.s.push_back(SolidTex{C.keep(name), color(n.get("color"))});
        });
        bool missing = false;   // the first missing image file ends the image textures (scene_loader.cpp:494-498)
        each(T, "image", [&](const Node& n) {
            const std::string name = named(n, "Image texture");
            std::string fp;
            look(&n, "filepath", fp);
            if (missing || fp.empty()) return;
            fp = resolve(dir, fp);
            if (!exists(fp)) {
                missing = true;
                skip("image texture file not found (later image textures are left out): " + fp);
                return;
            }
            if (!full(C.texturesCfg.im.size(), ci, "image texture"))
                C.texturesCfg.im.push_back(ImageTex{C.keep(name), C.keep(fp)});
        });
        each(T, "checker", [&](const Node& n) {
            const std::string name = named(n, "Checker texture");
            CheckerTex c{nullptr, nullptr, nullptr, color(n.get("oddColor")), color(n.get("evenColor")), 0.0f};
            std::string odd, even;
            look(&n, "scale", c.scale);
            look(&n, "oddTextureName", odd);
            look(&n, "evenTextureName", even);
            c.name = C.keep(name);
            c.oddTextureName = C.keep(odd);
            c.evenTextureName = C.keep(even);
            if (!full(C.texturesCfg.ch.size(), cc, "checker texture")) C.texturesCfg.ch.push_back(c);
        });
        for (const char* k : {"noise", "gradientColor", "bump", "normal", "displacement", "alpha", "emissive"})
            if (count(T, k)) skip(std::string(k) + " textures");
    }
    // materials (scene_loader.cpp:175-216, 916-1137).  The reference sizes the dielectric table from a
    // `dielectric` key and fills it from `glass` (scene_loader.cpp:191 and 1092).
    if (const Node* M = root.get("materials")) {
        const size_t cl = cap(M, "lambertian"), cm = cap(M, "metal"), cd = cap(M, "dielectric");
        each(M, "lambertian", [&](const Node& n) {
            const std::string name = named(n, "Material");
            std::string tex;
            look(&n, "texture", tex);
            if (!full(C.materialsCfg.l.size(), cl, "lambertian material"))
                C.materialsCfg.l.push_back(Lambertian{C.keep(name), C.keep(tex), color(n.get("color"))});
        });
        each(M, "metal", [&](const Node& n) {
            const std::string name = named(n, "Material");
            Metal m{nullptr, color(n.get("color")), 0.0f};
            look(&n, "fuzziness", m.fuzziness);
            m.name = C.keep(name);
            if (!full(C.materialsCfg.m.size(), cm, "metal material")) C.materialsCfg.m.push_back(m);
        });
        each(M, "glass", [&](const Node& n) {
            const std::string name = named(n, "Material");
            Dielectric d{nullptr, 0.0f};
            look(&n, "refraction", d.refraction);
            d.name = C.keep(name);
            if (!full(C.materialsCfg.d.size(), cd, "glass material (the reference sizes it from `dielectric`)"))
                C.materialsCfg.d.push_back(d);
        });
        for (const char* k : {"isotropic", "anisotropic", "orennayar", "phong"})
            if (count(M, k)) skip(std::string(k) + " materials");
    }
    // primitives (scene_loader.cpp:122-174, 1138-1308): spheres, quads and boxes with their transforms;
    // one without a material throws
    if (const Node* P2 = root.get("primitives")) {
        bool grouped = false, mapped = false;
        auto common = [&](const Node& n, std::string& mat) {
            look(&n, "material", mat);
            if (mat.empty()) throw SceneError{"line " + std::to_string(n.line) + ": Material name is empty"};
            bool active = true;
            look(&n, "active", active);
            std::string group;
            look(&n, "group", group);
            if (active && !group.empty()) grouped = true;
            if (active && n.get("uvmapping")) mapped = true;
            return active;
        };
        const size_t cs = cap(P2, "spheres"), cq = cap(P2, "quads"), cb = cap(P2, "boxes");
        each(P2, "spheres", [&](const Node& n) {
            SpherePrim sp{nullptr, point(n.get("position")), 0.0f, {}};
            look(&n, "radius", sp.radius);
            std::string mat;
            if (!common(n, mat) || full(C.primitivesCfg.s.size(), cs, "sphere")) return;
            sp.materialName = C.keep(mat);
            sp.transform = transform_of(n);
            C.primitivesCfg.s.push_back(sp);
        });
        each(P2, "quads", [&](const Node& n) {
            QuadPrim q{nullptr, point(n.get("position")), point(n.get("u")), point(n.get("v")), {}};
            std::string mat;
            if (!common(n, mat) || full(C.primitivesCfg.q.size(), cq, "quad")) return;
            q.materialName = C.keep(mat);
            q.transform = transform_of(n);
            C.primitivesCfg.q.push_back(q);
        });
        each(P2, "boxes", [&](const Node& n) {
            BoxPrim b{nullptr, point(n.get("position")), point(n.get("size")), {}};
            std::string mat;
            if (!common(n, mat) || full(C.primitivesCfg.b.size(), cb, "box")) return;
            b.materialName = C.keep(mat);
            b.transform = transform_of(n);
            C.primitivesCfg.b.push_back(b);
        });
        auto& PC = C.primitivesCfg;
        PC.planePrimitiveCount = (int)count(P2, "planes");
        PC.conePrimitiveCount = (int)count(P2, "cones");
        PC.cylinderPrimitiveCount = (int)count(P2, "cylinders");
        PC.diskPrimitiveCount = (int)count(P2, "disks");
        PC.torusPrimitiveCount = (int)count(P2, "toruses");
        PC.volumePrimitiveCount = (int)count(P2, "volumes");
        if (grouped) skip("groups of primitives (the reference's loadGroups reads none)");
        if (mapped) skip("uv mappings of primitives (the render path uses the default mapping)");
    }
    // meshes (scene_loader.cpp:369-435): the first missing OBJ file ends the meshes
    if (const Node* MS = root.get("meshes")) {
        const size_t cm = cap(MS, "obj");
        bool missing = false;
        each(MS, "obj", [&](const Node& n) {
            if (missing) return;
            std::string fp, mat;
            bool use_mtl = true, smooth = true, active = true;
            look(&n, "filepath", fp);
            look(&n, "material", mat);
            look(&n, "use_mtl", use_mtl);
            look(&n, "use_smoothing", smooth);
            look(&n, "active", active);
            fp = resolve(dir, fp);
            if (!fp.empty() && !exists(fp)) {
                missing = true;
                skip("obj file not found (later meshes are left out): " + fp);
                return;
            }
            if (!active || full(C.meshesCfg.o.size(), cm, "OBJ mesh")) return;
            C.meshesCfg.o.push_back(ObjMesh{C.keep(fp), C.keep(mat), point(n.get("position")), use_mtl, smooth,
                                            transform_of(n)});
        });
    }
    if (root.get("groups")) skip("groups");
    C.link();

    auto img = [&](const char* fp, int* w, int* h) -> const uint8_t* {
        if (!load_image) return nullptr;
        uint8_t* px = load_image(fp, w, h, user);
        if (px) F.pixels.emplace_back(px, std::free);
        return px;
    };
    auto obj = [&](const char* fp, std::vector<float>& v, std::vector<uint32_t>& idx, std::vector<float>& nrm,
                   std::vector<float>& uv) -> bool {
        rtc_obj_mesh m{};
        if (rtc_load_obj(fp, &m) != RTC_OK) return false;
        v.assign(m.vertices, m.vertices + 3 * (size_t)m.num_vertices);
        idx.assign(m.indices, m.indices + 3 * (size_t)m.num_triangles);
        if (m.normals) nrm.assign(m.normals, m.normals + 3 * (size_t)m.num_vertices);
        if (m.uvs) uv.assign(m.uvs, m.uvs + 2 * (size_t)m.num_vertices);
        rtc_free_obj(&m);
        return true;
    };
    F.desc = rtc_adapter::from_sceneconfig(C, F.holder, load_image ? rtc_adapter::ImageLoader(img) : nullptr, obj,
                                           (flags & RTC_SCENE_FILE_REFERENCE_MESHES) ? rtc_adapter::REFERENCE_MESHES : 0u);
    for (const auto& s : F.holder.skipped) F.skipped.push_back(s);
    F.info.num_skipped = (uint32_t)F.skipped.size();
    return RTC_OK;
}

}  // namespace

extern "C" rtc_status rtc_scene_file_load(const char* path, uint32_t flags, rtc_image_loader load_image, void* user,
                                          rtc_scene_file** out) {
    if (!path || !out) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    std::unique_ptr<rtc_scene_file> F(new (std::nothrow) rtc_scene_file());
    if (!F) return rtc_set_error(RTC_ERR_OOM, "host allocation failed");
    rtc_status r;
    try {
        r = read_file(*F, path, flags, load_image, user);
    } catch (const SceneError& e) {
        return rtc_set_error(RTC_ERR_BAD_SCENE, (std::string(path) + ": " + e.msg).c_str());
    } catch (const std::bad_alloc&) {
        return rtc_set_error(RTC_ERR_OOM, "host allocation failed");
    }
    if (r != RTC_OK) return r;
    *out = F.release();
    return RTC_OK;
}

extern "C" const rtc_scene_desc* rtc_scene_file_desc(const rtc_scene_file* f) { return f ? f->desc : nullptr; }

extern "C" rtc_status rtc_scene_file_get_info(const rtc_scene_file* f, rtc_scene_file_info* info) {
    if (!f || !info) return rtc_set_error(RTC_ERR_INVALID_ARGUMENT, "null argument");
    *info = f->info;
    return RTC_OK;
}

extern "C" const char* rtc_scene_file_skipped(const rtc_scene_file* f, uint32_t i) {
    return (f && i < f->skipped.size()) ? f->skipped[i].c_str() : nullptr;
}

extern "C" void rtc_scene_file_free(rtc_scene_file* f) { delete f; }
