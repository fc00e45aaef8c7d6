// sceneload.cu -- host side only: the reference's JSON scene files (SceneLoader,
// src/scene/sceneloader.cpp:11-131, 346-443) read into an AsimSceneDesc, with box and OBJ solids
// registered as static meshes (mesh.cu).  The reference parses with jsoncpp; this file carries
// its own small JSON reader (RFC 8259 values; for a repeated key the last value counts).
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/ariel.h"

namespace {

// ------------------------------------------------------------------------------------------
// JSON values and reader
// ------------------------------------------------------------------------------------------
struct JVal {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<JVal> arr;
    std::vector<std::pair<std::string, JVal>> obj;

    const JVal* get(const char* key) const {
        if (kind != Obj) return nullptr;
        for (auto it = obj.rbegin(); it != obj.rend(); ++it)
            if (it->first == key) return &it->second;
        return nullptr;
    }
    bool has(const char* key) const { return get(key) != nullptr; }
    // Python truthiness, as the reference's optional lists are tested
    bool truthy() const {
        switch (kind) {
            case Null: return false;
            case Bool: return b;
            case Num: return num != 0.0;
            case Str: return !str.empty();
            case Arr: return !arr.empty();
            case Obj: return !obj.empty();
        }
        return false;
    }
};

struct SceneFail {
    std::string why;
};

[[noreturn]] void fail(const std::string& why) { throw SceneFail{why}; }

class Reader {
   public:
    explicit Reader(const std::string& text) : s_(text) {}

    JVal document() {
        JVal v = value(0);
        ws();
        if (i_ != s_.size()) fail("JSON: trailing characters at offset " + std::to_string(i_));
        return v;
    }

   private:
    const std::string& s_;
    size_t i_ = 0;

    void ws() {
        while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\t' || s_[i_] == '\n' || s_[i_] == '\r')) ++i_;
    }
    [[noreturn]] void bad(const char* what) { fail(std::string("JSON: ") + what + " at offset " + std::to_string(i_)); }
    bool lit(const char* w) {
        size_t n = std::strlen(w);
        if (s_.compare(i_, n, w) == 0) {
            i_ += n;
            return true;
        }
        return false;
    }

    JVal value(int depth) {
        if (depth > 256) bad("nesting too deep");
        ws();
        if (i_ >= s_.size()) bad("unexpected end");
        JVal v;
        const char c = s_[i_];
        if (c == '{') {
            v.kind = JVal::Obj;
            ++i_;
            ws();
            if (i_ < s_.size() && s_[i_] == '}') {
                ++i_;
                return v;
            }
            for (;;) {
                ws();
                if (i_ >= s_.size() || s_[i_] != '"') bad("expected a key");
                std::string key = string();
                ws();
                if (i_ >= s_.size() || s_[i_] != ':') bad("expected ':'");
                ++i_;
                v.obj.emplace_back(std::move(key), value(depth + 1));
                ws();
                if (i_ < s_.size() && s_[i_] == ',') {
                    ++i_;
                    continue;
                }
                if (i_ < s_.size() && s_[i_] == '}') {
                    ++i_;
                    return v;
                }
                bad("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = JVal::Arr;
            ++i_;
            ws();
            if (i_ < s_.size() && s_[i_] == ']') {
                ++i_;
                return v;
            }
            for (;;) {
                v.arr.push_back(value(depth + 1));
                ws();
                if (i_ < s_.size() && s_[i_] == ',') {
                    ++i_;
                    continue;
                }
                if (i_ < s_.size() && s_[i_] == ']') {
                    ++i_;
                    return v;
                }
                bad("expected ',' or ']'");
            }
        }
        if (c == '"') {
            v.kind = JVal::Str;
            v.str = string();
            return v;
        }
        if (lit("true")) {
            v.kind = JVal::Bool;
            v.b = true;
            return v;
        }
        if (lit("false")) {
            v.kind = JVal::Bool;
            return v;
        }
        if (lit("null")) return v;
        // Python's json module also reads NaN and +-Infinity
        if (lit("NaN")) {
            v.kind = JVal::Num;
            v.num = NAN;
            return v;
        }
        if (lit("Infinity")) {
            v.kind = JVal::Num;
            v.num = INFINITY;
            return v;
        }
        if (lit("-Infinity")) {
            v.kind = JVal::Num;
            v.num = -INFINITY;
            return v;
        }
        return number();
    }

    JVal number() {
        const size_t b = i_;
        if (i_ < s_.size() && s_[i_] == '-') ++i_;
        auto digits = [&]() {
            size_t d = i_;
            while (i_ < s_.size() && s_[i_] >= '0' && s_[i_] <= '9') ++i_;
            return i_ > d;
        };
        if (!digits()) bad("bad value");
        if (i_ < s_.size() && s_[i_] == '.') {
            ++i_;
            if (!digits()) bad("bad number");
        }
        if (i_ < s_.size() && (s_[i_] == 'e' || s_[i_] == 'E')) {
            ++i_;
            if (i_ < s_.size() && (s_[i_] == '+' || s_[i_] == '-')) ++i_;
            if (!digits()) bad("bad number");
        }
        JVal v;
        v.kind = JVal::Num;
        const std::string tok = s_.substr(b, i_ - b);
        v.num = std::strtod(tok.c_str(), nullptr);  // correctly rounded, as Python's float()
        return v;
    }

    static void utf8(std::string& out, unsigned cp) {
        if (cp < 0x80) {
            out += (char)cp;
        } else if (cp < 0x800) {
            out += (char)(0xC0 | (cp >> 6));
            out += (char)(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            out += (char)(0xE0 | (cp >> 12));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
        } else {
            out += (char)(0xF0 | (cp >> 18));
            out += (char)(0x80 | ((cp >> 12) & 0x3F));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
        }
    }

    unsigned hex4() {
        if (i_ + 4 > s_.size()) bad("bad \\u escape");
        unsigned v = 0;
        for (int k = 0; k < 4; ++k) {
            const char h = s_[i_++];
            v <<= 4;
            if (h >= '0' && h <= '9')
                v |= (unsigned)(h - '0');
            else if (h >= 'a' && h <= 'f')
                v |= (unsigned)(h - 'a' + 10);
            else if (h >= 'A' && h <= 'F')
                v |= (unsigned)(h - 'A' + 10);
            else
                bad("bad \\u escape");
        }
        return v;
    }

    std::string string() {
        ++i_;  // opening quote
        std::string out;
        for (;;) {
            if (i_ >= s_.size()) bad("unterminated string");
            const char c = s_[i_++];
            if (c == '"') return out;
            if (c != '\\') {
                out += c;
                continue;
            }
            if (i_ >= s_.size()) bad("unterminated string");
            const char e = s_[i_++];
            switch (e) {
                case '"': out += '"'; break;
                case '\\': out += '\\'; break;
                case '/': out += '/'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'n': out += '\n'; break;
                case 'r': out += '\r'; break;
                case 't': out += '\t'; break;
                case 'u': {
                    unsigned cp = hex4();
                    if (cp >= 0xD800 && cp < 0xDC00 && s_.compare(i_, 2, "\\u") == 0) {
                        const size_t keep = i_;
                        i_ += 2;
                        const unsigned lo = hex4();
                        if (lo >= 0xDC00 && lo < 0xE000)
                            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                        else
                            i_ = keep;
                    }
                    utf8(out, cp);
                    break;
                }
                default: bad("bad escape");
            }
        }
    }
};

}  // namespace

namespace {

// ------------------------------------------------------------------------------------------
// SceneLoader (sceneloader.cpp:11-131, 346-443), with Python's conversions where the reference
// file gives a value: float(x) for numbers, int(x) for the grid size (truncation)
// ------------------------------------------------------------------------------------------
double num(const JVal& v, const char* what) {
    if (v.kind == JVal::Num) return v.num;
    if (v.kind == JVal::Bool) return v.b ? 1.0 : 0.0;
    if (v.kind == JVal::Str) {
        const char* b = v.str.c_str();
        char* e = nullptr;
        errno = 0;
        const double x = std::strtod(b, &e);
        while (e && (*e == ' ' || *e == '\t' || *e == '\n' || *e == '\r')) ++e;
        if (e != b && e && *e == '\0') return x;
    }
    fail(std::string(what) + " is not a number");
}

long long integer(const JVal& v, const char* what) {
    if (v.kind == JVal::Num) {
        if (!(std::fabs(v.num) < 9.0e18)) fail(std::string(what) + " is out of range");
        return (long long)std::trunc(v.num);
    }
    if (v.kind == JVal::Bool) return v.b ? 1 : 0;
    if (v.kind == JVal::Str) {
        const char* b = v.str.c_str();
        char* e = nullptr;
        const long long x = std::strtoll(b, &e, 10);
        if (e != b && *e == '\0') return x;
    }
    fail(std::string(what) + " is not an integer");
}

// A dictionary key as Python would hash the id (strings and numbers; True and 1 coincide).
std::string id_key(const JVal& v) {
    char buf[64];
    switch (v.kind) {
        case JVal::Str: return "s:" + v.str;
        case JVal::Num: std::snprintf(buf, sizeof buf, "n:%.17g", v.num); return buf;
        case JVal::Bool: return v.b ? "n:1" : "n:0";
        case JVal::Null: return "null";
        default: fail("an id must be a string or a number");
    }
}

const std::vector<JVal>& list(const JVal& root, const char* key) {
    static const std::vector<JVal> empty;
    const JVal* v = root.get(key);
    if (!v) return empty;
    if (v->kind != JVal::Arr) fail(std::string("'") + key + "' is not a list");
    return v->arr;
}

const JVal& object(const JVal& v, const char* what) {
    if (v.kind != JVal::Obj) fail(std::string(what) + " is not an object");
    return v;
}

struct Vec3 {
    double v[3];
};

Vec3 vec(const JVal& obj, const char* key, double dx, double dy, double dz) {
    const JVal* p = obj.get(key);
    if (!p) return Vec3{{dx, dy, dz}};
    const JVal& o = object(*p, key);
    Vec3 r{{0.0, 0.0, 0.0}};
    const char* names[3] = {"x", "y", "z"};
    for (int a = 0; a < 3; ++a) {
        const JVal* c = o.get(names[a]);
        r.v[a] = c ? num(*c, key) : 0.0;
    }
    return r;
}

struct MeshDef {
    enum Kind { Obj, Box, Sphere } kind = Box;
    std::vector<float> verts;  // OBJ
    std::vector<int32_t> tris;
    Vec3 p0{}, p1{};  // box corners
    Vec3 center{};
    double radius = 0.0;
};

struct Transform {
    Vec3 t, r, s;
};

struct Geom {
    const MeshDef* mesh;
    const Transform* tr;
    long long offset;
};

// OBJ records: "v x y z" and "f a b c ..." (1-based or negative indices, "a/b/c" forms); a
// polygon becomes a fan, so a quad v0 v1 v2 v3 gives the two triangles the reference tests
// (Obj::QuadTest, obj.cpp:344-352).
void read_obj(const std::string& path, std::vector<float>& verts, std::vector<int32_t>& tris) {
    std::ifstream f(path);
    if (!f) fail("cannot read OBJ file " + path);
    std::string line;
    std::vector<double> vx;
    while (std::getline(f, line)) {
        std::istringstream ls(line);
        std::vector<std::string> parts;
        for (std::string tok; ls >> tok;) parts.push_back(tok);
        if (parts.empty()) continue;
        if (parts[0] == "v" && parts.size() >= 4) {
            for (int a = 1; a <= 3; ++a) {
                JVal s;
                s.kind = JVal::Str;
                s.str = parts[a];
                vx.push_back(num(s, "an OBJ coordinate"));
            }
        } else if (parts[0] == "f" && parts.size() >= 4) {
            std::vector<long long> idx;
            const long long nv = (long long)(vx.size() / 3);
            for (size_t k = 1; k < parts.size(); ++k) {
                JVal s;
                s.kind = JVal::Str;
                s.str = parts[k].substr(0, parts[k].find('/'));
                const long long i = integer(s, "an OBJ face index");
                idx.push_back(i > 0 ? i - 1 : nv + i);
            }
            for (size_t j = 1; j + 1 < idx.size(); ++j) {
                tris.push_back((int32_t)idx[0]);
                tris.push_back((int32_t)idx[j]);
                tris.push_back((int32_t)idx[j + 1]);
            }
        }
    }
    if (vx.empty() || tris.empty()) fail("OBJ file " + path + " has no triangles");
    verts.assign(vx.begin(), vx.end());
}

// The eight corners (index x*4 + y*2 + z) and twelve triangles of an axis-aligned box.
void box_mesh(const Vec3& lo, const Vec3& hi, std::vector<float>& v, std::vector<int32_t>& t) {
    for (int x = 0; x < 2; ++x)
        for (int y = 0; y < 2; ++y)
            for (int z = 0; z < 2; ++z) {
                v.push_back((float)(x ? hi : lo).v[0]);
                v.push_back((float)(y ? hi : lo).v[1]);
                v.push_back((float)(z ? hi : lo).v[2]);
            }
    auto i = [](int x, int y, int z) { return x * 4 + y * 2 + z; };
    const int quads[6][4] = {{i(0, 0, 0), i(0, 1, 0), i(0, 1, 1), i(0, 0, 1)}, {i(1, 0, 0), i(1, 0, 1), i(1, 1, 1), i(1, 1, 0)},
                             {i(0, 0, 0), i(0, 0, 1), i(1, 0, 1), i(1, 0, 0)}, {i(0, 1, 0), i(1, 1, 0), i(1, 1, 1), i(0, 1, 1)},
                             {i(0, 0, 0), i(1, 0, 0), i(1, 1, 0), i(0, 1, 0)}, {i(0, 0, 1), i(0, 1, 1), i(1, 1, 1), i(1, 0, 1)}};
    for (const auto& q : quads) {
        const int tri[6] = {q[0], q[1], q[2], q[0], q[2], q[3]};
        t.insert(t.end(), tri, tri + 6);
    }
}

void copy_path(char* dst, const JVal* v, const char* what) {
    dst[0] = '\0';
    if (!v) return;
    if (v->kind != JVal::Str) fail(std::string(what) + " is not a string");
    if (v->str.size() >= 512) fail(std::string(what) + " is longer than 511 characters");
    std::memcpy(dst, v->str.c_str(), v->str.size() + 1);
}

struct Created {
    std::vector<int32_t> ids;
    ~Created() {
        for (int32_t id : ids) ariel_mesh_destroy(id);
    }
};

void load(const JVal& root, const std::string& base_dir, float jitter, uint64_t seed, AsimSceneDesc& d,
          AsimSceneInfo& info, Created& made) {
    object(root, "the scene");
    const std::vector<JVal>& settings_list = list(root, "settings");
    JVal empty_obj;
    empty_obj.kind = JVal::Obj;
    const JVal& settings = settings_list.empty() ? empty_obj : object(settings_list[0], "settings[0]");
    const double density = settings.has("density") ? num(*settings.get("density"), "density") : 0.5;
    const double step = settings.has("step_size") ? num(*settings.get("step_size"), "step_size") : 0.005;
    long long dims[3] = {32, 32, 32};
    if (const JVal* dim = settings.get("dim")) {
        object(*dim, "dim");
        const char* names[3] = {"x", "y", "z"};
        for (int a = 0; a < 3; ++a)
            if (const JVal* c = dim->get(names[a])) dims[a] = integer(*c, "dim");
    }
    if (!(dims[0] == dims[1] && dims[1] == dims[2]))
        fail("non-cubic grid: the step treats every axis as the largest one");
    if (dims[0] < 1 || dims[0] > (1 << 20)) fail("grid size out of range");
    const long long n = dims[0];

    std::map<std::string, Transform> transforms;
    for (const JVal& t : list(root, "transforms")) {
        object(t, "a transform");
        if (!t.has("id") || transforms.count(id_key(*t.get("id")))) continue;  // as the reference
        transforms[id_key(*t.get("id"))] =
            Transform{vec(t, "translation", 0, 0, 0), vec(t, "rotation", 0, 0, 0), vec(t, "scale", 1, 1, 1)};
    }
    std::map<std::string, MeshDef> meshes;
    for (const JVal& m : list(root, "meshfiles")) {
        object(m, "a mesh file");
        if (!m.has("id") || meshes.count(id_key(*m.get("id")))) continue;
        MeshDef md;
        if (const JVal* file = m.get("file")) {
            if (file->kind != JVal::Str) fail("a mesh file name is not a string");
            md.kind = MeshDef::Obj;
            const std::string p = (!file->str.empty() && file->str[0] == '/') ? file->str : base_dir + "/" + file->str;
            read_obj(p, md.verts, md.tris);
        } else {
            const JVal* gen = m.get("mesh_gen");
            const std::string g = gen && gen->kind == JVal::Str ? gen->str : std::string("(none)");
            if (g == "box") {
                md.kind = MeshDef::Box;
                md.p0 = vec(m, "point0", 0, 0, 0);
                md.p1 = vec(m, "point1", 0, 0, 0);
            } else if (g == "sphere") {
                md.kind = MeshDef::Sphere;
                md.center = vec(m, "center", 0, 0, 0);
                md.radius = m.has("radius") ? num(*m.get("radius"), "radius") : 0.0;
            } else {
                fail("mesh generator '" + g + "' is not supported");
            }
        }
        meshes[id_key(*m.get("id"))] = std::move(md);
    }
    if (const JVal* am = root.get("animatedmeshes"))
        if (am->truthy()) fail("animated meshes are not supported");
    std::map<std::string, Geom> geoms;
    for (const JVal& g : list(root, "geoms")) {
        object(g, "a geom");
        if (!g.has("id") || geoms.count(id_key(*g.get("id")))) continue;
        const JVal* type = g.get("type");
        if (!type || type->kind != JVal::Str || type->str != "mesh") fail("geom type is not 'mesh'");
        const std::vector<JVal>& frames = list(g, "geom_frames");
        const std::vector<JVal>& tframes = list(g, "transform_frames");
        if (frames.empty() || tframes.empty()) fail("a geom has no frame-0 mesh or transform");
        auto mi = meshes.find(id_key(frames[0]));
        auto ti = transforms.find(id_key(tframes[0]));
        if (mi == meshes.end()) fail("a geom names a mesh that is not defined");
        if (ti == transforms.end()) fail("a geom names a transform that is not defined");
        const long long off = g.has("frame_offset") ? integer(*g.get("frame_offset"), "frame_offset") : 0;
        geoms[id_key(*g.get("id"))] = Geom{&mi->second, &ti->second, off};
    }

    std::memset(&d, 0, sizeof d);
    std::memset(&info, 0, sizeof info);
    d.dim = (int32_t)n;
    d.density = (float)density;
    d.stepsize = (float)step;
    const std::vector<JVal>& forces = list(root, "globalforces");
    if (forces.size() > ARIEL_MAX_FORCES) fail("more global forces than the scene description holds");
    d.n_forces = (int32_t)forces.size();
    for (size_t i = 0; i < forces.size(); ++i) {
        const JVal& fo = object(forces[i], "a global force");
        const char* names[3] = {"x", "y", "z"};
        for (int a = 0; a < 3; ++a) d.forces[i][a] = fo.has(names[a]) ? (float)num(*fo.get(names[a]), "a force") : 0.0f;
    }
    int nl = 0, ns = 0;
    const double dn = (double)n;
    for (const JVal& node : list(root, "sim")) {
        object(node, "a sim node");
        const JVal* gid = node.get("geom");
        if (!gid) fail("a sim node names no geom");
        auto gi = geoms.find(id_key(*gid));
        if (gi == geoms.end()) fail("a sim node names a geom that is not defined");
        const Geom& geom = gi->second;
        if (geom.offset != 0) fail("geometry that appears after frame 0 is not supported");
        const Transform& tr = *geom.tr;
        for (int a = 0; a < 3; ++a)
            if (std::fabs(tr.r.v[a]) > 0.0) fail("rotated geometry is not supported (boxes and spheres stay axis-aligned)");
        for (int a = 0; a < 3; ++a)
            if (tr.s.v[a] <= 0.0) fail("non-positive scale");
        const bool uniform = tr.s.v[0] == tr.s.v[1] && tr.s.v[1] == tr.s.v[2];
        const MeshDef& mesh = *geom.mesh;
        Vec3 lo{}, hi{}, c{};
        double r = 0.0;
        if (mesh.kind == MeshDef::Obj) {
            if (!uniform) fail("non-uniformly scaled mesh");
        } else if (mesh.kind == MeshDef::Box) {
            for (int a = 0; a < 3; ++a) {
                const double p = mesh.p0.v[a], q = mesh.p1.v[a];
                lo.v[a] = tr.t.v[a] + tr.s.v[a] * (q < p ? q : p);
                hi.v[a] = tr.t.v[a] + tr.s.v[a] * (p < q ? q : p);
            }
        } else {
            if (!uniform) fail("non-uniformly scaled sphere");
            for (int a = 0; a < 3; ++a) c.v[a] = tr.t.v[a] + tr.s.v[a] * mesh.center.v[a];
            r = tr.s.v[0] * mesh.radius;
        }
        const JVal* type = node.get("type");
        const std::string kind = type && type->kind == JVal::Str ? type->str : std::string("(none)");
        if (kind == "liquid") {
            if (mesh.kind != MeshDef::Box) fail("only box liquids are supported");
            if (nl >= ARIEL_MAX_BOXES) fail("more liquids than the scene description holds");
            const Vec3 vel = vec(node, "velocity", 0, 0, 0);
            for (int a = 0; a < 3; ++a) {
                d.liquid[nl].lo[a] = (float)(lo.v[a] / dn);
                d.liquid[nl].hi[a] = (float)(hi.v[a] / dn);
                d.liquid[nl].vel[a] = (float)vel.v[a];
            }
            ++nl;
        } else if (kind == "solid") {
            if (mesh.kind == MeshDef::Sphere) {
                if (ns >= ARIEL_MAX_SPHERES) fail("more sphere solids than the scene description holds");
                for (int a = 0; a < 3; ++a) d.solid[ns].center[a] = (float)(c.v[a] / dn);
                d.solid[ns].radius = (float)(r / dn);
                ++ns;
            } else {
                // a box or OBJ solid: a static mesh in grid units, placed in the unit cube
                if (d.n_mesh >= ARIEL_MAX_MESHES) fail("more mesh solids than the scene description holds");
                std::vector<float> v;
                std::vector<int32_t> t;
                float translate[3] = {0.0f, 0.0f, 0.0f};
                float scale;
                if (mesh.kind == MeshDef::Box) {
                    box_mesh(lo, hi, v, t);
                    scale = (float)(1.0 / dn);
                } else {
                    v = mesh.verts;
                    t = mesh.tris;
                    for (int a = 0; a < 3; ++a) translate[a] = (float)(tr.t.v[a] / dn);
                    scale = (float)(tr.s.v[0] / dn);
                }
                int32_t id = 0;
                const ariel_status st = ariel_mesh_create(v.data(), (int32_t)(v.size() / 3), t.data(),
                                                          (int32_t)(t.size() / 3), translate, scale, &id);
                if (st != ARIEL_OK) fail("a solid mesh was refused (ariel_mesh_create status " + std::to_string(st) + ")");
                made.ids.push_back(id);
                d.mesh[d.n_mesh++] = id;
            }
        } else {
            fail("sim node type '" + kind + "' is not supported");
        }
    }
    d.n_liquid = nl;
    d.n_solid = ns;
    d.seed = seed;
    d.jitter = jitter;
    info.dim = (int32_t)n;
    info.density = density;
    info.step_size = step;
    copy_path(info.partio_output, settings.get("partio_output"), "partio_output");
    copy_path(info.vdb_output, settings.get("vdb_output"), "vdb_output");
    copy_path(info.mesh_output, settings.get("mesh_output"), "mesh_output");
}

ariel_status run(const std::string& text, const std::string& base_dir, float jitter, uint64_t seed,
                 AsimSceneDesc* desc, AsimSceneInfo* info, char* error, int32_t error_len) {
    if (error && error_len > 0) error[0] = '\0';
    if (!desc) return ARIEL_ERR_INVALID_ARG;
    Created made;
    AsimSceneDesc d;
    AsimSceneInfo in;
    try {
        const JVal root = Reader(text).document();
        load(root, base_dir, jitter, seed, d, in, made);
    } catch (const SceneFail& f) {
        if (error && error_len > 0) {
            std::strncpy(error, f.why.c_str(), (size_t)error_len - 1);
            error[error_len - 1] = '\0';
        }
        return ARIEL_ERR_INVALID_ARG;  // `made` destroys the meshes registered so far
    } catch (const std::bad_alloc&) {
        return ARIEL_ERR_OOM;
    }
    made.ids.clear();  // the caller owns them now
    *desc = d;
    if (info) *info = in;
    return ARIEL_OK;
}

}  // namespace

extern "C" {

ariel_status ariel_scene_parse(const char* json_text, const char* base_dir, float jitter, uint64_t seed,
                               AsimSceneDesc* desc, AsimSceneInfo* info, char* error, int32_t error_len) {
    if (!json_text) return ARIEL_ERR_INVALID_ARG;
    return run(json_text, base_dir && base_dir[0] ? base_dir : ".", jitter, seed, desc, info, error, error_len);
}

ariel_status ariel_scene_load(const char* path, float jitter, uint64_t seed, AsimSceneDesc* desc,
                              AsimSceneInfo* info, char* error, int32_t error_len) {
    if (!path) return ARIEL_ERR_INVALID_ARG;
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        if (error && error_len > 0) {
            std::snprintf(error, (size_t)error_len, "cannot read scene file %s", path);
        }
        return ARIEL_ERR_INVALID_ARG;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string p(path);
    const size_t slash = p.find_last_of('/');
    const std::string dir = slash == std::string::npos ? std::string(".") : (slash == 0 ? std::string("/") : p.substr(0, slash));
    return run(ss.str(), dir, jitter, seed, desc, info, error, error_len);
}

}  // extern "C"
