// urdf.cu - robot description input at run time (host code).
//
// The reference turns a URDF into a generated header of joint masks offline
// (scripts/URDFParser/urdfParserUtils.py:527-605, output RTCD/Robot/models/
// panda.h) and loads link meshes with tinyobjloader (RTCD/Meshes/mesh.h:311-
// 360).  Here both run inside the library, so a new serial-chain robot loads
// at run time: rtcd_urdf_chain_parse reads the URDF text and returns the
// masks of the local transform L_i(q) = cos q C_i + sin q S_i + O_i per
// revolute joint (fixed joints folded into the next joint's origin), the
// limits and each link's visual mesh file; rtcd_obj_load reads an OBJ file
// the way the reference's loader does (a vertex is identified by its exact
// float position, first occurrence wins; polygons fan-triangulated).
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/rtcd.h"
#include "engine.h"

namespace {

using rtcd::fail;

// ---------------------------------------------------------------- a small XML reader
struct Node {
    std::string tag;
    std::map<std::string, std::string> attr;
    std::vector<Node> kids;
    const Node* child(const char* t) const {
        for (const Node& k : kids)
            if (k.tag == t) return &k;
        return nullptr;
    }
    std::string get(const char* a, const char* dflt = "") const {
        auto it = attr.find(a);
        return it == attr.end() ? std::string(dflt) : it->second;
    }
};

struct XmlReader {
    const char* p;
    const char* end;
    void skip_ws() {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
    }
    bool starts(const char* s) const {
        size_t n = std::strlen(s);
        return (size_t) (end - p) >= n && std::memcmp(p, s, n) == 0;
    }
    void skip_until(const char* s) {
        size_t n = std::strlen(s);
        while (p < end && !starts(s)) ++p;
        if (p >= end) fail(RTCD_ERR_INVALID_ARGUMENT, std::string("URDF: unterminated markup, expected ") + s);
        p += n;
    }
    // skips text, comments, declarations; leaves p at '<' of an element or closing tag (or end)
    void skip_misc() {
        while (p < end) {
            while (p < end && *p != '<') ++p;
            if (starts("<!--")) {
                skip_until("-->");
            } else if (starts("<?")) {
                skip_until("?>");
            } else if (starts("<!")) {
                skip_until(">");
            } else {
                return;
            }
        }
    }
    std::string name() {
        const char* s = p;
        while (p < end && (std::isalnum((unsigned char) *p) || *p == '_' || *p == '-' || *p == ':' || *p == '.')) ++p;
        if (p == s) fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: malformed tag or attribute name");
        return std::string(s, p);
    }
    Node element() {
        if (p >= end || *p != '<') fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: expected an element");
        ++p;
        Node n;
        n.tag = name();
        while (true) {
            skip_ws();
            if (p >= end) fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: unterminated tag <" + n.tag + ">");
            if (starts("/>")) {
                p += 2;
                return n;
            }
            if (*p == '>') {
                ++p;
                break;
            }
            std::string a = name();
            skip_ws();
            if (p >= end || *p != '=') fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: attribute without a value");
            ++p;
            skip_ws();
            if (p >= end || (*p != '"' && *p != '\'')) fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: unquoted attribute");
            const char q = *p++;
            const char* s = p;
            while (p < end && *p != q) ++p;
            if (p >= end) fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: unterminated attribute value");
            n.attr[a] = std::string(s, p);
            ++p;
        }
        while (true) {
            skip_misc();
            if (p >= end) fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: element <" + n.tag + "> not closed");
            if (starts("</")) {
                p += 2;
                std::string t = name();
                if (t != n.tag) fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: </" + t + "> closes <" + n.tag + ">");
                skip_ws();
                if (p >= end || *p != '>') fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: malformed closing tag");
                ++p;
                return n;
            }
            n.kids.push_back(element());
        }
    }
};

std::vector<double> numbers(const std::string& s, size_t n, const char* what) {
    std::vector<double> v;
    const char* c = s.c_str();
    char* e = nullptr;
    while (true) {
        while (*c == ' ' || *c == '\t' || *c == '\n' || *c == '\r') ++c;
        if (!*c) break;
        double x = std::strtod(c, &e);
        if (e == c) fail(RTCD_ERR_INVALID_ARGUMENT, std::string("URDF: bad number in ") + what);
        v.push_back(x);
        c = e;
    }
    if (v.size() != n) fail(RTCD_ERR_INVALID_ARGUMENT, std::string("URDF: wrong number count in ") + what);
    return v;
}

// 4x4 rigid transforms (row-major 3x4 used)
struct Tf {
    double m[3][4];
};
Tf identity() {
    Tf t{};
    for (int i = 0; i < 3; ++i) t.m[i][i] = 1.0;
    return t;
}
Tf mul(const Tf& a, const Tf& b) {
    Tf r{};
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 4; ++j) {
            double s = j == 3 ? a.m[i][3] : 0.0;
            for (int k = 0; k < 3; ++k) s += a.m[i][k] * b.m[k][j];
            r.m[i][j] = s;
        }
    }
    return r;
}
// URDF origin: rotation R = Rz(yaw) Ry(pitch) Rx(roll) (fixed axes x, y, z), then xyz
Tf origin_of(const Node* j) {
    Tf t = identity();
    const Node* o = j->child("origin");
    if (!o) return t;
    std::vector<double> rpy = numbers(o->get("rpy", "0 0 0"), 3, "origin rpy");
    std::vector<double> xyz = numbers(o->get("xyz", "0 0 0"), 3, "origin xyz");
    const double cr = std::cos(rpy[0]), sr = std::sin(rpy[0]), cp = std::cos(rpy[1]), sp = std::sin(rpy[1]),
                 cy = std::cos(rpy[2]), sy = std::sin(rpy[2]);
    const double R[3][3] = {{cy * cp, cy * sp * sr - sy * cr, cy * sp * cr + sy * sr},
                            {sy * cp, sy * sp * sr + cy * cr, sy * sp * cr - cy * sr},
                            {-sp, cp * sr, cp * cr}};
    for (int i = 0; i < 3; ++i) {
        for (int k = 0; k < 3; ++k) t.m[i][k] = R[i][k];
        t.m[i][3] = xyz[i];
    }
    return t;
}

// values within 1e-5 of 0 or +-1 are set to them (the reference's rounding,
// which makes axis-aligned origins exact)
float snap(double v) {
    if (std::fabs(v) < 1e-5) return 0.0f;
    if (std::fabs(v - 1.0) < 1e-5) return 1.0f;
    if (std::fabs(v + 1.0) < 1e-5) return -1.0f;
    return (float) v;
}

void copy_name(char* dst, size_t cap, const std::string& s, const char* what) {
    if (s.size() >= cap) fail(RTCD_ERR_CAPACITY, std::string("URDF: ") + what + " longer than the field");
    std::memcpy(dst, s.c_str(), s.size() + 1);
}

template <class F>
rtcd_status guarded_host(F&& f) {
    try {
        f();
        rtcd::set_last_error("");
        return RTCD_OK;
    } catch (const rtcd::Error& e) {
        rtcd::set_last_error(e.msg);
        return (rtcd_status) e.status;
    } catch (const std::exception& e) {
        rtcd::set_last_error(e.what());
        return RTCD_ERR_INTERNAL;
    }
}

}  // namespace

extern "C" {

rtcd_status rtcd_urdf_chain_parse(const char* urdf, size_t len, rtcd_urdf_chain* out) {
    return guarded_host([&] {
        if (!urdf || !out) fail(RTCD_ERR_INVALID_ARGUMENT, "NULL argument");
        std::memset(out, 0, sizeof(*out));
        XmlReader rd{urdf, urdf + len};
        rd.skip_misc();
        Node robot = rd.element();
        if (robot.tag != "robot") fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: the root element is not <robot>");
        std::map<std::string, const Node*> links;
        std::map<std::string, std::vector<const Node*>> joints_from;  // parent link -> joints
        std::map<std::string, int> is_child;
        for (const Node& k : robot.kids) {
            if (k.tag == "link") {
                links[k.get("name")] = &k;
            } else if (k.tag == "joint") {
                const Node* pa = k.child("parent");
                const Node* ch = k.child("child");
                if (!pa || !ch) fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: joint without parent or child");
                joints_from[pa->get("link")].push_back(&k);
                is_child[ch->get("link")] = 1;
            }
        }
        std::string root;
        for (auto& kv : links)
            if (!is_child.count(kv.first)) {
                if (!root.empty()) fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: more than one root link");
                root = kv.first;
            }
        if (root.empty()) fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: no root link");
        auto add_link = [&](const std::string& name) {
            if (out->n_links >= RTCD_URDF_MAX_LINKS) fail(RTCD_ERR_CAPACITY, "URDF: more links than supported");
            const Node* l = links.count(name) ? links[name] : nullptr;
            copy_name(out->link_name[out->n_links], RTCD_URDF_NAME, name, "link name");
            const Node* v = l ? l->child("visual") : nullptr;
            const Node* g = v ? v->child("geometry") : nullptr;
            const Node* m = g ? g->child("mesh") : nullptr;
            copy_name(out->link_mesh[out->n_links], 2 * RTCD_URDF_NAME, m ? m->get("filename") : "", "mesh file name");
            ++out->n_links;
        };
        add_link(root);
        for (int k = 0; k < 12; ++k) out->base_tf[k] = (k % 5 == 0) ? 1.0f : 0.0f;
        Tf acc = identity();  // fixed joints since the last moving joint
        std::string cur = root;
        int guard = 0;
        while (joints_from.count(cur)) {
            if (++guard > 1024) fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: the joint graph has a cycle");
            const std::vector<const Node*>& js = joints_from[cur];
            if (js.size() != 1) fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: link " + cur + " branches (only serial chains)");
            const Node* j = js[0];
            const std::string type = j->get("type");
            const std::string child = j->child("child")->get("link");
            const Tf o = mul(acc, origin_of(j));
            if (type == "fixed") {
                acc = o;
                cur = child;
                continue;
            }
            if (type != "revolute" && type != "continuous")
                fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: joint type " + type + " is not supported");
            const uint32_t i = out->dof;
            if (i >= RTCD_URDF_MAX_LINKS - 1) fail(RTCD_ERR_CAPACITY, "URDF: more joints than supported");
            // axis u, K = [u]x: R(q) = I + sin q K + (1 - cos q) K^2, so
            // L(q) = origin * R(q) = cos q (-R0 K^2) + sin q (R0 K) + [R0 (I + K^2) | t]
            std::vector<double> u = numbers(j->child("axis") ? j->child("axis")->get("xyz", "1 0 0") : "1 0 0", 3,
                                            "axis");
            const double nu = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
            if (!(nu > 0)) fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: zero joint axis");
            for (double& x : u) x /= nu;
            const double K[3][3] = {{0, -u[2], u[1]}, {u[2], 0, -u[0]}, {-u[1], u[0], 0}};
            double K2[3][3];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    double s = 0;
                    for (int c = 0; c < 3; ++c) s += K[a][c] * K[c][b];
                    K2[a][b] = s;
                }
            for (int a = 0; a < 3; ++a) {
                for (int b = 0; b < 3; ++b) {
                    double c_ = 0, s_ = 0, o_ = 0;
                    for (int c = 0; c < 3; ++c) {
                        c_ += o.m[a][c] * -K2[c][b];
                        s_ += o.m[a][c] * K[c][b];
                        o_ += o.m[a][c] * ((c == b ? 1.0 : 0.0) + K2[c][b]);
                    }
                    out->cos_mask[12 * i + 4 * a + b] = snap(c_);
                    out->sin_mask[12 * i + 4 * a + b] = snap(s_);
                    out->one_mask[12 * i + 4 * a + b] = snap(o_);
                }
                out->cos_mask[12 * i + 4 * a + 3] = 0.0f;
                out->sin_mask[12 * i + 4 * a + 3] = 0.0f;
                out->one_mask[12 * i + 4 * a + 3] = snap(o.m[a][3]);
            }
            const Node* lim = j->child("limit");
            if (type == "revolute") {
                if (!lim) fail(RTCD_ERR_INVALID_ARGUMENT, "URDF: revolute joint without limits");
                out->lower[i] = (float) numbers(lim->get("lower", "0"), 1, "limit lower")[0];
                out->upper[i] = (float) numbers(lim->get("upper", "0"), 1, "limit upper")[0];
            } else {
                out->lower[i] = (float) -M_PI;
                out->upper[i] = (float) M_PI;
            }
            ++out->dof;
            acc = identity();
            cur = child;
            add_link(child);
        }
    });
}

rtcd_status rtcd_obj_load(const char* path, float* verts_out, uint32_t max_verts, uint32_t* n_verts,
                          uint32_t* tris_out, uint32_t max_tris, uint32_t* n_tris) {
    return guarded_host([&] {
        if (!path || !n_verts || !n_tris) fail(RTCD_ERR_INVALID_ARGUMENT, "NULL argument");
        FILE* fh = std::fopen(path, "r");
        if (!fh) fail(RTCD_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
        std::vector<float> raw;
        std::vector<uint32_t> faces;
        char line[4096];
        bool long_line = false;
        while (std::fgets(line, sizeof(line), fh)) {
            if (!std::strchr(line, '\n') && !std::feof(fh)) long_line = true;
            if (line[0] == 'v' && (line[1] == ' ' || line[1] == '\t')) {
                float x, y, z;
                if (std::sscanf(line + 2, "%f %f %f", &x, &y, &z) != 3) {
                    std::fclose(fh);
                    fail(RTCD_ERR_INVALID_ARGUMENT, "OBJ: bad vertex line");
                }
                raw.push_back(x); raw.push_back(y); raw.push_back(z);
            } else if (line[0] == 'f' && (line[1] == ' ' || line[1] == '\t')) {
                std::vector<long> idx;
                char* c = line + 2;
                while (*c) {
                    while (*c == ' ' || *c == '\t') ++c;
                    if (!*c || *c == '\n' || *c == '\r') break;
                    char* e = nullptr;
                    long v = std::strtol(c, &e, 10);
                    if (e == c) break;
                    idx.push_back(v);
                    c = e;
                    while (*c && *c != ' ' && *c != '\t' && *c != '\n') ++c;  // skip /vt/vn
                }
                const long nv = (long) (raw.size() / 3);
                for (long& v : idx) {
                    v = v > 0 ? v - 1 : nv + v;
                    if (v < 0 || v >= nv) {
                        std::fclose(fh);
                        fail(RTCD_ERR_INVALID_ARGUMENT, "OBJ: face index out of range");
                    }
                }
                for (size_t k = 1; k + 1 < idx.size(); ++k) {  // fan
                    faces.push_back((uint32_t) idx[0]);
                    faces.push_back((uint32_t) idx[k]);
                    faces.push_back((uint32_t) idx[k + 1]);
                }
            }
        }
        std::fclose(fh);
        if (long_line) fail(RTCD_ERR_CAPACITY, "OBJ: a line is longer than 4095 characters");
        // exact-position dedupe, first occurrence wins, in face order
        std::map<std::tuple<float, float, float>, uint32_t> known;
        std::vector<float> verts;
        std::vector<uint32_t> tris;
        tris.reserve(faces.size());
        for (uint32_t f : faces) {
            auto key = std::make_tuple(raw[3ull * f], raw[3ull * f + 1], raw[3ull * f + 2]);
            auto it = known.find(key);
            uint32_t id;
            if (it == known.end()) {
                id = (uint32_t) (verts.size() / 3);
                known.emplace(key, id);
                verts.push_back(raw[3ull * f]); verts.push_back(raw[3ull * f + 1]); verts.push_back(raw[3ull * f + 2]);
            } else {
                id = it->second;
            }
            tris.push_back(id);
        }
        *n_verts = (uint32_t) (verts.size() / 3);
        *n_tris = (uint32_t) (tris.size() / 3);
        if (verts_out) {
            if (*n_verts > max_verts) fail(RTCD_ERR_CAPACITY, "OBJ: more vertices than verts_out holds");
            std::memcpy(verts_out, verts.data(), verts.size() * sizeof(float));
        }
        if (tris_out) {
            if (*n_tris > max_tris) fail(RTCD_ERR_CAPACITY, "OBJ: more triangles than tris_out holds");
            std::memcpy(tris_out, tris.data(), tris.size() * sizeof(uint32_t));
        }
    });
}

}  // extern "C"
