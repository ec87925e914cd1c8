// mrt_obj.cu - Wavefront OBJ / MTL scene ingestion with the reference loader's conventions
// (OBJLoader::process + OBJLoader::fillScene, app/Components/ObjectLoaders/OBJLoader.cpp:21-248).
//
// The reference parses with tinyobjloader (an empty submodule in the checkout, version unpinned) and
// then converts every triangle; this file does both steps itself, host-side:
//   parsing   v x y z [r g b] (vertex colour 1,1,1 when absent), vn, f with v | v/vt | v//vn | v/vt/vn
//             and negative (relative) indices, usemtl; faces of n > 3 vertices split as a fan
//             (v0, vk, vk+1); materials come from the MTL file the caller names (the reference hands
//             its own MTL stream to the parser and ignores mtllib): newmtl, Kd, Ks, Kt / Tf, d, Tr
//             (d = 1 - Tr), Ni, Ke; defaults 0 for colours, 1 for d and Ni.
//   conversion (OBJLoader.cpp:81-243): x negated on vertices and normals; given normals normalised
//             and used only when all three are non-zero, else the Triangle constructor's
//             normalize(cross(C - A, B - A)); material Kd, Ks / 2, Kt * (1 - d), Ni, Ke divided by
//             its largest component when that exceeds 1; a face whose material emits becomes an
//             AreaLight (not a triangle); other materials are de-duplicated with Material::operator==
//             (components within Epsilon, Material.cpp:21-29), first occurrence first; faces
//             without a material get -1 (shaded by their vertex colours).
// Numbers are parsed with strtod (correctly rounded) and rounded to float.
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

#include "../../include/mrt_cuda.h"
#include "mrt_device.cuh"

using mrt::V3;

struct MrtObjScene {
    std::vector<float> abc, normals, colors;
    std::vector<int32_t> material;
    std::vector<MrtMaterial> materials;
    std::vector<MrtLightDesc> lights;
};

namespace {

struct ObjMtl {
    float kd[3] = {0, 0, 0}, ks[3] = {0, 0, 0}, kt[3] = {0, 0, 0}, ke[3] = {0, 0, 0};
    float ior = 1.0f, dissolve = 1.0f;
};

struct FaceVertex {
    int64_t v = -1, n = -1;
};

bool parse_floats(std::istringstream &in, float *out, int max_n, int &got) {
    got = 0;
    std::string tok;
    while (got < max_n && (in >> tok)) {
        char *end = nullptr;
        errno = 0;
        const double d = std::strtod(tok.c_str(), &end);
        if (end == tok.c_str()) return false;
        out[got++] = (float)d;
    }
    return true;
}

// OBJ index (1-based, or negative relative to the elements read so far) -> 0-based, -1 if invalid
int64_t fix_index(long long i, size_t n) {
    if (i > 0) return (int64_t)i - 1;
    if (i < 0) return (int64_t)n + i;
    return -1;
}

bool parse_face_vertex(const std::string &tok, size_t nv, size_t nn, FaceVertex &fv) {
    const size_t s1 = tok.find('/');
    fv.v = fix_index(std::strtoll(tok.c_str(), nullptr, 10), nv);
    if (fv.v < 0 || (size_t)fv.v >= nv) return false;
    if (s1 != std::string::npos) {
        const size_t s2 = tok.find('/', s1 + 1);
        if (s2 != std::string::npos && s2 + 1 < tok.size()) {
            fv.n = fix_index(std::strtoll(tok.c_str() + s2 + 1, nullptr, 10), nn);
            if (fv.n >= (int64_t)nn) fv.n = -1;
        }
    }
    return true;
}

bool read_mtl(const char *path, std::vector<ObjMtl> &mats, std::map<std::string, int> &names, std::string &err) {
    std::ifstream f(path);
    if (!f) { err = std::string("cannot open MTL file ") + path; return false; }
    std::string line;
    ObjMtl *cur = nullptr;
    while (std::getline(f, line)) {
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        std::istringstream in(line);
        std::string key;
        if (!(in >> key)) continue;
        int got = 0;
        float v[3] = {0, 0, 0};
        if (key == "newmtl") {
            std::string name;
            in >> name;
            names[name] = (int)mats.size();
            mats.emplace_back();
            cur = &mats.back();
        } else if (!cur) {
            continue;
        } else if (key == "Kd" || key == "Ks" || key == "Kt" || key == "Tf" || key == "Ke") {
            if (!parse_floats(in, v, 3, got) || got == 0) continue;
            if (got < 3) v[1] = v[2] = v[0];
            float *dst = key == "Kd" ? cur->kd : key == "Ks" ? cur->ks : key == "Ke" ? cur->ke : cur->kt;
            for (int k = 0; k < 3; ++k) dst[k] = v[k];
        } else if (key == "d") {
            if (parse_floats(in, v, 1, got) && got == 1) cur->dissolve = v[0];
        } else if (key == "Tr") {
            if (parse_floats(in, v, 1, got) && got == 1) cur->dissolve = 1.0f - v[0];
        } else if (key == "Ni") {
            if (parse_floats(in, v, 1, got) && got == 1) cur->ior = v[0];
        }
    }
    return true;
}

// Material::operator== (Material.cpp:21-29)
bool same_material(const MrtMaterial &a, const MrtMaterial &b) {
    auto close3 = [](const float *x, const float *y) {
        for (int k = 0; k < 3; ++k)
            if (!(std::fabs(x[k] - y[k]) <= mrt::kEpsilon)) return false;
        return true;
    };
    return close3(a.le, b.le) && close3(a.kd, b.kd) && close3(a.ks, b.ks) && close3(a.kt, b.kt) &&
           std::fabs(a.ior - b.ior) < mrt::kEpsilon;
}

void put3(std::vector<float> &dst, V3 v) {
    dst.push_back(v.x);
    dst.push_back(v.y);
    dst.push_back(v.z);
}

}  // namespace

extern "C" {

int mrt_obj_load(const char *obj_path, const char *mtl_path, MrtObjScene **out, MrtSceneDesc *desc, char *error,
                 size_t error_len) {
    auto fail = [&](int st, const std::string &msg) {
        if (error && error_len) std::snprintf(error, error_len, "%s", msg.c_str());
        return st;
    };
    if (!obj_path || !out || !desc) return fail(MRT_ERR_ARG, "mrt_obj_load: null argument");
    *out = nullptr;
    std::vector<ObjMtl> mtls;
    std::map<std::string, int> mtl_names;
    std::string err;
    if (mtl_path && *mtl_path && !read_mtl(mtl_path, mtls, mtl_names, err)) return fail(MRT_ERR_ARG, err);
    std::ifstream f(obj_path);
    if (!f) return fail(MRT_ERR_ARG, std::string("cannot open OBJ file ") + obj_path);

    std::vector<float> pos, col, nrm;
    struct Tri {
        FaceVertex a, b, c;
        int material;
    };
    std::vector<Tri> tris;
    int current_mtl = -1;
    std::string line;
    size_t line_no = 0;
    while (std::getline(f, line)) {
        ++line_no;
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        std::istringstream in(line);
        std::string key;
        if (!(in >> key)) continue;
        if (key == "v") {
            float v[7];
            int got = 0;
            if (!parse_floats(in, v, 7, got) || got < 3) return fail(MRT_ERR_ARG, "bad vertex on line " + std::to_string(line_no));
            pos.insert(pos.end(), v, v + 3);
            if (got >= 6) col.insert(col.end(), v + 3, v + 6);
            else col.insert(col.end(), {1.0f, 1.0f, 1.0f});
        } else if (key == "vn") {
            float v[3];
            int got = 0;
            if (!parse_floats(in, v, 3, got) || got < 3) return fail(MRT_ERR_ARG, "bad normal on line " + std::to_string(line_no));
            nrm.insert(nrm.end(), v, v + 3);
        } else if (key == "usemtl") {
            std::string name;
            in >> name;
            const auto it = mtl_names.find(name);
            current_mtl = it == mtl_names.end() ? -1 : it->second;
        } else if (key == "f") {
            std::vector<FaceVertex> face;
            std::string tok;
            while (in >> tok) {
                FaceVertex fv;
                if (!parse_face_vertex(tok, pos.size() / 3, nrm.size() / 3, fv))
                    return fail(MRT_ERR_ARG, "bad face index on line " + std::to_string(line_no));
                face.push_back(fv);
            }
            for (size_t k = 1; k + 1 < face.size(); ++k) tris.push_back(Tri{face[0], face[k], face[k + 1], current_mtl});
        }
    }

    MrtObjScene *s = new MrtObjScene();
    const bool have_normals = !nrm.empty();
    for (const Tri &t : tris) {
        const FaceVertex fvs[3] = {t.a, t.b, t.c};
        V3 p[3], n[3], c[3];
        for (int k = 0; k < 3; ++k) {
            const float *q = &pos[3 * (size_t)fvs[k].v];
            p[k] = V3{-q[0], q[1], q[2]};
            const float *cc = &col[3 * (size_t)fvs[k].v];
            c[k] = V3{cc[0], cc[1], cc[2]};
            n[k] = V3{0.0f, 0.0f, 0.0f};
            if (have_normals && fvs[k].n >= 0) {
                const float *m = &nrm[3 * (size_t)fvs[k].n];
                n[k] = mrt::normalize(V3{-m[0], m[1], m[2]});
            }
        }
        const bool has_normal = mrt::length(n[0]) > 0 && mrt::length(n[1]) > 0 && mrt::length(n[2]) > 0;
        int32_t mat_index = -1;
        if (t.material >= 0) {
            const ObjMtl &m = mtls[(size_t)t.material];
            MrtMaterial mm{};
            for (int k = 0; k < 3; ++k) {
                mm.kd[k] = m.kd[k];
                mm.ks[k] = m.ks[k] / 2.0f;
                mm.kt[k] = m.kt[k] * (1.0f - m.dissolve);
            }
            float e1 = m.ke[0], e2 = m.ke[1], e3 = m.ke[2];
            const float mx12 = (e1 < e2) ? e2 : e1;     // std::max
            const float mx = (mx12 < e3) ? e3 : mx12;
            if (mx > 1.0f) {
                e1 /= mx;
                e2 /= mx;
                e3 /= mx;
            }
            mm.le[0] = e1; mm.le[1] = e2; mm.le[2] = e3;
            mm.ior = m.ior;
            if (e1 > 0.0f || e2 > 0.0f || e3 > 0.0f) {   // an emitting face is an AreaLight
                MrtLightDesc l{};
                l.kind = MRT_LIGHT_AREA;
                l.p0[0] = p[0].x; l.p0[1] = p[0].y; l.p0[2] = p[0].z;
                l.p1[0] = p[1].x; l.p1[1] = p[1].y; l.p1[2] = p[1].z;
                l.p2[0] = p[2].x; l.p2[1] = p[2].y; l.p2[2] = p[2].z;
                l.radiance = mm;
                s->lights.push_back(l);
                continue;
            }
            size_t found = s->materials.size();
            for (size_t k = 0; k < s->materials.size(); ++k)
                if (same_material(s->materials[k], mm)) { found = k; break; }
            if (found == s->materials.size()) s->materials.push_back(mm);
            mat_index = (int32_t)found;
        }
        for (int k = 0; k < 3; ++k) put3(s->abc, p[k]);
        if (!has_normal) {   // Triangle.cpp:10-17 / 40-54
            const V3 ac = p[2] - p[0], ab = p[1] - p[0];
            const V3 g = mrt::normalize(mrt::cross(ac, ab));
            n[0] = n[1] = n[2] = g;
        }
        for (int k = 0; k < 3; ++k) put3(s->normals, n[k]);
        for (int k = 0; k < 3; ++k) put3(s->colors, c[k]);
        s->material.push_back(mat_index);
    }
    std::memset(desc, 0, sizeof(*desc));
    desc->n_triangles = (uint32_t)s->material.size();
    desc->tri_abc = s->abc.empty() ? nullptr : s->abc.data();
    desc->tri_normals = s->normals.empty() ? nullptr : s->normals.data();
    desc->tri_colors = s->colors.empty() ? nullptr : s->colors.data();
    desc->tri_material = s->material.empty() ? nullptr : s->material.data();
    desc->n_materials = (uint32_t)s->materials.size();
    desc->materials = s->materials.empty() ? nullptr : s->materials.data();
    desc->n_lights = (uint32_t)s->lights.size();
    desc->lights = s->lights.empty() ? nullptr : s->lights.data();
    *out = s;
    if (error && error_len) error[0] = '\0';
    return MRT_OK;
}

void mrt_obj_free(MrtObjScene *scene) { delete scene; }

}  // extern "C"
