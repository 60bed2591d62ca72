// Wavefront OBJ/MTL ingest into the triangle soup + shading records, the way the
// reference's PathTracingApp::extractScene fills them (PathTracingApp.cpp:31-124):
//   * one CUDA::Triangle per face triangle, in file order, vertices in world space
//     (here: position * scale + translate), info_idx = running triangle index;
//   * per vertex: uv (if given), colour (per-vertex "v x y z r g b" colours if
//     given, else the material's diffuse colour), normal (if given — as the
//     reference, not transformed — else the triangle's geometric normal
//     normalize(cross(v1 - v0, v2 - v0)) of the world-space triangle);
//   * material emission (Ke) and shininess (Ns) into the record; texture maps are
//     not supported by this library's shader (indices stay CPT_INVALID_INDEX).
// The reference imports through assimp (a Windows binary here); this parser follows
// the OBJ format itself: polygons are fanned (v0, vk, vk+1), negative indices count
// back from the last vertex, trailing comments are ignored, lines may be of any
// length, and an `mtllib` line may name several files. A face index (position, uv or
// normal) of 0 or outside the elements read so far makes the call fail with
// CPT_ERR_INVALID_ARGUMENT, as a missing file does.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <limits.h>
#include <string.h>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#include "cpt.h"
#include "cpt_internal.h"

namespace {

struct Mtl {
    float kd[3] = {-1.f, -1.f, -1.f};  // unset
    float ke[3] = {0.f, 0.f, 0.f};
    float ns = 0.f;
};

struct FaceVert {
    int v = 0, t = -1, n = -1;        // 0-based after resolve(); t, n = -1: not given
    bool has_t = false, has_n = false;
};

std::string dir_of(const std::string& p)
{
    const size_t k = p.find_last_of('/');
    return k == std::string::npos ? std::string() : p.substr(0, k + 1);
}

// Next line of f without its terminator; false at the end of the file.
bool read_line(FILE* f, std::string& line)
{
    line.clear();
    char buf[4096];
    while (fgets(buf, sizeof(buf), f)) {
        line += buf;
        if (!line.empty() && line.back() == '\n') return true;
    }
    return !line.empty();
}

std::string strip_comment(const std::string& s)
{
    const size_t k = s.find('#');
    return k == std::string::npos ? s : s.substr(0, k);
}

void load_mtl(const std::string& path, std::map<std::string, Mtl>& out)
{
    FILE* f = fopen(path.c_str(), "r");
    if (!f) return;
    std::string line, cur;
    while (read_line(f, line)) {
        std::istringstream ss(strip_comment(line));
        std::string tag;
        if (!(ss >> tag)) continue;
        if (tag == "newmtl") { ss >> cur; out[cur] = Mtl(); }
        else if (cur.empty()) continue;
        else if (tag == "Kd") ss >> out[cur].kd[0] >> out[cur].kd[1] >> out[cur].kd[2];
        else if (tag == "Ke") ss >> out[cur].ke[0] >> out[cur].ke[1] >> out[cur].ke[2];
        else if (tag == "Ns") ss >> out[cur].ns;
    }
    fclose(f);
}

int resolve(int idx, size_t count)
{
    if (idx > 0) return idx - 1;
    if (idx < 0) return (int)count + idx;
    return -1;
}

}  // namespace

extern "C" int cpt_obj_load(const char* path, float scale, const float* translate, float default_grey,
                            cpt_triangle* tris, cpt_triangle_info* infos, uint32_t capacity, uint32_t* n_out)
{
    CPT_RANGE("cpt_obj_load");
    if (!path || !n_out) return CPT_ERR_INVALID_ARGUMENT;
    FILE* f = fopen(path, "r");
    if (!f) return CPT_ERR_INVALID_ARGUMENT;
    const float tr[3] = {translate ? translate[0] : 0.f, translate ? translate[1] : 0.f, translate ? translate[2] : 0.f};
    std::vector<float> pos, col, uvs, nrm;
    std::map<std::string, Mtl> mtls;
    Mtl cur_mtl;
    bool have_mtl = false;
    const std::string base = dir_of(path);
    uint32_t n = 0;
    int rc = CPT_OK;
    std::string line;
    while (read_line(f, line)) {
        std::istringstream ss(strip_comment(line));
        std::string tag;
        if (!(ss >> tag)) continue;
        if (tag == "v") {
            float x = 0, y = 0, z = 0, r, g, b;
            ss >> x >> y >> z;
            pos.push_back(x * scale + tr[0]);
            pos.push_back(y * scale + tr[1]);
            pos.push_back(z * scale + tr[2]);
            if (ss >> r >> g >> b) { col.push_back(r); col.push_back(g); col.push_back(b); }
            else { col.push_back(-1.f); col.push_back(-1.f); col.push_back(-1.f); }
        } else if (tag == "vt") {
            float u = 0, v = 0;
            ss >> u >> v;
            uvs.push_back(u);
            uvs.push_back(v);
        } else if (tag == "vn") {
            float x = 0, y = 0, z = 0;
            ss >> x >> y >> z;
            nrm.push_back(x); nrm.push_back(y); nrm.push_back(z);
        } else if (tag == "mtllib") {
            std::string name;
            while (ss >> name) load_mtl(base + name, mtls);
        } else if (tag == "usemtl") {
            std::string name;
            ss >> name;
            auto it = mtls.find(name);
            have_mtl = it != mtls.end();
            if (have_mtl) cur_mtl = it->second;
        } else if (tag == "f") {
            std::vector<FaceVert> fv;
            std::string tok;
            while (ss >> tok) {
                FaceVert v;
                int a = 0, b = 0, c = 0;
                if (sscanf(tok.c_str(), "%d/%d/%d", &a, &b, &c) == 3) { v.has_t = v.has_n = true; }
                else if (sscanf(tok.c_str(), "%d//%d", &a, &c) == 2) { v.has_n = true; }
                else if (sscanf(tok.c_str(), "%d/%d", &a, &b) == 2) { v.has_t = true; }
                else if (sscanf(tok.c_str(), "%d", &a) != 1) continue;
                v.v = resolve(a, pos.size() / 3);
                if (v.has_t) v.t = resolve(b, uvs.size() / 2);
                if (v.has_n) v.n = resolve(c, nrm.size() / 3);
                if (v.v < 0 || (size_t)v.v >= pos.size() / 3 ||
                    (v.has_t && (v.t < 0 || (size_t)v.t >= uvs.size() / 2)) ||
                    (v.has_n && (v.n < 0 || (size_t)v.n >= nrm.size() / 3))) {
                    rc = CPT_ERR_INVALID_ARGUMENT;
                    break;
                }
                fv.push_back(v);
            }
            if (rc != CPT_OK) break;
            for (size_t k = 1; k + 1 < fv.size(); ++k) {
                const FaceVert c3[3] = {fv[0], fv[k], fv[k + 1]};
                if (tris) {
                    if (n >= capacity) { rc = CPT_ERR_SCRATCH_TOO_SMALL; break; }
                    cpt_triangle& t = tris[n];
                    float* dst[3] = {t.v0, t.v1, t.v2};
                    for (int j = 0; j < 3; ++j)
                        for (int a = 0; a < 3; ++a) dst[j][a] = pos[3 * c3[j].v + a];
                    t.info_idx = n;
                    if (infos) {
                        cpt_triangle_info& in = infos[n];
                        memset(&in, 0, sizeof(in));
                        // Triangle::computeNormal (geometry.h:27): normalize(cross(v1 - v0, v2 - v0))
                        float e1[3], e2[3], gn[3];
                        for (int a = 0; a < 3; ++a) { e1[a] = t.v1[a] - t.v0[a]; e2[a] = t.v2[a] - t.v0[a]; }
                        gn[0] = e1[1] * e2[2] - e2[1] * e1[2];
                        gn[1] = e1[2] * e2[0] - e2[2] * e1[0];
                        gn[2] = e1[0] * e2[1] - e2[0] * e1[1];
                        const float dd = (gn[0] * gn[0] + gn[1] * gn[1]) + gn[2] * gn[2];
                        const float s = 1.0f / sqrtf(dd);
                        for (int a = 0; a < 3; ++a) gn[a] = gn[a] * s;
                        for (int j = 0; j < 3; ++j) {
                            cpt_vertex& vx = in.vertices[j];
                            if (c3[j].t >= 0) { vx.uv[0] = uvs[2 * c3[j].t]; vx.uv[1] = uvs[2 * c3[j].t + 1]; }
                            const float* vc = &col[3 * c3[j].v];
                            for (int a = 0; a < 3; ++a) {
                                vx.color[a] = vc[0] >= 0.f ? vc[a] : (have_mtl && cur_mtl.kd[0] >= 0.f ? cur_mtl.kd[a]
                                                                                                       : default_grey);
                                vx.normal[a] = c3[j].n >= 0 ? nrm[3 * c3[j].n + a] : gn[a];
                            }
                        }
                        if (have_mtl) {
                            for (int a = 0; a < 3; ++a) in.material.emission[a] = cur_mtl.ke[a];
                            in.material.specularity = cur_mtl.ns;
                        }
                        in.material.albedo_idx = CPT_INVALID_INDEX;
                        in.material.normal_map_idx = CPT_INVALID_INDEX;
                    }
                }
                ++n;
            }
            if (rc != CPT_OK) break;
        }
    }
    fclose(f);
    *n_out = n;
    return rc;
}
