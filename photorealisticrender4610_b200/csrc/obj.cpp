// OBJ ingest with the semantics of the reference's MeshTriangle(filename,
// offset, m) (Triangle.cpp:4-32), which reads the file with the OBJ loader
// bundled in the reference tree (OBJ_Loader.hpp, Loader::LoadFile:427-700)
// and then takes the FIRST loaded mesh's vertex list three entries at a time
// as triangles, each position shifted by `offset`.
//
// What that loader puts into a mesh's vertex list, restated here:
//  - every "f" line appends one vertex per face corner, in line order; a
//    corner is "p", "p/t", "p//n" or "p/t/n" and only its position matters
//    for the triangles (GenVerticesFromRawOBJ:723-830). Polygons with more
//    than three corners append all their corners, so the triangles the
//    reference forms from them straddle faces; that is kept as is.
//  - indices are 1-based, negative ones count back from the end
//    (algorithm::getElement:392-401).
//  - a mesh is closed (and the next begins) at an "o"/"g" line (or any line
//    starting with 'g') once one has been seen before, at a "usemtl" line,
//    and at the end of the file; a mesh with no face is not created.
//  - tokens: the first token of a line is what precedes the first blank or
//    tab; the rest of the line is split on single spaces, empty pieces
//    included (algorithm::split:317-352), so numbers are separated by one
//    space; numbers are read with strtof / strtol as std::stof / std::stoi.
// The reference asserts that the file holds exactly one mesh and reads past
// its vertex list when the corner count is not a multiple of three; both are
// reported as errors here, as are unreadable numbers and indices out of range.
#include "prr_internal.h"

#include <cerrno>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

namespace prr {
namespace {

std::string first_token(const std::string &s) {
    const size_t a = s.find_first_not_of(" \t");
    if (a == std::string::npos)
        return "";
    const size_t b = s.find_first_of(" \t", a);
    return b == std::string::npos ? s.substr(a) : s.substr(a, b - a);
}

std::string rest_of(const std::string &s) {
    const size_t a = s.find_first_not_of(" \t");
    if (a == std::string::npos)
        return "";
    const size_t sp = s.find_first_of(" \t", a);
    if (sp == std::string::npos)
        return "";
    const size_t b = s.find_first_not_of(" \t", sp);
    if (b == std::string::npos)
        return "";
    const size_t e = s.find_last_not_of(" \t");
    return s.substr(b, e - b + 1);
}

// Pieces of `in` between single `sep` characters: a separator with nothing
// pending gives an empty piece; the tail after the last separator is a piece
// when non-empty.
std::vector<std::string> pieces(const std::string &in, char sep) {
    std::vector<std::string> out;
    std::string cur;
    for (size_t i = 0; i < in.size(); i++) {
        if (in[i] == sep) {
            out.push_back(cur);
            cur.clear();
        } else {
            cur += in[i];
            if (i + 1 == in.size())
                out.push_back(cur);
        }
    }
    return out;
}

bool read_float(const std::string &s, float &v) {
    const char *p = s.c_str();
    char *end = nullptr;
    errno = 0;
    v = std::strtof(p, &end);
    return end != p && errno != ERANGE;
}

bool read_index(const std::string &s, size_t count, size_t &out) {
    const char *p = s.c_str();
    char *end = nullptr;
    errno = 0;
    const long v = std::strtol(p, &end, 10);
    if (end == p || errno == ERANGE)
        return false;
    const long k = v < 0 ? (long) count + v : v - 1;
    if (k < 0 || k >= (long) count)
        return false;
    out = (size_t) k;
    return true;
}

} // namespace

// The positions of the first mesh's corners (x, y, z each) plus `offset`.
int obj_first_mesh(const char *path, const float offset[3], std::vector<float> &verts) {
    const std::string p = path;
    if (p.size() < 4 || p.compare(p.size() - 4, 4, ".obj") != 0)
        return fail(PRR_ERR_INVALID_ARGUMENT, "OBJ: the file name must end in .obj");
    std::ifstream f(p);
    if (!f)
        return fail(PRR_ERR_INVALID_ARGUMENT, "OBJ: cannot open " + p);
    std::vector<float> pos;           // x y z per "v" line
    std::vector<float> cur, first;    // corners of the open mesh / of the first mesh
    bool cur_faces = false;           // the open mesh has a face
    bool grouping = false;            // an "o"/"g" line has been seen
    int meshes = 0;
    auto close_mesh = [&] {
        if (!cur_faces)
            return;
        if (meshes == 0)
            first = cur;
        meshes++;
        cur.clear();
        cur_faces = false;
    };
    std::string line;
    int64_t lineno = 0;
    while (std::getline(f, line)) {
        lineno++;
        const std::string tok = first_token(line);
        auto bad = [&](const char *what) {
            return fail(PRR_ERR_INVALID_ARGUMENT,
                        "OBJ: " + std::string(what) + " on line " + std::to_string(lineno));
        };
        if (tok == "o" || tok == "g" || (!line.empty() && line[0] == 'g')) {
            if (grouping)
                close_mesh();
            grouping = true;
        }
        if (tok == "v") {
            const std::vector<std::string> c = pieces(rest_of(line), ' ');
            float x, y, z;
            if (c.size() < 3 || !read_float(c[0], x) || !read_float(c[1], y) ||
                !read_float(c[2], z))
                return bad("unreadable vertex position");
            pos.push_back(x);
            pos.push_back(y);
            pos.push_back(z);
        } else if (tok == "f") {
            const std::vector<std::string> corners = pieces(rest_of(line), ' ');
            int added = 0;
            for (const std::string &c : corners) {
                const std::vector<std::string> parts = pieces(c, '/');
                if (parts.empty() || parts.size() > 3)
                    continue; // not a corner form the loader knows: no vertex
                size_t k;
                if (!read_index(parts[0], pos.size() / 3, k))
                    return bad("face corner with a bad position index");
                cur.push_back(pos[3 * k]);
                cur.push_back(pos[3 * k + 1]);
                cur.push_back(pos[3 * k + 2]);
                added++;
            }
            if (added >= 3)
                cur_faces = true;
        } else if (tok == "usemtl") {
            close_mesh();
        }
    }
    close_mesh();
    if (meshes != 1)
        return fail(PRR_ERR_INVALID_ARGUMENT,
                    "OBJ: MeshTriangle takes a file with exactly one mesh; " + p + " holds " +
                        std::to_string(meshes));
    if ((first.size() / 3) % 3 != 0)
        return fail(PRR_ERR_INVALID_ARGUMENT,
                    "OBJ: the mesh's corner count is not a multiple of three");
    const float ox = offset ? offset[0] : 0.f, oy = offset ? offset[1] : 0.f,
                oz = offset ? offset[2] : 0.f;
    verts.resize(first.size());
    for (size_t i = 0; i < first.size(); i += 3) {
        verts[i] = first[i] + ox;
        verts[i + 1] = first[i + 1] + oy;
        verts[i + 2] = first[i + 2] + oz;
    }
    return PRR_OK;
}

} // namespace prr

using namespace prr;

extern "C" {

int prr_obj_read(const char *path, const float *offset, float *out_verts, int64_t capacity,
                 int64_t *out_ntri) {
    if (!path || !out_ntri)
        return fail(PRR_ERR_INVALID_ARGUMENT, "path and out_ntri are required");
    std::vector<float> v;
    if (int rc = obj_first_mesh(path, offset, v))
        return rc;
    const int64_t ntri = (int64_t) v.size() / 9;
    *out_ntri = ntri;
    if (out_verts) {
        if (capacity < ntri)
            return fail(PRR_ERR_INVALID_ARGUMENT, "out_verts holds fewer triangles than the mesh");
        std::copy(v.begin(), v.end(), out_verts);
    }
    return PRR_OK;
}

int prr_scene_add_obj(prr_scene *scene, const char *path, const float *offset, int material,
                      int *out_object) {
    if (!scene || !path)
        return fail(PRR_ERR_INVALID_ARGUMENT, "scene and path are required");
    std::vector<float> v;
    if (int rc = obj_first_mesh(path, offset, v))
        return rc;
    if (v.empty())
        return fail(PRR_ERR_INVALID_ARGUMENT, "OBJ: the mesh has no triangle");
    return prr_scene_add_mesh(scene, v.data(), (int64_t) v.size() / 9, material, out_object);
}

} // extern "C"
