// risemesh.cpp -- reader for the reference's .risemesh files
// (TriangleMeshGeometryIndexed::Serialize / Deserialize,
// Geometry/TriangleMeshGeometryIndexed.cpp:585-980) and their BVH2 cache
// (BVH::Serialize / Deserialize, Acceleration/BVH.h:338-423).
//
// Layout (little-endian, as the reference's MemoryBuffer writes it):
//   "RISETMGI"  8 bytes, uint32 version (1..5)
//   v1..v3:     uint32 + char (legacy octree settings, discarded)
//   char        face normals
//   uint32 n, n x 3 doubles     points
//   uint32 n, n x 3 doubles     normals
//   uint32 n, n x 2 doubles     texture coordinates
//   v5:         uint32 n, n x 3 doubles (vertex colours)
//   uint32 n, n x 3 x (uint32 point, uint32 normal, uint32 coord)   triangles
//   char        double sided
//   v1..v3:     char use-BSP, char have-tree (+ the legacy tree's bytes)
//   v3+, n > 0: char have-BVH; "BVH2", uint32 1, uint32 nodes, nodes x 32
//               bytes, uint32 prims, prims x uint32, 6 doubles (root box)
//
// Files of v1..v3 that carry a legacy BSP / octree block are refused: the
// block is only skipped by parsing it, and the trees are not used anyway.
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "core.h"

using namespace rtb200;

struct rtb200_risemesh {
    int32_t version = 0;
    bool face_normals = false;
    bool double_sided = false;
    std::vector<double> points;        // 3 per point
    std::vector<uint32_t> tri;         // point indices, 3 per triangle
    std::vector<double> normals;       // 3 per normal (none when the mesh uses face normals)
    std::vector<uint32_t> tri_nrm;     // normal indices, 3 per triangle
    bool has_bvh = false;
    std::vector<Node2> nodes2;
    std::vector<uint32_t> prims;
};

namespace {

class Reader {
public:
    Reader(const uint8_t* p, size_t n) : p_(p), n_(n) {}
    bool Bytes(void* dst, size_t k)
    {
        if (k > n_ - at_) return false;
        std::memcpy(dst, p_ + at_, k);
        at_ += k;
        return true;
    }
    bool U32(uint32_t& v) { return Bytes(&v, 4); }
    bool Char(char& c) { return Bytes(&c, 1); }
    bool Skip(size_t k)
    {
        if (k > n_ - at_) return false;
        at_ += k;
        return true;
    }
    // n items of `item` bytes must fit in what is left.
    bool Fits(uint64_t n, uint64_t item) const { return item == 0 || n <= (uint64_t)(n_ - at_) / item; }

private:
    const uint8_t* p_;
    size_t n_;
    size_t at_ = 0;
};

bool Parse(const uint8_t* bytes, size_t len, rtb200_risemesh& m)
{
    Reader r(bytes, len);
    char sig[8];
    if (!r.Bytes(sig, 8) || std::memcmp(sig, "RISETMGI", 8) != 0) return false;
    uint32_t ver = 0;
    if (!r.U32(ver) || ver < 1 || ver > 5) return false;
    m.version = (int32_t)ver;
    char c = 0;
    if (ver < 4 && !(r.Skip(4) && r.Skip(1))) return false;
    if (!r.Char(c)) return false;
    m.face_normals = c != 0;
    uint32_t n = 0;
    if (!r.U32(n) || !r.Fits(n, 24)) return false;
    m.points.resize(3 * (size_t)n);
    if (!r.Bytes(m.points.data(), 24 * (size_t)n)) return false;
    const uint32_t n_points = n;
    if (!r.U32(n) || !r.Fits(n, 24)) return false;     // normals
    m.normals.resize(3 * (size_t)n);
    if (!r.Bytes(m.normals.data(), 24 * (size_t)n)) return false;
    const uint32_t n_normals = n;
    if (!r.U32(n) || !r.Fits(n, 16) || !r.Skip(16 * (size_t)n)) return false;     // texture coordinates
    const uint32_t n_coords = n;
    if (ver >= 5 && !(r.U32(n) && r.Fits(n, 24) && r.Skip(24 * (size_t)n))) return false;   // colours
    if (!r.U32(n) || !r.Fits(n, 36)) return false;
    m.tri.resize(3 * (size_t)n);
    m.tri_nrm.resize(3 * (size_t)n);
    for (uint32_t t = 0; t < n; ++t)
        for (int i = 0; i < 3; ++i) {
            uint32_t v[3];
            if (!r.Bytes(v, 12)) return false;
            // The reference indexes the point, normal and coordinate lists
            // without checks; here every point index must be valid, and
            // normal / coordinate indices too where those lists are present.
            if (v[0] >= n_points) return false;
            if (n_normals > 0 && !m.face_normals && v[1] >= n_normals) return false;
            if (n_coords > 0 && v[2] >= n_coords) return false;
            m.tri[3 * (size_t)t + i] = v[0];
            m.tri_nrm[3 * (size_t)t + i] = v[1];
        }
    const uint32_t n_tri = n;
    if (!r.Char(c)) return false;
    m.double_sided = c != 0;
    if (ver < 4) {
        char use_bsp = 0, have_tree = 0;
        if (!r.Char(use_bsp) || !r.Char(have_tree)) return false;
        if (have_tree) return false;
    }
    if (ver >= 3 && n_tri > 0) {
        char have = 0;
        if (!r.Char(have)) return false;
        if (have) {
            char magic[4];
            uint32_t bver = 0, nn = 0, np = 0;
            if (!r.Bytes(magic, 4) || std::memcmp(magic, "BVH2", 4) != 0 || !r.U32(bver) || bver != 1) return false;
            if (!r.U32(nn) || !r.Fits(nn, sizeof(Node2))) return false;
            m.nodes2.resize(nn);
            if (!r.Bytes(m.nodes2.data(), sizeof(Node2) * (size_t)nn)) return false;
            // A cache lists every triangle once in leaf order.
            if (!r.U32(np) || np != n_tri || !r.Fits(np, 4)) return false;
            m.prims.resize(np);
            if (!r.Bytes(m.prims.data(), 4 * (size_t)np)) return false;
            for (uint32_t i = 0; i < np; ++i)
                if (m.prims[i] >= n_tri) return false;
            double box[6];
            if (!r.Bytes(box, sizeof(box))) return false;
            m.has_bvh = true;
        }
    }
    return true;
}

}  // namespace

extern "C" {

int rtb200_risemesh_parse(const void* bytes, size_t n_bytes, rtb200_risemesh** out)
{
    if (!bytes || !out) return RTB200_E_INVALID;
    *out = nullptr;
    rtb200_risemesh* m = new (std::nothrow) rtb200_risemesh();
    if (!m) return RTB200_E_OOM;
    bool ok = false;
    try {
        ok = Parse((const uint8_t*)bytes, n_bytes, *m);
    } catch (const std::bad_alloc&) {
        delete m;
        return RTB200_E_OOM;
    }
    if (!ok) {
        delete m;
        return RTB200_E_INVALID;
    }
    *out = m;
    return RTB200_OK;
}

int rtb200_risemesh_info(const rtb200_risemesh* m, int32_t* version, int64_t* n_points, int64_t* n_tri,
                         int32_t* double_sided, int64_t* n_bvh_nodes)
{
    if (!m) return RTB200_E_INVALID;
    if (version) *version = m->version;
    if (n_points) *n_points = (int64_t)(m->points.size() / 3);
    if (n_tri) *n_tri = (int64_t)(m->tri.size() / 3);
    if (double_sided) *double_sided = m->double_sided ? 1 : 0;
    if (n_bvh_nodes) *n_bvh_nodes = m->has_bvh ? (int64_t)m->nodes2.size() : 0;
    return RTB200_OK;
}

int rtb200_risemesh_triangles(const rtb200_risemesh* m, float* tri9)
{
    if (!m || (!tri9 && !m->tri.empty())) return RTB200_E_INVALID;
    for (size_t i = 0; i < m->tri.size(); ++i)
        for (int k = 0; k < 3; ++k) tri9[3 * i + k] = (float)m->points[3 * (size_t)m->tri[i] + k];
    return RTB200_OK;
}

int rtb200_risemesh_normals(const rtb200_risemesh* m, float* nrm9)
{
    if (!m || m->face_normals || m->normals.empty() || (!nrm9 && !m->tri.empty())) return RTB200_E_INVALID;
    for (size_t i = 0; i < m->tri_nrm.size(); ++i)
        for (int k = 0; k < 3; ++k) nrm9[3 * i + k] = (float)m->normals[3 * (size_t)m->tri_nrm[i] + k];
    return RTB200_OK;
}

int rtb200_risemesh_destroy(rtb200_risemesh* m)
{
    delete m;
    return RTB200_OK;
}

}  // extern "C"

namespace rtb200 {

bool RisemeshTriangles(const rtb200_risemesh* m, std::vector<float>& xyz, std::vector<uint32_t>& tri)
{
    xyz.resize(m->points.size());
    for (size_t i = 0; i < m->points.size(); ++i) xyz[i] = (float)m->points[i];
    tri = m->tri;
    return true;
}

const std::vector<Node2>* RisemeshBvh(const rtb200_risemesh* m, const std::vector<uint32_t>** prims)
{
    if (!m->has_bvh) return nullptr;
    *prims = &m->prims;
    return &m->nodes2;
}

bool RisemeshDoubleSided(const rtb200_risemesh* m) { return m->double_sided; }

// Vertex normals for shading: the file's normal list and per-corner indices,
// unless the mesh shades with face normals or stores no normals.
bool RisemeshNormals(const rtb200_risemesh* m, std::vector<float>& nrm, std::vector<uint32_t>& tri_nrm)
{
    if (m->face_normals || m->normals.empty()) return false;
    nrm.resize(m->normals.size());
    for (size_t i = 0; i < m->normals.size(); ++i) nrm[i] = (float)m->normals[i];
    tri_nrm = m->tri_nrm;
    return true;
}

}  // namespace rtb200
