// bvh_build.h -- host-side BVH construction for the B200 ray caster.
//
// Builds the reference renderer's BVH exactly (src/Library/Acceleration/BVH.h:
// SAH-binned BVH2, 32 bins, leaf <= 4, Ctrav = Cint = 1, float boxes rounded
// outward by one ulp, then the BVH4 collapse) so hit ids can be compared with
// the reference bit for bit.  The build runs subtrees on all host cores and
// then renumbers nodes into the reference's depth-first pair order, which
// makes the node arrays byte-identical to a single-threaded reference build.
//
// The collapsed BVH4 is then re-encoded into one of two device layouts
// (GpuNode4 with FP32 child boxes, or QNode4 with 8-bit child boxes quantised
// conservatively against a per-node origin and power-of-two scale).
#pragma once
#include <cstdint>
#include <vector>

namespace rtb200 {

// Reference BVH2 node, 32 bytes (BVH.h:87-96).
struct Node2 {
    float bmin[3];
    float bmax[3];
    uint32_t first_or_left;
    uint16_t count;
    uint8_t axis;
    uint8_t pad;
};
static_assert(sizeof(Node2) == 32, "Node2 must be 32 bytes");

// Reference BVH4 node, 128 bytes (BVH.h:124-137).
struct alignas(16) Node4 {
    float minx[4], miny[4], minz[4];
    float maxx[4], maxy[4], maxz[4];
    int32_t child[4];
    uint16_t count[4];
    uint8_t nchild;
    uint8_t axis;
    uint8_t pad[6];
};
static_assert(sizeof(Node4) == 128, "Node4 must be 128 bytes");

struct BuiltBVH {
    std::vector<Node2> nodes2;
    std::vector<uint32_t> prims;   // leaf order -> input triangle index
    std::vector<Node4> nodes4;
};

// tri9: n_tri triangles, 9 floats each (v0, v1, v2).  threads <= 0 uses all
// host cores.
void BuildReferenceBVH(const float* tri9, int64_t n_tri, int threads, BuiltBVH& out);

// A BVH2 read from a file (the reference's .risemesh cache): valid when every
// internal node's child pair lies after it and inside the array, every node
// is reached once from the root, leaf ranges lie inside the n_prims leaf-order
// entries, and no path is deeper than kMaxBVH2Depth.
constexpr int kMaxBVH2Depth = 1024;
bool ValidBVH2(const std::vector<Node2>& nodes2, size_t n_prims);

// One mesh's BVH2 (prims: mesh-local triangle indices in leaf order) and the
// scene-wide index of its first triangle.
struct MeshBVH2 {
    const std::vector<Node2>* nodes2;
    const std::vector<uint32_t>* prims;
    int64_t first;
};

// Scene BVH over meshes with their own BVH2s (two levels, as the reference
// keeps one BVH per mesh): a binary top level over the meshes' root boxes,
// split at the median mesh centre along the widest axis, with each mesh's tree
// copied below it in depth-first pair order and its leaf ranges moved to the
// mesh's place in the scene-wide leaf order; then the BVH4 collapse.  One mesh
// alone keeps its node array as it is.
void MergeMeshBVHs(const std::vector<MeshBVH2>& meshes, BuiltBVH& out);

// ---- device layouts -------------------------------------------------------

// FP32 wide node: 4 child boxes as SoA float4 + child links, 128 bytes.
// child[i] >= 0: internal node index; child[i] == INT32_MIN: empty slot;
// other child[i] < 0: a leaf whose first triangle (in leaf order) is
// ~child[i], holding count[i] triangles (the last one carries
// GpuTri::v1[3] == 1).  The traversal reads the first 112 bytes only (empty
// slots are known from the link); count[i] (-1 for an empty slot) is kept
// for the host's view of the node.
struct alignas(16) GpuNode4 {
    float lox[4], loy[4], loz[4];
    float hix[4], hiy[4], hiz[4];
    int32_t child[4];
    int32_t count[4];
};
static_assert(sizeof(GpuNode4) == 128, "GpuNode4 must be 128 bytes");

// Quantised wide node, 64 bytes.  Child box bounds are 8-bit integers q with
// box = origin + q * 2^exp per axis; lower bounds are rounded down and upper
// bounds up, and the encoder verifies the FP32 decode still contains the FP32
// box, so culling is conservative.
struct alignas(16) QNode4 {
    float ox, oy, oz;              // origin (min corner of the union box)
    int8_t ex, ey, ez;             // power-of-two scale exponents
    uint8_t nchild;
    uint8_t qlo[3][4];             // [axis][child]
    uint8_t qhi[3][4];
    int32_t child[4];
    int16_t count[4];
};
static_assert(sizeof(QNode4) == 64, "QNode4 must be 64 bytes");

// Half-precision wide node, 64 bytes: the FP32 node's child boxes as IEEE
// binary16 (lower bounds rounded towards -inf, upper bounds towards +inf, so
// each decoded box contains the FP32 box; coordinates beyond the half range
// become -inf / +inf), the same links (kEmpty for an empty slot) and no
// counts (leaves end at the triangle flagged last, as for GpuNode4).
struct alignas(16) HNode4 {
    uint16_t lox[4], loy[4], loz[4];
    uint16_t hix[4], hiy[4], hiz[4];
    int32_t child[4];
};
static_assert(sizeof(HNode4) == 64, "HNode4 must be 64 bytes");

// binary16 <-> float on the host: the value of a half, and the half nearest
// to x in the given direction (-1 down, +1 up), exactly.
float HalfToFloat(uint16_t h);
uint16_t FloatToHalfDirected(float x, int dir);

// One triangle in leaf order: v0.w carries the input triangle index.
struct alignas(16) GpuTri {
    float v0[4];
    float v1[4];
    float v2[4];
};
static_assert(sizeof(GpuTri) == 48, "GpuTri must be 48 bytes");

// Eight-wide compressed node, 80 bytes (bvh_wide.cpp): per-node origin,
// power-of-two scale exponents and internal-child mask; the first internal
// child's node index (the others follow in slot order) and the first
// triangle of the leaf slots; per slot a meta byte (leaf: triangle count in
// unary in bits 5-7 above a 5-bit offset from tri_base; 0 otherwise) and
// 8-bit conservative bounds per axis.
struct alignas(16) WNode8 {
    float px, py, pz;
    int8_t ex, ey, ez;
    uint8_t imask;
    uint32_t child_base;
    uint32_t tri_base;
    uint8_t meta[8];
    uint8_t qlox[8], qloy[8], qloz[8];
    uint8_t qhix[8], qhiy[8], qhiz[8];
};
static_assert(sizeof(WNode8) == 80, "WNode8 must be 80 bytes");

// Collapse the BVH2 of `b` to eight-wide nodes in breadth-first order;
// prims receives the triangle order the nodes' triangle bases index, depth
// the number of node levels.  False when a leaf holds more than 24 triangles.
bool EncodeWideNodes(const BuiltBVH& b, std::vector<WNode8>& nodes, std::vector<uint32_t>& prims, int& depth);
void EncodeWideTriangles(const float* tri9, const std::vector<uint32_t>& prims, std::vector<GpuTri>& out);

// Both four-wide device layouts store the nodes in breadth-first order (root first), so
// the top levels, which every ray visits, share cache lines and pages.
void EncodeGpuNodes(const BuiltBVH& b, std::vector<GpuNode4>& out);
void EncodeQuantNodes(const BuiltBVH& b, std::vector<QNode4>& out);
void EncodeHalfNodes(const BuiltBVH& b, std::vector<HNode4>& out);
void EncodeTriangles(const float* tri9, const BuiltBVH& b, std::vector<GpuTri>& out);

// Upper bound on the traversal stack depth of the BVH4: the largest sum of
// (children - 1) over the internal nodes of one root-to-node path.  A
// depth-first walk that continues into one child and pushes the others holds
// at most this many deferred entries.
int TraceStackBound(const BuiltBVH& b);

// Traversal stack of the device kernels: kTraceStackShared entries per thread
// in shared memory; scenes whose bound is larger run kernels that continue the
// stack in local memory up to kTraceStackMax entries.  A scene whose bound
// exceeds kTraceStackMax is refused at commit.
constexpr int kTraceStackShared = 40;
constexpr int kTraceStackMax = 128;
// Eight-wide traversal: one stack entry per node level below the root, the
// rest for postponed triangle groups; trees deeper than kW8MaxLevels levels
// below the root are refused at commit.
constexpr int kW8StackEntries = 24;
constexpr int kW8MaxLevels = 12;

}  // namespace rtb200
