// ftb_layout.h -- device-resident data layout shared by the host baker (ftb_api.cpp,
// bvh_build.cpp) and the kernels (ftb_kernels.cu).
//
// HBM layout of a baked scene:
//   nodes   : FNode[n_nodes], 208 B each, 16 B aligned -- 8-wide BVH.  The builders make
//             compressed 80-byte WNodes (child boxes 8-bit quantized against the node's
//             float grid (p, 2^e), rounded outward, so the fp32 traversal never culls a
//             primitive the exact fp64 test would accept); the upload widens each to an
//             FNode holding the float planes that the bytes decode to.
//   recs    : PrimRec[n_recs], 80 B each -- one record per primitive, in leaf order.
//             Triangles keep their three vertices in double (the exact watertight test
//             reads them); the last 8 B carry the global primitive index, material and
//             type.  Leaf children of a node reference a contiguous run of records.
//   tri_n   : optional per-triangle shading normals (9 doubles), by triangle index.
//   planes  : DevPlane[n_planes] -- the planar mirrors the camera connections reflect in.
//   inst    : DevInst[n_inst], 128 B each -- instances of shared BLAS assets.  The world
//             hierarchy (TLAS) holds one REC_INST record per instance; a BLAS is a wide
//             BVH and triangle records of its own, in its local space.
//   spectra, tables, materials, emitters, media: small tables.
#pragma once
#include <stdint.h>

#define FTB_WIDTH 8
#define FTB_LEAF_MAX 4
#define FTB_STACK 64

enum { REC_TRI = 0, REC_SPHERE = 1, REC_CURVE = 2, REC_INST = 3 };

// meta byte of a child slot: 0 = empty; otherwise count<<5 | offset.  For an internal child
// (imask bit set) count is 1 and offset is the child's index relative to child_base; for a
// leaf child count is its number of records and offset is relative to prim_base.
struct alignas(16) WNode {
    float px, py, pz;
    uint8_t ex, ey, ez, imask;   // exponents biased by 127 (float exponent field)
    uint32_t child_base;
    uint32_t prim_base;
    uint8_t meta[8];
    uint8_t qlo_x[8], qlo_y[8], qlo_z[8];
    uint8_t qhi_x[8], qhi_y[8], qhi_z[8];
};
static_assert(sizeof(WNode) == 80, "WNode must be 80 bytes");

// The device form of a wide node: the same children, with each child plane stored as the
// float the 8-bit form decodes to (fmaf(q, 2^e, p), the value the builders check against
// the exact box), so traversal reads planes instead of decoding bytes.  Planes are kept
// per axis and side, so a ray takes its near and far planes by its direction's signs with
// no per-child select.  meta byte: 0 = empty; count<<5 | offset for a leaf (count 1..4,
// offset from prim_base); 7<<5 | offset for an inner child (offset from child_base).  An
// empty child has lo = +inf and hi = -inf on every axis, which every ray's slab test misses.
struct alignas(16) FNode {
    uint32_t child_base;
    uint32_t prim_base;
    uint8_t meta[8];
    float lo[3][8];
    float hi[3][8];
};
static_assert(sizeof(FNode) == 208, "FNode must be 208 bytes");
#define FNODE_INNER 7u

// 80-byte primitive record.  d[9] holds two int32: prim (global index) and
// info = mat | type << 24 | smooth << 30.  An instance record (REC_INST) keeps its instance
// index in d[0] (as an int64 bit pattern); a BLAS triangle's prim is its index in the BLAS.
struct alignas(16) PrimRec {
    double d[9];
    int32_t prim;
    int32_t info;
};
static_assert(sizeof(PrimRec) == 80, "PrimRec must be 80 bytes");

struct DevSpec {
    int32_t kind, n;
    int64_t offset;
    double p[6];
};

struct DevMat {
    int32_t type, priority, reflect, ior, absorb, transmit;
    double roughness;
};

struct DevEmit {
    int32_t shape, collimated, n, pad;
    double step, power;
    double origin[3], u[3], v[3], normal[3], beam[3];
    double radius;
    const double* cdf;
};

struct DevMed {
    int32_t sa, ss, bound, pad;
    double g;
    double bmin[3], bmax[3], center[3];
    double radius;
};

// One placement of a BLAS (MeshInstance, scene.h:1035-1063).
struct DevInst {
    double xl[12];            // world -> local map (toLocal): 3x3 row-major, then translation
    const FNode* nodes;       // the BLAS hierarchy and triangle records
    const PrimRec* recs;
    const double* tri_n;      // 9 per BLAS triangle or null
    int32_t mat_override, pad;
};
static_assert(sizeof(DevInst) == 128, "DevInst must be 128 bytes");

// A planar mirror (Scene::MirrorPlane, scene.h:1617-1623): the plane dot(n, x) == d of a
// group of coplanar planar-mirror triangles (unit normal flipped so its largest component
// is positive) and their AABB padded by 1e-6 (1 + diagonal).
struct DevPlane {
    double n[3], d;
    double lo[3], hi[3];
};

struct DevScene {
    const FNode* nodes;
    const PrimRec* recs;
    const double* tri_n;      // 9 per triangle (global index) or null
    const DevSpec* spec;
    const double* tw;
    const double* tv;
    const DevMat* mats;
    const DevEmit* emit;
    const double* emit_cdf;   // selection CDF over emitters
    const DevMed* med;
    const DevInst* inst;
    const DevPlane* planes;   // planar mirrors (camera connections by reflection)
    int32_t n_nodes, n_recs, n_mats, n_emit, n_med, n_spec;
    int32_t root2;            // second hierarchy (the curves') in nodes, or -1; with two, the
                              // last three nodes are a top node over both and copies of the roots
    int32_t n_planes;
    int64_t n_tris;
    int64_t n_inst;
    double total_power;
};

struct DevCam {
    double eye[3], u[3], v[3], w[3];
    double thx, thy;
    int32_t rx, ry;
};
