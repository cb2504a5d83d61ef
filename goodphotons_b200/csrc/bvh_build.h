// bvh_build.h -- host builder of the compressed 8-wide BVH.
#pragma once
#include <cfloat>
#include <string>
#include <vector>

#include "ftb_layout.h"

namespace ftb {

struct Box {
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX};
    double hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    void grow(const Box& b) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = b.lo[a] < lo[a] ? b.lo[a] : lo[a];
            hi[a] = b.hi[a] > hi[a] ? b.hi[a] : hi[a];
        }
    }
    void grow_point(const double* p) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = p[a] < lo[a] ? p[a] : lo[a];
            hi[a] = p[a] > hi[a] ? p[a] : hi[a];
        }
    }
};

struct WideBvh {
    std::vector<WNode> nodes;   // root at 0
    std::vector<int> order;     // record i holds primitive order[i]
    // Per node, FTB_PLANES floats: lo[3][8] then hi[3][8], each child's (grown) box rounded
    // outward to float; an empty slot is +inf / -inf.  Empty when a producer keeps only the
    // 8-bit planes (the device form then uses their decoded values).
    std::vector<float> planes;
};
#define FTB_PLANES 48

// A binary tree: root 0; a node with count > 0 is a leaf over idx[first, first + count).
struct BinNode {
    Box box;
    int left = -1, right = -1, first = 0, count = 0;
};

enum class BuildMethod {
    kHostSah,      // binned SAH (32 bins, 3 axes) on the host: the better tree
    kDeviceLbvh    // Morton-ordered radix tree on the GPU: a faster build, a looser tree
};

// Build over primitive boxes grown by `margin` (absolute, in scene units): a binary tree by
// `method`, collapsed to 8-wide nodes with conservative 8-bit child planes.
bool build_wide_bvh(const std::vector<Box>& boxes, double margin, WideBvh& out,
                    std::string& err, BuildMethod method = BuildMethod::kHostSah, int device = 0);

// The collapse: each wide node opens the binary child of largest surface area until it has
// 8 children; leaf children become runs of records laid out per wide node.
bool collapse_to_wide(const std::vector<BinNode>& nodes, const std::vector<int>& idx, WideBvh& out,
                      std::string& err);

// Linear BVH on `device` (bvh_device.cu): 63-bit Morton codes of the box centres, a radix
// sort, the Karras radix tree and bottom-up boxes (subtrees of at most leaf_size primitives
// become leaves), collapsed to 8-wide nodes on the device as well.  Boxes are grown already.
bool build_wide_lbvh_device(const std::vector<Box>& boxes, int leaf_size, int device, WideBvh& out,
                            std::string& err);

// Refit: the same topology over new primitive boxes (grown by `margin`).  Every node's
// child boxes are recomputed bottom-up and quantized afresh, so the result is exactly as
// conservative as a build; only the tree's shape may be worse for the new boxes.
bool refit_wide_bvh(WideBvh& b, const std::vector<Box>& boxes, double margin, std::string& err);

// The device form of a tree: each child's box as `planes` holds it (the exact box rounded
// outward to float), or, without planes, as the floats its bytes decode to (fmaf(q, 2^e, p),
// the values the quantization was checked against); inner children marked in the meta byte,
// empty children as boxes no ray enters.
std::vector<FNode> widen_nodes(const WideBvh& bvh);

// Outward float rounding of a box bound.
float round_down(double x);
float round_up(double x);

// Structural check run on every bake: child and record indices in range, every node
// reachable once, every primitive referenced exactly once, children after parents.
bool validate_wide_bvh(const WideBvh& b, int n_prims, std::string& err);

}  // namespace ftb
