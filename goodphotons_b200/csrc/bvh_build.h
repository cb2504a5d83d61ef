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

#ifdef __CUDACC__
#define FTB_HD __host__ __device__
#else
#define FTB_HD
#endif

// Child slots of a wide node by direction.  Slot s stands for the octant direction v_s
// whose component a is -1 where bit a of s is set and +1 where it is clear; the children
// (box centres cen[k], k < nk) are placed greedily, the (child, slot) pair with the largest
// projection of (centre - node centre) on v_s first.  A ray whose direction has its
// positive components where the bits of s are set then meets slot s's child first, the
// slots one bit away next, and so on: traversal visits children in slot order s ^ x for a
// per-ray x, an approximate near-to-far order that needs no sorting.
FTB_HD inline void octant_slots(const double (*cen)[3], int nk, const double* node_c, int* slot_of) {
    double cost[8][8];
    for (int k = 0; k < nk; ++k)
        for (int s = 0; s < 8; ++s) {
            double c = 0.0;
            for (int a = 0; a < 3; ++a) c += ((s >> a) & 1) ? node_c[a] - cen[k][a] : cen[k][a] - node_c[a];
            cost[k][s] = c;
        }
    unsigned used = 0, placed = 0;
    for (int it = 0; it < nk; ++it) {
        int bk = -1, bs = -1;
        double bc = 0.0;
        for (int k = 0; k < nk; ++k) {
            if ((placed >> k) & 1) continue;
            for (int s = 0; s < 8; ++s) {
                if ((used >> s) & 1) continue;
                if (bk < 0 || cost[k][s] > bc) { bk = k; bs = s; bc = cost[k][s]; }
            }
        }
        slot_of[bk] = bs;
        placed |= 1u << bk;
        used |= 1u << bs;
    }
}

struct WideBvh {
    std::vector<WNode> nodes;   // root at 0
    std::vector<int> order;     // record i holds primitive order[i]
};

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

// Structural check run on every bake: child and record indices in range, every node
// reachable once, every primitive referenced exactly once, children after parents.
bool validate_wide_bvh(const WideBvh& b, int n_prims, std::string& err);

}  // namespace ftb
