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
};

// Build over primitive boxes grown by `margin` (absolute, in scene units).
bool build_wide_bvh(const std::vector<Box>& boxes, double margin, WideBvh& out,
                    std::string& err);

// Refit: the same topology over new primitive boxes (grown by `margin`).  Every node's
// child boxes are recomputed bottom-up and quantized afresh, so the result is exactly as
// conservative as a build; only the tree's shape may be worse for the new boxes.
bool refit_wide_bvh(WideBvh& b, const std::vector<Box>& boxes, double margin, std::string& err);

// Structural check run on every bake: child and record indices in range, every node
// reachable once, every primitive referenced exactly once, children after parents.
bool validate_wide_bvh(const WideBvh& b, int n_prims, std::string& err);

}  // namespace ftb
