// Host-side check of the wide BVH's float planes (test infrastructure, built and run by
// tests/test_bvh_planes.py).  Builds trees over seeded box sets with the host builder, widens
// them to the device form and checks that every primitive's grown box lies inside the planes
// of every child slot on its path from the root -- the property that makes fp32 culling
// conservative -- for the builder's own float planes, for the planes decoded from the 8-bit
// form, and after a refit over moved boxes.  Prints one line per case; exit status 0 when
// every case holds.
#include <cmath>
#include <cstdio>
#include <random>
#include <string>
#include <vector>

#include "bvh_build.h"

namespace ftb {
// the device builder is not part of this check
bool build_wide_lbvh_device(const std::vector<Box>&, int, int, WideBvh&, std::string& err) {
    err = "no device";
    return false;
}
}  // namespace ftb

using namespace ftb;

namespace {

struct Checker {
    const WideBvh& b;
    const std::vector<FNode>& f;
    const std::vector<Box>& boxes;
    double margin;
    std::string err;

    // primitives of the subtree under slot k of node i
    void collect_slot(uint32_t i, int k, std::vector<int>& out) const {
        const FNode& n = f[i];
        const uint32_t m = n.meta[k];
        if ((m >> 5) == FNODE_INNER) {
            const uint32_t c = n.child_base + (m & 31u);
            for (int q = 0; q < FTB_WIDTH; ++q)
                if (f[c].meta[q]) collect_slot(c, q, out);
        } else {
            for (uint32_t r = 0; r < (m >> 5); ++r) out.push_back(b.order[n.prim_base + (m & 31u) + r]);
        }
    }

    bool node(uint32_t i) {
        const FNode& n = f[i];
        for (int k = 0; k < FTB_WIDTH; ++k) {
            const uint32_t m = n.meta[k];
            if (!m) {
                for (int a = 0; a < 3; ++a)
                    if (!(std::isinf(n.lo[a][k]) && n.lo[a][k] > 0 && std::isinf(n.hi[a][k]) && n.hi[a][k] < 0)) {
                        err = "empty slot without +inf / -inf planes";
                        return false;
                    }
                continue;
            }
            const uint32_t cnt = m >> 5;
            if (cnt != FNODE_INNER && (cnt < 1 || cnt > FTB_LEAF_MAX)) { err = "bad meta byte"; return false; }
            std::vector<int> prims;
            collect_slot(i, k, prims);
            for (int p : prims)
                for (int a = 0; a < 3; ++a) {
                    const double lo = boxes[(size_t)p].lo[a] - margin, hi = boxes[(size_t)p].hi[a] + margin;
                    if (!((double)n.lo[a][k] <= lo && hi <= (double)n.hi[a][k])) {
                        char buf[160];
                        std::snprintf(buf, sizeof buf, "node %u slot %d axis %d: [%.17g, %.17g] not inside [%.9g, %.9g]",
                                      i, k, a, lo, hi, (double)n.lo[a][k], (double)n.hi[a][k]);
                        err = buf;
                        return false;
                    }
                }
            if (cnt == FNODE_INNER && !node(n.child_base + (m & 31u))) return false;
        }
        return true;
    }
};

bool check(const WideBvh& b, const std::vector<Box>& boxes, double margin, std::string& err) {
    if (!validate_wide_bvh(b, (int)boxes.size(), err)) return false;
    const std::vector<FNode> f = widen_nodes(b);
    Checker c{b, f, boxes, margin, {}};
    if (!c.node(0)) { err = c.err; return false; }
    return true;
}

double maxabs(const std::vector<Box>& boxes) {
    double m = 1.0;
    for (const Box& b : boxes)
        for (int a = 0; a < 3; ++a) m = std::fmax(m, std::fmax(std::fabs(b.lo[a]), std::fabs(b.hi[a])));
    return m;
}

Box box_at(const double* c, const double* h) {
    Box b;
    for (int a = 0; a < 3; ++a) { b.lo[a] = c[a] - h[a]; b.hi[a] = c[a] + h[a]; }
    return b;
}

std::vector<Box> make_set(int kind, int n, std::mt19937_64& rng) {
    std::uniform_real_distribution<double> u(0.0, 1.0);
    std::vector<Box> out;
    for (int i = 0; i < n; ++i) {
        double c[3], h[3];
        for (int a = 0; a < 3; ++a) {
            switch (kind) {
                case 0: c[a] = 2.0 * u(rng) - 1.0; h[a] = 0.01 * u(rng); break;                 // unit cube
                case 1: c[a] = 1000.0 + 0.5 * u(rng); h[a] = 1e-5 * u(rng); break;              // far from 0, tiny
                case 2: c[a] = (i % 7) * 0.25; h[a] = (a == 1) ? 0.0 : 0.1; break;              // repeated, flat
                default: c[a] = std::ldexp(2.0 * u(rng) - 1.0, (int)(40 * u(rng)) - 20);       // mixed scales
                         h[a] = std::ldexp(u(rng), (int)(30 * u(rng)) - 25); break;
            }
        }
        out.push_back(box_at(c, h));
    }
    return out;
}

}  // namespace

int main() {
    std::mt19937_64 rng(12345);
    const char* names[4] = {"unit", "far", "repeated_flat", "mixed_scales"};
    int failures = 0;
    for (int kind = 0; kind < 4; ++kind) {
        for (int n : {1, 5, 33, 4000}) {
            std::vector<Box> boxes = make_set(kind, n, rng);
            const double margin = std::ldexp(maxabs(boxes), -18);
            WideBvh b;
            std::string err;
            bool ok = build_wide_bvh(boxes, margin, b, err) && check(b, boxes, margin, err);
            // the same tree through the 8-bit planes alone
            if (ok) {
                WideBvh q = b;
                q.planes.clear();
                ok = check(q, boxes, margin, err);
                if (!ok) err = "decoded planes: " + err;
            }
            // a refit over moved boxes
            if (ok) {
                std::uniform_real_distribution<double> u(-0.05, 0.05);
                std::vector<Box> moved = boxes;
                for (Box& x : moved)
                    for (int a = 0; a < 3; ++a) { const double d = u(rng) * (x.hi[a] - x.lo[a] + 1e-3); x.lo[a] += d; x.hi[a] += d; }
                const double m2 = std::ldexp(maxabs(moved), -18);
                ok = refit_wide_bvh(b, moved, m2, err) && check(b, moved, m2, err);
                if (!ok) err = "refit: " + err;
            }
            std::printf("%s n=%d nodes=%zu: %s\n", names[kind], n, b.nodes.size(), ok ? "ok" : err.c_str());
            failures += ok ? 0 : 1;
        }
    }
    // the check itself: one leaf plane moved inward by one float step must be caught
    {
        std::vector<Box> boxes = make_set(0, 500, rng);
        const double margin = std::ldexp(maxabs(boxes), -18);
        WideBvh b;
        std::string err;
        bool built = build_wide_bvh(boxes, margin, b, err);
        bool caught = false;
        for (size_t i = 0; built && i < b.nodes.size() && !caught; ++i)
            for (int k = 0; k < FTB_WIDTH && !caught; ++k)
                if (b.nodes[i].meta[k] && !((b.nodes[i].imask >> k) & 1)) {
                    float& lo = b.planes[i * FTB_PLANES + k];   // lo x of slot k
                    lo = std::nextafterf(lo, INFINITY);
                    caught = !check(b, boxes, margin, err);
                    break;
                }
        std::printf("planted one-step plane error: %s\n", caught ? "caught" : "missed");
        failures += caught ? 0 : 1;
    }
    return failures == 0 ? 0 : 1;
}
