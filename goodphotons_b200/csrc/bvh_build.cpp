// bvh_build.cpp -- host builder of the compressed 8-wide BVH (layout in ftb_layout.h).
//
// The reference builds a binary binned-SAH tree (bvh.h:89-176, 16 bins, leaves of <= 4)
// and walks it with a double slab test.  Here the binary SAH tree is only an intermediate:
// it is collapsed into 8-wide nodes (each step opens the child with the largest surface
// area) and every child box is quantized to 8 bits against the node's float grid, rounded
// outward, after growing it by a margin that covers the fp32 rounding of the device's slab
// test.  The result is conservative: a primitive whose exact (fp64) intersection would be
// accepted is never culled.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "bvh_build.h"

namespace ftb {

namespace {
// One float step toward -inf / +inf (f not NaN), by the bit pattern: the builders round every
// child plane outward, millions per scene, so this avoids a library call per plane.
inline float step_down(float f) {
    if (f == 0.0f) return -std::numeric_limits<float>::denorm_min();
    uint32_t b;
    std::memcpy(&b, &f, sizeof b);
    b = f > 0.0f ? b - 1u : b + 1u;   // +inf steps to FLT_MAX; -inf is never stepped down
    std::memcpy(&f, &b, sizeof f);
    return f;
}
inline float step_up(float f) { return -step_down(-f); }
}  // namespace

float round_down(double x) {
    const float f = (float)x;
    return (double)f > x ? step_down(f) : f;
}

float round_up(double x) {
    const float f = (float)x;
    return (double)f < x ? step_up(f) : f;
}

namespace {
// A node's child boxes, outward to float, into its FTB_PLANES floats (n filled slots).
void put_planes(float* dst, const double (&clo)[3][8], const double (&chi)[3][8], int n) {
    for (int a = 0; a < 3; ++a)
        for (int k = 0; k < FTB_WIDTH; ++k) {
            dst[8 * a + k] = k < n ? round_down(clo[a][k]) : INFINITY;
            dst[24 + 8 * a + k] = k < n ? round_up(chi[a][k]) : -INFINITY;
        }
}
}  // namespace

namespace {

// Largest leaf of the binary build (<= FTB_LEAF_MAX, which the node encoding allows);
// 2 measured fastest on B200 (leaf sizes 1-4 on the glass, Cornell and fog workloads).
#ifndef FTB_BUILD_LEAF
#define FTB_BUILD_LEAF 2
#endif
constexpr int kLeafSize = FTB_BUILD_LEAF;

using BNode = BinNode;

double area(const Box& b) {
    double dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    if (dx < 0 || dy < 0 || dz < 0) return 0.0;
    return 2.0 * (dx * dy + dy * dz + dz * dx);
}

struct Builder {
    const std::vector<Box>& boxes;
    std::vector<int> idx;
    std::vector<double> cx, cy, cz;
    std::vector<BNode> nodes;
    explicit Builder(const std::vector<Box>& b) : boxes(b) {}

    double cent(int p, int a) const { return a == 0 ? cx[p] : (a == 1 ? cy[p] : cz[p]); }

    int build(int start, int end) {
        int ni = (int)nodes.size();
        nodes.push_back(BNode{});
        Box b, cb;
        for (int i = start; i < end; ++i) {
            int p = idx[i];
            b.grow(boxes[p]);
            double c[3] = {cx[p], cy[p], cz[p]};
            cb.grow_point(c);
        }
        int count = end - start;
        nodes[ni].box = b;
        if (count <= kLeafSize) {
            nodes[ni].first = start; nodes[ni].count = count;
            return ni;
        }
        // binned SAH over all three axes
        const int NB = 32;
        int best_axis = -1, best_split = -1;
        double best_cost = DBL_MAX;
        for (int a = 0; a < 3; ++a) {
            double lo = cb.lo[a], hi = cb.hi[a];
            if (!(hi - lo > 1e-12)) continue;
            double scale = NB / (hi - lo);
            Box bb[NB]; int bc[NB] = {0};
            for (int i = start; i < end; ++i) {
                int p = idx[i];
                int k = (int)((cent(p, a) - lo) * scale);
                k = k < 0 ? 0 : (k >= NB ? NB - 1 : k);
                bc[k]++; bb[k].grow(boxes[p]);
            }
            double ra[NB]; int rc[NB];
            Box acc; int n = 0;
            for (int k = NB - 1; k >= 1; --k) {
                acc.grow(bb[k]); n += bc[k];
                ra[k] = area(acc); rc[k] = n;
            }
            Box lacc; int ln = 0;
            for (int k = 0; k < NB - 1; ++k) {
                lacc.grow(bb[k]); ln += bc[k];
                if (ln == 0 || rc[k + 1] == 0) continue;
                double cost = ln * area(lacc) + rc[k + 1] * ra[k + 1];
                if (cost < best_cost) { best_cost = cost; best_axis = a; best_split = k; }
            }
        }
        int mid = start;
        if (best_axis >= 0) {
            double lo = cb.lo[best_axis], hi = cb.hi[best_axis];
            double scale = NB / (hi - lo);
            auto it = std::partition(idx.begin() + start, idx.begin() + end, [&](int p) {
                int k = (int)((cent(p, best_axis) - lo) * scale);
                k = k < 0 ? 0 : (k >= NB ? NB - 1 : k);
                return k <= best_split;
            });
            mid = (int)(it - idx.begin());
        }
        if (mid == start || mid == end) {
            // degenerate: median split on the widest centroid axis, or by index
            int a = 0;
            double ext = -1.0;
            for (int k = 0; k < 3; ++k)
                if (cb.hi[k] - cb.lo[k] > ext) { ext = cb.hi[k] - cb.lo[k]; a = k; }
            mid = (start + end) / 2;
            std::nth_element(idx.begin() + start, idx.begin() + mid, idx.begin() + end,
                             [&](int p, int q) { return cent(p, a) < cent(q, a); });
        }
        int l = build(start, mid);
        int r = build(mid, end);
        nodes[ni].left = l; nodes[ni].right = r;
        return ni;
    }
};

// Float value the device computes for a quantized plane: fmaf(q, 2^e, p).
inline float plane(int q, float scale, float p) { return std::fmaf((float)q, scale, p); }


struct Quant {
    float p;
    int e;   // unbiased exponent
};

// Choose p and e for one axis so that every child [lo, hi] quantizes into 0..255 with the
// device's float reconstruction enclosing it.
bool quantize_axis(double nlo, double nhi, const double* clo, const double* chi, int n,
                   float& p_out, int& e_out, uint8_t* qlo, uint8_t* qhi) {
    float p = round_down(nlo);
    double ext = nhi - (double)p;
    int e = -126;
    if (ext > 0) {
        e = (int)std::ceil(std::log2(ext / 255.0));
        if (e < -126) e = -126;
    }
    for (; e <= 127; ++e) {
        float s = std::ldexp(1.0f, e);
        bool ok = true;
        for (int i = 0; i < n && ok; ++i) {
            int ql = (int)std::floor((clo[i] - (double)p) / (double)s);
            if (ql < 0) ql = 0;
            if (ql > 255) ql = 255;
            while (ql > 0 && (double)plane(ql, s, p) > clo[i]) --ql;
            if ((double)plane(ql, s, p) > clo[i]) ok = false;
            int qh = (int)std::ceil((chi[i] - (double)p) / (double)s);
            if (qh < 0) qh = 0;
            while (qh <= 255 && (double)plane(qh, s, p) < chi[i]) ++qh;
            if (qh > 255) ok = false;
            if (ok) { qlo[i] = (uint8_t)ql; qhi[i] = (uint8_t)qh; }
        }
        if (ok) { p_out = p; e_out = e; return true; }
    }
    return false;
}

}  // namespace

bool build_wide_bvh(const std::vector<Box>& boxes_in, double margin, WideBvh& out,
                    std::string& err, BuildMethod method, int device) {
    out.nodes.clear();
    out.order.clear();
    const int n = (int)boxes_in.size();
    if (n == 0) return true;
    std::vector<Box> boxes(boxes_in);
    for (auto& b : boxes)
        for (int a = 0; a < 3; ++a) { b.lo[a] -= margin; b.hi[a] += margin; }
    if (method == BuildMethod::kDeviceLbvh) return build_wide_lbvh_device(boxes, kLeafSize, device, out, err);
    std::vector<BinNode> nodes;
    std::vector<int> idx;
    {
        Builder B(boxes);
        B.idx.resize(n);
        B.cx.resize(n); B.cy.resize(n); B.cz.resize(n);
        for (int i = 0; i < n; ++i) {
            B.idx[i] = i;
            B.cx[i] = 0.5 * (boxes[i].lo[0] + boxes[i].hi[0]);
            B.cy[i] = 0.5 * (boxes[i].lo[1] + boxes[i].hi[1]);
            B.cz[i] = 0.5 * (boxes[i].lo[2] + boxes[i].hi[2]);
        }
        B.nodes.reserve(2 * (size_t)n / FTB_LEAF_MAX + 16);
        B.build(0, n);
        nodes.swap(B.nodes);
        idx.swap(B.idx);
    }
    return collapse_to_wide(nodes, idx, out, err);
}

bool collapse_to_wide(const std::vector<BinNode>& bnodes, const std::vector<int>& bidx, WideBvh& out,
                      std::string& err) {
    struct {
        const std::vector<BinNode>& nodes;
        const std::vector<int>& idx;
    } B{bnodes, bidx};
    out.nodes.clear();
    out.order.clear();
    out.planes.clear();
    if (bnodes.empty()) return true;
    // Collapse.  A wide node is described by the binary node ids of its (<= 8) children.
    struct Pending { int bnode; int wide; };
    std::vector<Pending> queue;
    out.nodes.push_back(WNode{});
    queue.push_back({0, 0});
    size_t qi = 0;
    while (qi < queue.size()) {
        Pending pd = queue[qi++];
        std::vector<int> kids;
        const BNode& root = B.nodes[pd.bnode];
        if (root.count > 0) kids.push_back(pd.bnode);   // a leaf-only scene
        else { kids.push_back(root.left); kids.push_back(root.right); }
        while ((int)kids.size() < FTB_WIDTH) {
            int best = -1;
            double ba = -1.0;
            for (int k = 0; k < (int)kids.size(); ++k) {
                const BNode& c = B.nodes[kids[k]];
                if (c.count > 0) continue;
                double a = area(c.box);
                if (a > ba) { ba = a; best = k; }
            }
            if (best < 0) break;
            int id = kids[best];
            kids[best] = B.nodes[id].left;
            kids.push_back(B.nodes[id].right);
        }
        // assign: internal children get consecutive wide-node slots, leaves consecutive
        // record runs.
        WNode w;
        std::memset(&w, 0, sizeof w);
        w.child_base = (uint32_t)out.nodes.size();
        w.prim_base = (uint32_t)out.order.size();
        int n_int = 0, prim_off = 0;
        double clo[3][8], chi[3][8];
        Box nb;
        for (int k = 0; k < (int)kids.size(); ++k) {
            const BNode& c = B.nodes[kids[k]];
            nb.grow(c.box);
            for (int a = 0; a < 3; ++a) { clo[a][k] = c.box.lo[a]; chi[a][k] = c.box.hi[a]; }
            if (c.count > 0) {
                if (prim_off > 31) { err = "leaf record offset exceeds 5 bits"; return false; }
                w.meta[k] = (uint8_t)((c.count << 5) | prim_off);
                for (int i = 0; i < c.count; ++i) out.order.push_back(B.idx[c.first + i]);
                prim_off += c.count;
            } else {
                w.meta[k] = (uint8_t)((1 << 5) | n_int);
                w.imask |= (uint8_t)(1u << k);
                out.nodes.push_back(WNode{});
                queue.push_back({kids[k], (int)w.child_base + n_int});
                ++n_int;
            }
        }
        float p[3]; int e[3];
        uint8_t* qlo[3] = {w.qlo_x, w.qlo_y, w.qlo_z};
        uint8_t* qhi[3] = {w.qhi_x, w.qhi_y, w.qhi_z};
        for (int a = 0; a < 3; ++a)
            if (!quantize_axis(nb.lo[a], nb.hi[a], clo[a], chi[a], (int)kids.size(), p[a], e[a],
                               qlo[a], qhi[a])) {
                err = "BVH quantization failed (scene extent out of float range)";
                return false;
            }
        w.px = p[0]; w.py = p[1]; w.pz = p[2];
        w.ex = (uint8_t)(e[0] + 127); w.ey = (uint8_t)(e[1] + 127); w.ez = (uint8_t)(e[2] + 127);
        out.nodes[pd.wide] = w;
        out.planes.resize(out.nodes.size() * FTB_PLANES);
        put_planes(&out.planes[(size_t)pd.wide * FTB_PLANES], clo, chi, (int)kids.size());
    }
    return true;
}

std::vector<FNode> widen_nodes(const WideBvh& bvh) {
    const std::vector<WNode>& nodes = bvh.nodes;
    const bool tight = bvh.planes.size() == nodes.size() * FTB_PLANES;
    std::vector<FNode> out(nodes.size());
    for (size_t i = 0; i < nodes.size(); ++i) {
        const WNode& w = nodes[i];
        FNode& f = out[i];
        f.child_base = w.child_base;
        f.prim_base = w.prim_base;
        const float p[3] = {w.px, w.py, w.pz};
        const int eb[3] = {w.ex, w.ey, w.ez};
        float sc[3] = {0.0f, 0.0f, 0.0f};
        if (!tight)
            for (int a = 0; a < 3; ++a) sc[a] = std::ldexp(1.0f, eb[a] - 127);
        const uint8_t* qlo[3] = {w.qlo_x, w.qlo_y, w.qlo_z};
        const uint8_t* qhi[3] = {w.qhi_x, w.qhi_y, w.qhi_z};
        for (int k = 0; k < FTB_WIDTH; ++k) {
            const uint8_t m = w.meta[k];
            f.meta[k] = (m != 0 && ((w.imask >> k) & 1u)) ? (uint8_t)((FNODE_INNER << 5) | (m & 31u)) : m;
            for (int a = 0; a < 3; ++a) {
                const float s = sc[a];
                if (!m) {
                    f.lo[a][k] = INFINITY;
                    f.hi[a][k] = -INFINITY;
                } else if (tight) {
                    f.lo[a][k] = bvh.planes[i * FTB_PLANES + 8 * a + k];
                    f.hi[a][k] = bvh.planes[i * FTB_PLANES + 24 + 8 * a + k];
                } else {
                    f.lo[a][k] = plane(qlo[a][k], s, p[a]);
                    f.hi[a][k] = plane(qhi[a][k], s, p[a]);
                }
            }
        }
    }
    return out;
}

bool refit_wide_bvh(WideBvh& b, const std::vector<Box>& boxes, double margin, std::string& err) {
    const size_t nn = b.nodes.size();
    if (b.order.empty()) return true;
    std::vector<Box> nb(nn);
    b.planes.resize(nn * FTB_PLANES);
    // children always follow their parent, so a reverse sweep sees every child first
    for (size_t i = nn; i-- > 0;) {
        WNode& w = b.nodes[i];
        double clo[3][8], chi[3][8];
        int n = 0;
        Box all;
        for (int k = 0; k < FTB_WIDTH; ++k) {
            uint32_t m = w.meta[k];
            if (!m) break;   // the builder fills slots 0..n-1
            Box c;
            if ((w.imask >> k) & 1) {
                c = nb[w.child_base + (m & 31)];
            } else {
                for (uint32_t r = 0; r < (m >> 5); ++r) {
                    Box p = boxes[(size_t)b.order[w.prim_base + (m & 31) + r]];
                    for (int a = 0; a < 3; ++a) { p.lo[a] -= margin; p.hi[a] += margin; }
                    c.grow(p);
                }
            }
            for (int a = 0; a < 3; ++a) { clo[a][k] = c.lo[a]; chi[a][k] = c.hi[a]; }
            all.grow(c);
            ++n;
        }
        nb[i] = all;
        float p[3]; int e[3];
        uint8_t* qlo[3] = {w.qlo_x, w.qlo_y, w.qlo_z};
        uint8_t* qhi[3] = {w.qhi_x, w.qhi_y, w.qhi_z};
        for (int a = 0; a < 3; ++a)
            if (!quantize_axis(all.lo[a], all.hi[a], clo[a], chi[a], n, p[a], e[a], qlo[a], qhi[a])) {
                err = "BVH quantization failed (scene extent out of float range)";
                return false;
            }
        w.px = p[0]; w.py = p[1]; w.pz = p[2];
        w.ex = (uint8_t)(e[0] + 127); w.ey = (uint8_t)(e[1] + 127); w.ez = (uint8_t)(e[2] + 127);
        put_planes(&b.planes[i * FTB_PLANES], clo, chi, n);
    }
    return true;
}

bool validate_wide_bvh(const WideBvh& b, int n_prims, std::string& err) {
    const size_t nn = b.nodes.size(), nr = b.order.size();
    if (nn == 0) { err = "BVH has no root"; return false; }
    if ((int)nr != n_prims) { err = "BVH record count differs from primitive count"; return false; }
    std::vector<char> seen_rec(nr, 0), seen_node(nn, 0);
    seen_node[0] = 1;
    for (size_t i = 0; i < nn; ++i) {
        const WNode& w = b.nodes[i];
        for (int k = 0; k < FTB_WIDTH; ++k) {
            uint32_t m = w.meta[k];
            if (!m) { if ((w.imask >> k) & 1) { err = "internal bit on an empty slot"; return false; } continue; }
            uint32_t cnt = m >> 5, off = m & 31;
            if ((w.imask >> k) & 1) {
                uint64_t c = (uint64_t)w.child_base + off;
                if (cnt != 1 || c >= nn || c <= i || seen_node[c]) { err = "bad child node index"; return false; }
                seen_node[c] = 1;
            } else {
                if (cnt < 1 || cnt > FTB_LEAF_MAX) { err = "bad leaf size"; return false; }
                for (uint32_t r = 0; r < cnt; ++r) {
                    uint64_t ri = (uint64_t)w.prim_base + off + r;
                    if (ri >= nr || seen_rec[ri]) { err = "bad record index"; return false; }
                    seen_rec[ri] = 1;
                }
            }
        }
    }
    for (size_t i = 0; i < nn; ++i) if (!seen_node[i]) { err = "unreachable node"; return false; }
    for (size_t r = 0; r < nr; ++r) if (!seen_rec[r]) { err = "unreferenced record"; return false; }
    std::vector<char> seen_prim((size_t)n_prims, 0);
    for (int p : b.order) {
        if (p < 0 || p >= n_prims || seen_prim[(size_t)p]) { err = "bad primitive permutation"; return false; }
        seen_prim[(size_t)p] = 1;
    }
    return true;
}

}  // namespace ftb
