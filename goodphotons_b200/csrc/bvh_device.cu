// bvh_device.cu -- binary BVH built on the GPU (the fast bake; bvh_build.h).
//
// The reference builds its BVH on the host at scene load (binned SAH, bvh.h:89-176) and the
// GPU path re-uploads it per render call (render_cuda.cu:12692-13546).  This is a linear BVH
// instead: each primitive box's centre gets a 63-bit Morton code (21 bits per axis over the
// centre bounds), the codes are radix-sorted, the radix tree over the sorted codes is built
// one internal node per thread (Karras 2012, "Maximizing parallelism in the construction of
// BVHs, octrees, and k-d trees": ranges from the common-prefix lengths of neighbouring codes,
// split at the highest differing bit, equal codes ordered by index), and boxes are merged
// bottom-up (one thread per leaf; the second thread to reach a node merges its children).
// Subtrees of at most leaf_size primitives become leaves.  The binary tree is then collapsed
// into 8-wide nodes on the device too, one level of wide nodes per launch and one thread per
// wide node, with the same rules as the host collapse (open the child of largest surface
// area; leaf children as per-node runs of records) and the same conservative 8-bit
// quantization, checked against the device's own fmaf.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <string>
#include <vector>

#include "bvh_build.h"

namespace ftb {
namespace {

struct DBox { double lo[3], hi[3]; };

struct DBin {   // BinNode as the kernels write it
    double lo[3], hi[3];
    int left, right, first, count;
};

__device__ __forceinline__ uint64_t spread21(uint64_t v) {   // bit k -> bit 3k
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__global__ void k_morton(const DBox* __restrict__ boxes, int n, double3 lo, double3 inv_ext,
                         uint64_t* __restrict__ keys, int* __restrict__ ids) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DBox b = boxes[i];
    const double c[3] = {0.5 * (b.lo[0] + b.hi[0]), 0.5 * (b.lo[1] + b.hi[1]), 0.5 * (b.lo[2] + b.hi[2])};
    const double l[3] = {lo.x, lo.y, lo.z}, s[3] = {inv_ext.x, inv_ext.y, inv_ext.z};
    uint64_t q[3];
    for (int a = 0; a < 3; ++a) {
        double t = (c[a] - l[a]) * s[a] * 2097152.0;
        t = t < 0.0 ? 0.0 : (t > 2097151.0 ? 2097151.0 : t);
        q[a] = (uint64_t)t;
    }
    keys[i] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
    ids[i] = i;
}

// Length of the common prefix of sorted keys i and j (equal keys: 64 + prefix of the
// indices); -1 outside [0, n).
__device__ __forceinline__ int delta(const uint64_t* __restrict__ k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint64_t a = k[i], b = k[j];
    if (a == b) return 64 + __clz((uint32_t)(i ^ j));
    return __clzll((long long)(a ^ b));
}

// Internal node i of n - 1 (Karras 2012, section 4): range, split, children.  Internal nodes
// are 0 .. n-2, leaf k is node n-1+k; parent[] covers both.
__global__ void k_radix_tree(const uint64_t* __restrict__ k, int n, int* __restrict__ left,
                             int* __restrict__ right, int* __restrict__ parent, int* __restrict__ first,
                             int* __restrict__ count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (delta(k, n, i, i + 1) - delta(k, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(k, n, i, i - d);
    int lmax = 2;
    while (delta(k, n, i, i + lmax * d) > dmin) lmax *= 2;   // ends: delta is -1 past the ends
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta(k, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = delta(k, n, i, j);
    int s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (delta(k, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int g = i + s * d + (d < 0 ? -1 : 0);
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    const int lc = (lo == g) ? (n - 1 + g) : g;
    const int rc = (hi == g + 1) ? (n - 1 + g + 1) : (g + 1);
    left[i] = lc;
    right[i] = rc;
    parent[lc] = i;
    parent[rc] = i;
    first[i] = lo;
    count[i] = hi - lo + 1;
}

// Leaf boxes, then merges up the tree: the second thread to reach a node merges its children.
__global__ void k_boxes_up(const DBox* __restrict__ boxes, const int* __restrict__ ids, int n,
                           const int* __restrict__ left, const int* __restrict__ right,
                           const int* __restrict__ parent, int* __restrict__ visits, DBox* __restrict__ nb) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int node = n - 1 + k;
    nb[node] = boxes[ids[k]];
    __threadfence();
    int p = parent[node];
    while (p >= 0) {
        if (atomicAdd(&visits[p], 1) == 0) return;   // the sibling's thread merges
        __threadfence();
        // the children were written by other threads, possibly on other SMs: read past L1
        const double* a = nb[left[p]].lo;
        const double* b = nb[right[p]].lo;
        DBox m;
        for (int c = 0; c < 3; ++c) {
            const double al = __ldcg(a + c), bl = __ldcg(b + c), ah = __ldcg(a + 3 + c), bh = __ldcg(b + 3 + c);
            m.lo[c] = al < bl ? al : bl;
            m.hi[c] = ah > bh ? ah : bh;
        }
        nb[p] = m;
        __threadfence();
        p = parent[p];
    }
}

// BinNode form: an internal node over at most leaf_size primitives becomes a leaf.
__global__ void k_emit_bins(const DBox* __restrict__ nb, int n, const int* __restrict__ left,
                            const int* __restrict__ right, const int* __restrict__ first,
                            const int* __restrict__ count, int leaf_size, DBin* __restrict__ out) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= 2 * n - 1) return;
    DBin o;
    for (int c = 0; c < 3; ++c) { o.lo[c] = nb[v].lo[c]; o.hi[c] = nb[v].hi[c]; }
    if (v >= n - 1) {
        o.left = o.right = -1; o.first = v - (n - 1); o.count = 1;
    } else if (count[v] <= leaf_size) {
        o.left = o.right = -1; o.first = first[v]; o.count = count[v];
    } else {
        o.left = left[v]; o.right = right[v]; o.first = 0; o.count = 0;
    }
    out[v] = o;
}

__device__ __forceinline__ double area_of(const DBin& b) {
    const double dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
    if (dx < 0 || dy < 0 || dz < 0) return 0.0;
    return 2.0 * (dx * dy + dy * dz + dz * dx);
}

// Conservative quantization of one axis (the device form of bvh_build.cpp's quantize_axis):
// grid origin p = nlo rounded down to float, step 2^e; each child [lo, hi] gets bytes whose
// planes fmaf(q, 2^e, p) enclose it, e growing until every child fits in 0..255.
__device__ bool quantize_axis_dev(double nlo, double nhi, const double* clo, const double* chi, int n,
                                  float& p_out, int& e_out, uint8_t* qlo, uint8_t* qhi) {
    const float p = __double2float_rd(nlo);
    const double ext = nhi - (double)p;
    int e = -126;
    if (ext > 0) {
        e = (int)ceil(log2(ext / 255.0));
        if (e < -126) e = -126;
    }
    for (; e <= 127; ++e) {
        const float sc = __int_as_float((e + 127) << 23);
        bool ok = true;
        for (int i = 0; i < n && ok; ++i) {
            double fl = floor((clo[i] - (double)p) / (double)sc);
            int ql = fl < 0.0 ? 0 : (fl > 255.0 ? 255 : (int)fl);
            while (ql > 0 && (double)fmaf((float)ql, sc, p) > clo[i]) --ql;
            if ((double)fmaf((float)ql, sc, p) > clo[i]) ok = false;
            double ce = ceil((chi[i] - (double)p) / (double)sc);
            int qh = ce < 0.0 ? 0 : (ce > 256.0 ? 256 : (int)ce);
            while (qh <= 255 && (double)fmaf((float)qh, sc, p) < chi[i]) ++qh;
            if (qh > 255) ok = false;
            if (ok) { qlo[i] = (uint8_t)ql; qhi[i] = (uint8_t)qh; }
        }
        if (ok) { p_out = p; e_out = e; return true; }
    }
    return false;
}

// One level of the collapse: wide node w (in [begin, end)) is rooted at binary node src[w].
// counters[0] = wide nodes allocated, counters[1] = records allocated, counters[2] = errors.
__global__ void k_collapse_level(const DBin* __restrict__ bins, const int* __restrict__ idx, int begin, int end,
                                 int* __restrict__ src, WNode* __restrict__ nodes, float* __restrict__ planes,
                                 int* __restrict__ order, int* __restrict__ counters) {
    const int w = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= end) return;
    const int root = src[w];
    int kids[FTB_WIDTH];
    int nk = 0;
    if (bins[root].count > 0) kids[nk++] = root;   // a leaf-only scene
    else { kids[nk++] = bins[root].left; kids[nk++] = bins[root].right; }
    while (nk < FTB_WIDTH) {
        int best = -1;
        double ba = -1.0;
        for (int k = 0; k < nk; ++k) {
            const DBin& c = bins[kids[k]];
            if (c.count > 0) continue;
            const double a = area_of(c);
            if (a > ba) { ba = a; best = k; }
        }
        if (best < 0) break;
        const int id = kids[best];
        kids[best] = bins[id].left;
        kids[nk++] = bins[id].right;
    }
    int n_int = 0, n_rec = 0;
    for (int k = 0; k < nk; ++k) {
        if (bins[kids[k]].count > 0) n_rec += bins[kids[k]].count;
        else ++n_int;
    }
    const int child_base = n_int ? atomicAdd(&counters[0], n_int) : 0;
    const int prim_base = atomicAdd(&counters[1], n_rec);
    WNode o;
    memset(&o, 0, sizeof o);
    o.child_base = (uint32_t)child_base;
    o.prim_base = (uint32_t)prim_base;
    double clo[3][FTB_WIDTH], chi[3][FTB_WIDTH], nlo[3] = {1e300, 1e300, 1e300}, nhi[3] = {-1e300, -1e300, -1e300};
    int ii = 0, off = 0;
    for (int k = 0; k < nk; ++k) {
        const DBin& c = bins[kids[k]];
        for (int a = 0; a < 3; ++a) {
            clo[a][k] = c.lo[a]; chi[a][k] = c.hi[a];
            nlo[a] = c.lo[a] < nlo[a] ? c.lo[a] : nlo[a];
            nhi[a] = c.hi[a] > nhi[a] ? c.hi[a] : nhi[a];
        }
        if (c.count > 0) {
            o.meta[k] = (uint8_t)((c.count << 5) | off);
            for (int r = 0; r < c.count; ++r) order[prim_base + off + r] = idx[c.first + r];
            off += c.count;
        } else {
            o.meta[k] = (uint8_t)((1 << 5) | ii);
            o.imask |= (uint8_t)(1u << k);
            src[child_base + ii] = kids[k];
            ++ii;
        }
    }
    float p[3];
    int e[3];
    uint8_t* qlo[3] = {o.qlo_x, o.qlo_y, o.qlo_z};
    uint8_t* qhi[3] = {o.qhi_x, o.qhi_y, o.qhi_z};
    for (int a = 0; a < 3; ++a)
        if (!quantize_axis_dev(nlo[a], nhi[a], clo[a], chi[a], nk, p[a], e[a], qlo[a], qhi[a])) {
            atomicAdd(&counters[2], 1);
            p[a] = 0.f; e[a] = 0;
        }
    o.px = p[0]; o.py = p[1]; o.pz = p[2];
    o.ex = (uint8_t)(e[0] + 127); o.ey = (uint8_t)(e[1] + 127); o.ez = (uint8_t)(e[2] + 127);
    nodes[w] = o;
    // the child boxes rounded outward to float (empty slots: +inf / -inf)
    float* pl = planes + (size_t)w * FTB_PLANES;
    for (int a = 0; a < 3; ++a)
        for (int k = 0; k < FTB_WIDTH; ++k) {
            pl[8 * a + k] = k < nk ? __double2float_rd(clo[a][k]) : __int_as_float(0x7f800000);
            pl[24 + 8 * a + k] = k < nk ? __double2float_ru(chi[a][k]) : __int_as_float(0xff800000);
        }
}

struct DevBuf {
    std::vector<void*> ptrs;
    ~DevBuf() { for (void* p : ptrs) cudaFree(p); }
    template <class T>
    cudaError_t get(T** out, size_t n) {
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, n * sizeof(T) + 16);
        if (e == cudaSuccess) { ptrs.push_back(p); *out = (T*)p; }
        return e;
    }
};

}  // namespace

bool build_wide_lbvh_device(const std::vector<Box>& boxes, int leaf_size, int device, WideBvh& out,
                            std::string& err) {
    static_assert(sizeof(DBox) == 6 * sizeof(double), "DBox layout");
    const int n = (int)boxes.size();
    out.nodes.clear();
    out.order.clear();
    if (n == 0) return true;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaError_t e = cudaSuccess;
    auto fail = [&](const char* what) {
        err = std::string("device BVH build: ") + what + (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : "");
        cudaGetLastError();
        cudaSetDevice(prev);
        return false;
    };
    // centre bounds on the host (one pass over the boxes)
    double clo[3] = {1e300, 1e300, 1e300}, chi[3] = {-1e300, -1e300, -1e300};
    std::vector<DBox> hb((size_t)n);
    for (int i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) {
            hb[i].lo[a] = boxes[i].lo[a];
            hb[i].hi[a] = boxes[i].hi[a];
            double c = 0.5 * (boxes[i].lo[a] + boxes[i].hi[a]);
            clo[a] = c < clo[a] ? c : clo[a];
            chi[a] = c > chi[a] ? c : chi[a];
        }
    }
    double inv[3];
    for (int a = 0; a < 3; ++a) inv[a] = chi[a] > clo[a] ? 1.0 / (chi[a] - clo[a]) : 0.0;
    {
        DevBuf buf;
        DBox *d_boxes, *d_nb;
        uint64_t *d_k, *d_ks;
        int *d_id, *d_ids, *d_left, *d_right, *d_parent, *d_first, *d_count, *d_visit, *d_src, *d_order, *d_ctr;
        DBin* d_bins;
        WNode* d_nodes;
        float* d_planes = nullptr;
        const size_t nn = (size_t)n;
        if ((e = buf.get(&d_boxes, nn)) || (e = buf.get(&d_nb, 2 * nn)) || (e = buf.get(&d_k, nn)) ||
            (e = buf.get(&d_ks, nn)) || (e = buf.get(&d_id, nn)) || (e = buf.get(&d_ids, nn)) ||
            (e = buf.get(&d_left, nn)) || (e = buf.get(&d_right, nn)) || (e = buf.get(&d_parent, 2 * nn)) ||
            (e = buf.get(&d_first, nn)) || (e = buf.get(&d_count, nn)) || (e = buf.get(&d_visit, nn)) ||
            (e = buf.get(&d_bins, 2 * nn)) || (e = buf.get(&d_src, nn + 1)) || (e = buf.get(&d_order, nn)) ||
            (e = buf.get(&d_nodes, nn + 1)) || (e = buf.get(&d_ctr, 4)))
            return fail("allocation");
        if ((e = cudaMemcpy(d_boxes, hb.data(), sizeof(DBox) * nn, cudaMemcpyHostToDevice))) return fail("upload");
        const int T = 256, G = (n + T - 1) / T, G2 = (2 * n - 1 + T - 1) / T;
        if (n == 1) {   // one leaf: the root of the collapse is leaf 0
            DBin leaf;
            for (int a = 0; a < 3; ++a) { leaf.lo[a] = hb[0].lo[a]; leaf.hi[a] = hb[0].hi[a]; }
            leaf.left = leaf.right = -1; leaf.first = 0; leaf.count = 1;
            const int zero = 0;
            if ((e = cudaMemcpy(d_bins, &leaf, sizeof leaf, cudaMemcpyHostToDevice)) ||
                (e = cudaMemcpy(d_ids, &zero, sizeof zero, cudaMemcpyHostToDevice)))
                return fail("upload");
        } else {
            k_morton<<<G, T>>>(d_boxes, n, make_double3(clo[0], clo[1], clo[2]), make_double3(inv[0], inv[1], inv[2]),
                               d_k, d_id);
            if ((e = cudaGetLastError())) return fail("morton codes");
            size_t tmp_bytes = 0;
            if ((e = cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_k, d_ks, d_id, d_ids, n, 0, 63)))
                return fail("sort sizing");
            char* d_tmp = nullptr;
            if ((e = buf.get(&d_tmp, tmp_bytes))) return fail("sort scratch");
            if ((e = cub::DeviceRadixSort::SortPairs(d_tmp, tmp_bytes, d_k, d_ks, d_id, d_ids, n, 0, 63)))
                return fail("sort");
            if ((e = cudaMemset(d_parent, 0xff, sizeof(int) * 2 * nn))) return fail("memset");
            if ((e = cudaMemset(d_visit, 0, sizeof(int) * nn))) return fail("memset");
            k_radix_tree<<<G, T>>>(d_ks, n, d_left, d_right, d_parent, d_first, d_count);
            if ((e = cudaGetLastError())) return fail("radix tree");
            k_boxes_up<<<G, T>>>(d_boxes, d_ids, n, d_left, d_right, d_parent, d_visit, d_nb);
            if ((e = cudaGetLastError())) return fail("boxes");
            k_emit_bins<<<G2, T>>>(d_nb, n, d_left, d_right, d_first, d_count, leaf_size, d_bins);
            if ((e = cudaGetLastError())) return fail("nodes");
        }
        // collapse, one level of wide nodes per launch
        const int ctr0[4] = {1, 0, 0, 0}, zero = 0;
        if ((e = cudaMemcpy(d_ctr, ctr0, sizeof ctr0, cudaMemcpyHostToDevice)) ||
            (e = cudaMemcpy(d_src, &zero, sizeof zero, cudaMemcpyHostToDevice)))
            return fail("upload");
        int begin = 0, end = 1, ctr[4] = {0, 0, 0, 0};
        // the planes of the wide nodes grow with the levels (a tree has far fewer wide nodes
        // than primitives; nn + 1 bounds them)
        size_t cap = std::min(nn + 1, nn / 4 + 64);
        if ((e = cudaMalloc(&d_planes, cap * FTB_PLANES * sizeof(float)))) return fail("allocation");
        struct PlaneBuf { float*& p; ~PlaneBuf() { if (p) cudaFree(p); } } planes_guard{d_planes};
        while (begin < end) {
            if ((size_t)end > cap) {
                const size_t nc = std::min(nn + 1, std::max((size_t)end, 2 * cap));
                float* np = nullptr;
                if ((e = cudaMalloc(&np, nc * FTB_PLANES * sizeof(float)))) return fail("allocation");
                if ((e = cudaMemcpy(np, d_planes, (size_t)begin * FTB_PLANES * sizeof(float), cudaMemcpyDeviceToDevice))) {
                    cudaFree(np);
                    return fail("planes");
                }
                cudaFree(d_planes);
                d_planes = np;
                cap = nc;
            }
            k_collapse_level<<<(end - begin + 127) / 128, 128>>>(d_bins, d_ids, begin, end, d_src, d_nodes, d_planes,
                                                                d_order, d_ctr);
            if ((e = cudaGetLastError())) return fail("collapse");
            if ((e = cudaMemcpy(ctr, d_ctr, sizeof ctr, cudaMemcpyDeviceToHost))) return fail("collapse");
            if (ctr[0] > n + 1 || ctr[1] > n) { e = cudaSuccess; return fail("collapse overran its arrays"); }
            begin = end;
            end = ctr[0];
        }
        if (ctr[2] != 0) { e = cudaSuccess; return fail("quantization failed (scene extent out of float range)"); }
        if (ctr[1] != n) { e = cudaSuccess; return fail("collapse lost records"); }
        out.nodes.resize((size_t)ctr[0]);
        out.order.resize(nn);
        out.planes.resize((size_t)ctr[0] * FTB_PLANES);
        if ((e = cudaMemcpy(out.nodes.data(), d_nodes, sizeof(WNode) * out.nodes.size(), cudaMemcpyDeviceToHost)) ||
            (e = cudaMemcpy(out.planes.data(), d_planes, sizeof(float) * out.planes.size(), cudaMemcpyDeviceToHost)) ||
            (e = cudaMemcpy(out.order.data(), d_order, sizeof(int) * nn, cudaMemcpyDeviceToHost)))
            return fail("download");
    }
    cudaSetDevice(prev);
    return true;
}

}  // namespace ftb
