// ftb_kernels.cu -- sm_100a wavefront kernels of the forward pinhole light tracer.
//
// Up to W photon paths are in flight at once, traced with four kernels:
//   k_emit    seed the per-photon PCG32 stream, pick emitter / point / direction /
//             wavelength, book `emitted`, queue the emitter's direct camera connection
//             (reference: Renderer::tracePhoton emission, render.h:1827-1984)
//   k_extend  closest hit of every queued path over the 8-wide BVH (Scene::closestHit,
//             scene.h:2194-2242)
//   k_shade   media, interior absorption and the material interaction of one bounce;
//             queues camera connections and copies the surviving paths into the other
//             path buffer (render.h:2013-2238)
//   k_shadow  any-hit test of the queued connections (Scene::occluded, scene.h:2249) and
//             the splat into the 64-bit fixed-point film (Film::add, scene_film.h:12)
//
// Path state is compacted (a queue of n paths is entries 0..n-1 of structure-of-arrays
// buffers, no index lists) and two-ended (paths inside a dielectric grow from the top
// entry down, so each end holds paths of similar traversal cost).  The queue kernels hand
// out work to warps 32 entries at a time from a per-launch counter.  A streaming pass
// (launch_stream) refills the room freed by finished paths with the next photons every
// half-iteration and runs as one CUDA graph with a device-driven while loop; a wave
// (launch_wave) traces W photons to their last bounce.
//
// Variants: k_emit_hero / k_shade_hero / k_shadow_hero trace hero-wavelength bundles (one
// path carries up to kHeroMax wavelengths), and the kernels are templated on whether the
// scenes have instances, participating media or spheres/curves, so a launch runs only the
// code its scenes need.  k_sort_queue optionally orders a closest-hit queue by direction.
//
// Numerics.  Everything that decides a path -- triangle/sphere/curve tests, hit points,
// normals, BSDF sampling, Russian roulette, the camera projection -- is computed in fp64
// in the reference's operation order, and this file is compiled with -fmad=false so no
// product is fused.  Only the BVH culling runs in fp32, against boxes that were rounded
// outward (see bvh_build.cpp) and with the ray interval widened by 2^-21, so it never
// drops a primitive the fp64 test would accept.  Paths therefore follow the reference CPU
// tracer photon for photon; the remaining differences are last-bit ones from CUDA's
// exp/log/sin/cos/pow, and exact ties in t.
#include <cooperative_groups.h>
#include <algorithm>
#include <vector>
#include <cuda_runtime.h>
#include <float.h>
#include <limits.h>
#include <stdint.h>

#include "ftb_kernels.h"

namespace cg = cooperative_groups;

// Resident blocks per SM each kernel is compiled for (register budget 65536 / (128 x minB)),
// chosen by measurement on B200: latency hiding beats the spills the smaller budget costs.
#ifndef FTB_EMIT_MINB
#define FTB_EMIT_MINB 8
#endif
#ifndef FTB_TRAV_MINB
#define FTB_TRAV_MINB 8
#endif
#ifndef FTB_SHADE_MINB
#define FTB_SHADE_MINB 8
#endif
#ifndef FTB_SHADE_MEDIA_MINB   // shading with participating media: more registers pay off
#define FTB_SHADE_MEDIA_MINB 4
#endif

namespace ftb {

#define PI_D 3.141592653589793
#define LAMBDA_MIN 360.0
#define LAMBDA_MAX 830.0
#define EPS_RAY 1e-6

// ------------------------------------------------------------------ vectors (fp64) -----
struct D3 { double x, y, z; };
__device__ __forceinline__ D3 mk(double x, double y, double z) { D3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ D3 operator*(D3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ D3 operator/(D3 a, double s) { return mk(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ D3 neg(D3 a) { return mk(-a.x, -a.y, -a.z); }
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross(D3 a, D3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double len(D3 a) { return sqrt(dot(a, a)); }
__device__ __forceinline__ D3 normalize(D3 a) { return a / len(a); }
__device__ __forceinline__ double comp(D3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
__device__ __forceinline__ D3 ld3(const double* p) { return mk(p[0], p[1], p[2]); }
// reflect (linalg.h:82)
__device__ __forceinline__ D3 reflect(D3 d, D3 n) { return d - n * (2.0 * dot(d, n)); }
// onb (linalg.h:85-91)
__device__ __forceinline__ void onb(D3 n, D3& t, D3& b) {
    double sign = copysign(1.0, n.z);
    double a = -1.0 / (sign + n.z);
    double d = n.x * n.y * a;
    t = mk(1.0 + sign * n.x * n.x * a, sign * d, -sign * n.x);
    b = mk(d, sign + n.y * n.y * a, -n.y);
}

// ------------------------------------------------------------------ RNG (rng.h) --------
struct Pcg { uint64_t s, inc; };
__device__ __forceinline__ uint32_t pcg_next(Pcg& r) {
    uint64_t old = r.s;
    r.s = old * 6364136223846793005ULL + r.inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((~rot + 1u) & 31));
}
__device__ __forceinline__ double uniform(Pcg& r) { return (pcg_next(r) >> 8) * (1.0 / 16777216.0); }
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
// seedUnit (rng.h:40) with the forward-tracer salt (main.cpp:11326)
__device__ __forceinline__ Pcg seed_photon(uint64_t k) {
    const uint64_t salt = 0x9E3779B97F4A7C15ULL;
    Pcg r;
    r.s = 0; r.inc = (mix64(k ^ salt) << 1u) | 1u;
    pcg_next(r);
    r.s += mix64(k + salt);
    pcg_next(r);
    return r;
}

// cosineHemisphere (rng.h:45-52)
__device__ D3 cosine_hemisphere(D3 n, Pcg& rng) {
    double u1 = uniform(rng), u2 = uniform(rng);
    double r = sqrt(u1);
    double phi = 6.283185307179586 * u2;
    double lx = r * cos(phi), ly = r * sin(phi), lz = sqrt(1.0 - u1);
    D3 t, b; onb(n, t, b);
    return normalize(t * lx + b * ly + n * lz);
}
// glossyDirUV / sampleGlossy (render.h:46-64)
__device__ D3 sample_glossy(D3 mdir, double roughness, Pcg& rng) {
    double u1 = uniform(rng), u2 = uniform(rng);
    if (u1 >= 1.0) return mdir;
    double rr = roughness < 1e-3 ? 1e-3 : roughness;
    double e = 2.0 / (rr * rr) - 2.0; if (e < 0) e = 0;
    double cos_t = pow(u1, 1.0 / (e + 1.0));
    double s = 1.0 - cos_t * cos_t;
    double sin_t = sqrt(s > 0.0 ? s : 0.0);
    double phi = 2.0 * PI_D * u2;
    D3 t, b; onb(mdir, t, b);
    return normalize(t * (sin_t * cos(phi)) + b * (sin_t * sin(phi)) + mdir * cos_t);
}
// hgPhase / sampleHG (phase.h:18-40)
__device__ __forceinline__ double hg_phase(double cos_t, double g) {
    double d = 1.0 + g * g - 2.0 * g * cos_t;
    if (d < 1e-9) d = 1e-9;
    return (1.0 - g * g) / (4.0 * PI_D * d * sqrt(d));
}
__device__ D3 sample_hg(D3 wi, double g, Pcg& rng) {
    double u1 = uniform(rng), u2 = uniform(rng);
    double cos_t;
    if (fabs(g) < 1e-3) cos_t = 1.0 - 2.0 * u1;
    else {
        double sq = (1.0 - g * g) / (1.0 + g - 2.0 * g * u1);
        cos_t = (1.0 + g * g - sq * sq) / (2.0 * g);
    }
    double s = 1.0 - cos_t * cos_t;
    double sin_t = sqrt(s > 0.0 ? s : 0.0);
    double phi = 2.0 * PI_D * u2;
    D3 t, b; onb(wi, t, b);
    return normalize(t * (sin_t * cos(phi)) + b * (sin_t * sin(phi)) + wi * cos_t);
}

// ------------------------------------------------------------------ spectra ------------
__device__ double spec_eval(const DevScene& sc, int idx, double w) {
    const DevSpec& s = sc.spec[idx];
    switch (s.kind) {
    case FTB_SPEC_CONST: return s.p[0];
    case FTB_SPEC_TABLE: {   // tabulatedSpectrum (spectrum.h:264-281)
        const double* x = sc.tw + s.offset;
        const double* y = sc.tv + s.offset;
        int n = s.n;
        if (w <= x[0]) return y[0];
        if (w >= x[n - 1]) return y[n - 1];
        int lo = 0, hi = n - 1;
        while (lo + 1 < hi) { int mid = (lo + hi) / 2; if (x[mid] <= w) lo = mid; else hi = mid; }
        double w0 = x[lo], w1 = x[lo + 1], v0 = y[lo], v1 = y[lo + 1];
        double f = (w1 > w0) ? (w - w0) / (w1 - w0) : 0.0;
        return v0 + (v1 - v0) * f;
    }
    case FTB_SPEC_CAUCHY: { double um = w * 1e-3; return s.p[0] + s.p[1] / (um * um); }
    case FTB_SPEC_SELLMEIER: {
        double l2 = (w * 1e-3) * (w * 1e-3);
        double n2 = 1.0 + s.p[0] * l2 / (l2 - s.p[3]) + s.p[1] * l2 / (l2 - s.p[4]) +
                    s.p[2] * l2 / (l2 - s.p[5]);
        return sqrt(n2 > 1.0 ? n2 : 1.0);
    }
    default: return 0.0;
    }
}
__device__ __forceinline__ double spec_slot(const DevScene& sc, int s, double w, double dflt) {
    return s >= 0 ? spec_eval(sc, s, w) : dflt;
}
__device__ __forceinline__ double clamp01(double x) { return x < 0 ? 0 : (x > 1 ? 1 : x); }

// CIE 1931 multi-Gaussian fit (color.h:8-24)
__device__ __forceinline__ double gauss_piece(double x, double mu, double s1, double s2) {
    double t = (x - mu) * ((x < mu) ? s1 : s2);
    return exp(-0.5 * t * t);
}
__device__ __forceinline__ double cie_x(double w) {
    return 0.362 * gauss_piece(w, 442.0, 0.0624, 0.0374) + 1.056 * gauss_piece(w, 599.8, 0.0264, 0.0323) -
           0.065 * gauss_piece(w, 501.1, 0.0490, 0.0382);
}
__device__ __forceinline__ double cie_y(double w) {
    return 0.821 * gauss_piece(w, 568.8, 0.0213, 0.0247) + 0.286 * gauss_piece(w, 530.9, 0.0613, 0.0322);
}
__device__ __forceinline__ double cie_z(double w) {
    return 1.217 * gauss_piece(w, 437.0, 0.0845, 0.0278) + 0.681 * gauss_piece(w, 459.0, 0.0385, 0.0725);
}

// ------------------------------------------------------------------ exact prim tests ---
struct Shear { int kx, ky, kz; double sx, sy, sz; };
// makeTriShear (geometry.h:261-276)
__device__ __forceinline__ Shear make_shear(D3 d) {
    Shear s;
    double ax = fabs(d.x), ay = fabs(d.y), az = fabs(d.z);
    if (ax >= ay && ax >= az) s.kz = 0; else if (ay >= az) s.kz = 1; else s.kz = 2;
    s.kx = s.kz + 1; if (s.kx == 3) s.kx = 0;
    s.ky = s.kx + 1; if (s.ky == 3) s.ky = 0;
    if (comp(d, s.kz) < 0.0) { int t = s.kx; s.kx = s.ky; s.ky = t; }
    s.sx = comp(d, s.kx) / comp(d, s.kz);
    s.sy = comp(d, s.ky) / comp(d, s.kz);
    s.sz = 1.0 / comp(d, s.kz);
    return s;
}
// The reference recomputes an exactly-zero edge function in long double (x87, 64-bit
// mantissa).  The device has no extended type: a*b - c*d is formed from exact products
// (two FMA residuals), which has the same sign whenever the extended-precision result is
// nonzero.  Reached only when a ray meets an edge line exactly.
__device__ __forceinline__ double zero_fallback(double a, double b, double c, double d) {
    double ph = a * b, qh = c * d;
    double pl = fma(a, b, -ph), ql = fma(c, d, -qh);
    return (ph - qh) + (pl - ql);
}
struct TriHitW { double u, v, w, inv_det; };
// intersectTri acceptance (geometry.h:280-324); returns t or -1 (rejected)
__device__ __forceinline__ bool tri_test(const Shear& sh, D3 ro, const double* v, double tmin,
                                         double tbest, double& t_out, TriHitW* bw) {
    D3 A = mk(v[0], v[1], v[2]) - ro, B = mk(v[3], v[4], v[5]) - ro, C = mk(v[6], v[7], v[8]) - ro;
    double Akz = comp(A, sh.kz), Bkz = comp(B, sh.kz), Ckz = comp(C, sh.kz);
    double Ax = comp(A, sh.kx) - sh.sx * Akz, Ay = comp(A, sh.ky) - sh.sy * Akz;
    double Bx = comp(B, sh.kx) - sh.sx * Bkz, By = comp(B, sh.ky) - sh.sy * Bkz;
    double Cx = comp(C, sh.kx) - sh.sx * Ckz, Cy = comp(C, sh.ky) - sh.sy * Ckz;
    double U = Cx * By - Cy * Bx;
    double V = Ax * Cy - Ay * Cx;
    double W = Bx * Ay - By * Ax;
    if (U == 0.0 || V == 0.0 || W == 0.0) {
        if (U == 0.0) U = zero_fallback(Cx, By, Cy, Bx);
        if (V == 0.0) V = zero_fallback(Ax, Cy, Ay, Cx);
        if (W == 0.0) W = zero_fallback(Bx, Ay, By, Ax);
    }
    if ((U < 0.0 || V < 0.0 || W < 0.0) && (U > 0.0 || V > 0.0 || W > 0.0)) return false;
    double det = U + V + W;
    if (det == 0.0) return false;
    double T = U * (sh.sz * Akz) + V * (sh.sz * Bkz) + W * (sh.sz * Ckz);
    double inv_det = 1.0 / det;
    double t = T * inv_det;
    if (t < tmin || t >= tbest) return false;
    t_out = t;
    if (bw) { bw->u = U; bw->v = V; bw->w = W; bw->inv_det = inv_det; }
    return true;
}
// intersectSphere acceptance (geometry.h:377-387)
__device__ __forceinline__ bool sphere_test(D3 ro, D3 rd, const double* s, double tmin, double tbest,
                                            double& t_out) {
    D3 oc = ro - mk(s[0], s[1], s[2]);
    double r = s[3];
    double a = dot(rd, rd);
    double b = 2.0 * dot(oc, rd);
    double c = dot(oc, oc) - r * r;
    double disc = b * b - 4.0 * a * c;
    if (disc < 0.0) return false;
    double sq = sqrt(disc);
    double t = (-b - sq) / (2.0 * a);
    if (t < tmin) t = (-b + sq) / (2.0 * a);
    if (t < tmin || t >= tbest) return false;
    t_out = t;
    return true;
}
// makeCurveRay (curve.h:126-135)
struct CurveRay { D3 dn; double inv_len; };
__device__ __forceinline__ CurveRay make_curve_ray(D3 d) {
    CurveRay c; c.dn = mk(0, 0, 1); c.inv_len = 1.0;
    double l2 = dot(d, d);
    if (l2 > 0.0) { double l = sqrt(l2); c.inv_len = 1.0 / l; c.dn = d * c.inv_len; }
    return c;
}
struct CurveWin { double tn, y, shift; int piece; };
__device__ __forceinline__ void offer(CurveWin& a, double inv_len, double tmin, double tbest, double tn,
                                      int w, double y) {
    if (tn >= a.tn) return;
    double t = (tn + a.shift) * inv_len;
    if (t < tmin || t >= tbest) return;
    a.tn = tn; a.piece = w; a.y = y;
}
// curveSegCrossings<double> + intersectCurveSeg acceptance (curve.h:199-309)
__device__ bool curve_test(const CurveRay& cr, D3 ro, const double* s, double tmin, double tbest,
                           double& t_out, CurveWin* win) {
    D3 rd = cr.dn;
    D3 p0 = mk(s[0], s[1], s[2]), p1 = mk(s[3], s[4], s[5]);
    double r0 = s[6], r1 = s[7];
    CurveWin a; a.tn = DBL_MAX; a.y = 0.0; a.piece = -1;
    D3 ba = p1 - p0;
    double m0 = dot(ba, ba);
    if (!(m0 > 0.0)) return false;
    a.shift = dot(p0 - ro, rd);
    D3 o = mk(ro.x + rd.x * a.shift, ro.y + rd.y * a.shift, ro.z + rd.z * a.shift);
    D3 oa = o - p0, ob = o - p1;
    double rr = r0 - r1;
    double m1 = dot(ba, oa), m2 = dot(ba, rd), m3 = dot(rd, oa), m5 = dot(oa, oa);
    double m6 = dot(ob, rd), m7 = dot(ob, ob);
    double d2 = m0 - rr * rr;
    const double il = cr.inv_len;
    if (d2 > 0.0) {
        double k2 = d2 - m2 * m2;
        double k1 = d2 * m3 - m1 * m2 + m2 * rr * r0;
        double k0 = d2 * m5 - m1 * m1 + m1 * rr * r0 * 2.0 - m0 * r0 * r0;
        double h = k1 * k1 - k0 * k2;
        if (h >= 0.0 && k2 != 0.0) {
            double sq = sqrt(h);
            double ta = (-sq - k1) / k2, tb = (sq - k1) / k2;
            if (ta > tb) { double tmp = ta; ta = tb; tb = tmp; }
            double base = m1 - r0 * rr;
            double ya = base + ta * m2, yb = base + tb * m2;
            if (ya > 0.0 && ya < d2) offer(a, il, tmin, tbest, ta, 0, ya);
            if (yb > 0.0 && yb < d2) offer(a, il, tmin, tbest, tb, 0, yb);
        }
        double h1 = m3 * m3 - m5 + r0 * r0;
        if (h1 > 0.0) {
            double q = sqrt(h1), base = m1 - r0 * rr;
            double ta = -m3 - q, tb = -m3 + q;
            if (base + ta * m2 <= 0.0) offer(a, il, tmin, tbest, ta, 1, 0.0);
            if (base + tb * m2 <= 0.0) offer(a, il, tmin, tbest, tb, 1, 0.0);
        }
        double h2 = m6 * m6 - m7 + r1 * r1;
        if (h2 > 0.0) {
            double q = sqrt(h2), base = m1 - r0 * rr;
            double ta = -m6 - q, tb = -m6 + q;
            if (base + ta * m2 >= d2) offer(a, il, tmin, tbest, ta, 2, d2);
            if (base + tb * m2 >= d2) offer(a, il, tmin, tbest, tb, 2, d2);
        }
    } else {
        bool use_p0 = (r0 >= r1);
        double rc = use_p0 ? r0 : r1, mm = use_p0 ? m3 : m6, mq = use_p0 ? m5 : m7;
        double hh = mm * mm - mq + rc * rc;
        if (hh > 0.0) {
            double q = sqrt(hh);
            offer(a, il, tmin, tbest, -mm - q, use_p0 ? 1 : 2, use_p0 ? 0.0 : d2);
            offer(a, il, tmin, tbest, -mm + q, use_p0 ? 1 : 2, use_p0 ? 0.0 : d2);
        }
    }
    if (a.piece < 0) return false;
    t_out = (a.tn + a.shift) * il;
    if (win) *win = a;
    return true;
}

__device__ __forceinline__ int rec_type(const PrimRec& r) { return (r.info >> 24) & 3; }
__device__ __forceinline__ int rec_mat(const PrimRec& r) { return r.info & 0xffffff; }
__device__ __forceinline__ bool rec_smooth(const PrimRec& r) { return (r.info >> 30) & 1; }

__device__ __forceinline__ void load_rec(const PrimRec* recs, int i, PrimRec& r) {
    const double2* p = reinterpret_cast<const double2*>(recs + i);
    double2 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3), e = __ldg(p + 4);
    r.d[0] = a.x; r.d[1] = a.y; r.d[2] = b.x; r.d[3] = b.y; r.d[4] = c.x; r.d[5] = c.y;
    r.d[6] = d.x; r.d[7] = d.y; r.d[8] = e.x;
    long long tail = __double_as_longlong(e.y);
    r.prim = (int32_t)(tail & 0xffffffffLL);
    r.info = (int32_t)(tail >> 32);
}

struct RayCtx {
    D3 o, d;
    Shear sh;
    CurveRay cr;
};

// SHAPES: the scene has spheres or curves besides triangles; without them the record test
// is the triangle test alone (a smaller traversal kernel with fewer spills).
template <bool SHAPES>
__device__ __forceinline__ bool rec_test(const RayCtx& R, const PrimRec& r, double tmin, double tbest,
                                         double& t) {
    if (!SHAPES) return tri_test(R.sh, R.o, r.d, tmin, tbest, t, nullptr);
    int ty = rec_type(r);
    if (ty == REC_TRI) return tri_test(R.sh, R.o, r.d, tmin, tbest, t, nullptr);
    if (ty == REC_SPHERE) return sphere_test(R.o, R.d, r.d, tmin, tbest, t);
    return curve_test(R.cr, R.o, r.d, tmin, tbest, t, nullptr);
}

// Hit attributes of the winning record (geometry.h:325-368, :388-396, curve.h:310-335)
struct Hit {
    double t;
    D3 p, n, ng;
    int mat, prim;
};
template <bool SHAPES>
__device__ void hit_attributes(const double* __restrict__ tri_n, const RayCtx& R, const PrimRec& r, Hit& h) {
    int ty = SHAPES ? rec_type(r) : REC_TRI;
    h.mat = rec_mat(r);
    h.prim = r.prim;
    double t = 0.0;
    if (ty == REC_TRI) {
        TriHitW w;
        tri_test(R.sh, R.o, r.d, EPS_RAY, DBL_MAX, t, &w);
        double b0 = w.u * w.inv_det, b1 = w.v * w.inv_det, b2 = w.w * w.inv_det;
        D3 v0 = mk(r.d[0], r.d[1], r.d[2]), v1 = mk(r.d[3], r.d[4], r.d[5]), v2 = mk(r.d[6], r.d[7], r.d[8]);
        D3 tgn = normalize(cross(v1 - v0, v2 - v0));     // Tri::finalize (geometry.h:52)
        D3 n0 = tgn, n1 = tgn, n2 = tgn;
        if (rec_smooth(r)) {
            const double* nn = tri_n + 9 * (size_t)r.prim;
            D3 a = ld3(nn), b = ld3(nn + 3), c = ld3(nn + 6);
            if (!(dot(a, a) < 1e-12)) n0 = a;
            if (!(dot(b, b) < 1e-12)) n1 = b;
            if (!(dot(c, c) < 1e-12)) n2 = c;
        }
        h.t = t;
        h.p = R.o + R.d * t;
        D3 ns = n0 * b0 + n1 * b1 + n2 * b2;
        double nl = dot(ns, ns);
        ns = (nl > 1e-18) ? ns * (1.0 / sqrt(nl)) : tgn;
        D3 gn = (dot(tgn, ns) < 0.0) ? neg(tgn) : tgn;
        bool flipped = !(dot(R.d, gn) < 0.0);
        h.ng = gn;
        h.n = flipped ? neg(ns) : ns;
    } else if (ty == REC_SPHERE) {
        sphere_test(R.o, R.d, r.d, EPS_RAY, DBL_MAX, t);
        h.t = t;
        h.p = R.o + R.d * t;
        D3 ng = normalize(h.p - mk(r.d[0], r.d[1], r.d[2]));
        h.ng = ng;
        h.n = (!(dot(R.d, ng) < 0.0)) ? neg(ng) : ng;
    } else {
        CurveWin win;
        curve_test(R.cr, R.o, r.d, EPS_RAY, DBL_MAX, t, &win);
        h.t = t;
        D3 rd = R.cr.dn;
        D3 p0 = mk(r.d[0], r.d[1], r.d[2]), p1 = mk(r.d[3], r.d[4], r.d[5]);
        D3 ba = p1 - p0;
        double rr = r.d[6] - r.d[7];
        double d2 = dot(ba, ba) - rr * rr;
        D3 ro = R.o + rd * win.shift;
        D3 oa = ro - p0, ob = ro - p1;
        h.p = R.o + R.d * t;
        D3 ng;
        if (win.piece == 0) ng = (oa + rd * win.tn) * d2 - ba * win.y;
        else if (win.piece == 1) ng = oa + rd * win.tn;
        else ng = ob + rd * win.tn;
        double nl = sqrt(dot(ng, ng));
        ng = (nl > 1e-18) ? ng * (1.0 / nl) : normalize(ba);
        h.ng = ng;
        h.n = (dot(R.d, ng) < 0.0) ? ng : neg(ng);
    }
}

// ------------------------------------------------------------------ traversal (fp32) ---
// Culling is conservative by construction.  Child planes are floats that enclose the child's
// box grown by 2^-18 x the scene's largest coordinate M (the builders check each against the
// exact box), and a plane x is entered at t = fmaf(x, ix, cx) with ix = 1/d and cx = -o*ix
// rounded to float.  The rounding of o, of cx and of the fma move t by at most ~2^-23 M |ix|
// (far inside the box growth, 2^-18 M |ix|); the rounding of d, of 1/d and of the fma's
// result scale t by at most ~(1 +- 2^-22), inside the interval's widening by 2^-21 (T_LO,
// T_HI).  So no ray culls a child whose primitives the exact fp64 test would hit.
struct RayF {
    float ix, iy, iz;
    float cx, cy, cz;   // -o * ix per axis
    bool nx, ny, nz;    // direction component negative: near plane is the box's hi side
};
__device__ __forceinline__ RayF make_rayf(D3 o, D3 d) {
    RayF r;
    float dx = (float)d.x, dy = (float)d.y, dz = (float)d.z;
    // a zero component is replaced by +-1e-20: the ray moves by at most 1e-20*t, far below
    // the box margin, and the reciprocals stay finite (no inf*0 NaNs in the slab test)
    dx = fabsf(dx) > 1e-20f ? dx : copysignf(1e-20f, dx);
    dy = fabsf(dy) > 1e-20f ? dy : copysignf(1e-20f, dy);
    dz = fabsf(dz) > 1e-20f ? dz : copysignf(1e-20f, dz);
    r.ix = 1.0f / dx; r.iy = 1.0f / dy; r.iz = 1.0f / dz;
    r.cx = -(float)o.x * r.ix; r.cy = -(float)o.y * r.iy; r.cz = -(float)o.z * r.iz;
    r.nx = dx < 0.0f; r.ny = dy < 0.0f; r.nz = dz < 0.0f;
    return r;
}

__device__ __forceinline__ uint32_t byte_of(uint2 w, int i) {
    uint32_t word = (i < 4) ? w.x : w.y;
    return (word >> (8 * (i & 3))) & 0xffu;
}

#define T_LO (1.0f - 4.76837158203125e-7f)   // 1 - 2^-21
#define T_HI (1.0f + 4.76837158203125e-7f)
#define T_CULL (1.0f + 1.9073486328125e-6f)  // 1 + 2^-19: covers the key's slot bits (< 8 ulps)

// Slab test of one child from its near and far planes; the entry distance, or +inf when
// missed.  An empty child's planes (+inf near, -inf far on every axis) give +inf.
__device__ __forceinline__ float slab(float nx, float fx, float ny, float fy, float nz, float fz, const RayF& R,
                                      float tmin_f, float tmax_f) {
    const float a = fmaxf(fmaxf(__fmaf_rn(nx, R.ix, R.cx), __fmaf_rn(ny, R.iy, R.cy)),
                          fmaxf(__fmaf_rn(nz, R.iz, R.cz), tmin_f)) * T_LO;
    const float b = fminf(fminf(__fmaf_rn(fx, R.ix, R.cx), __fmaf_rn(fy, R.iy, R.cy)),
                          fminf(__fmaf_rn(fz, R.iz, R.cz), tmax_f)) * T_HI;
    return a <= b ? a : __int_as_float(0x7f800000);
}

// Entry distances of the eight children of node i, and the node's header (child_base,
// prim_base, meta).  The near planes of an axis are the box's lo side unless the ray's
// direction is negative there.
__device__ __forceinline__ void node_children(const FNode* __restrict__ nodes, uint32_t i, const RayF& R,
                                              float tmin_f, float tmax_f, float (&t)[8], uint4& hdr) {
    const FNode* n = nodes + i;
    hdr = __ldg(reinterpret_cast<const uint4*>(n));
    const float4* nx = reinterpret_cast<const float4*>(R.nx ? n->hi[0] : n->lo[0]);
    const float4* fx = reinterpret_cast<const float4*>(R.nx ? n->lo[0] : n->hi[0]);
    const float4* ny = reinterpret_cast<const float4*>(R.ny ? n->hi[1] : n->lo[1]);
    const float4* fy = reinterpret_cast<const float4*>(R.ny ? n->lo[1] : n->hi[1]);
    const float4* nz = reinterpret_cast<const float4*>(R.nz ? n->hi[2] : n->lo[2]);
    const float4* fz = reinterpret_cast<const float4*>(R.nz ? n->lo[2] : n->hi[2]);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const float4 a = __ldg(nx + h), b = __ldg(fx + h), c = __ldg(ny + h);
        const float4 d = __ldg(fy + h), e = __ldg(nz + h), f = __ldg(fz + h);
        t[4 * h + 0] = slab(a.x, b.x, c.x, d.x, e.x, f.x, R, tmin_f, tmax_f);
        t[4 * h + 1] = slab(a.y, b.y, c.y, d.y, e.y, f.y, R, tmin_f, tmax_f);
        t[4 * h + 2] = slab(a.z, b.z, c.z, d.z, e.z, f.z, R, tmin_f, tmax_f);
        t[4 * h + 3] = slab(a.w, b.w, c.w, d.w, e.w, f.w, R, tmin_f, tmax_f);
    }
}

struct TravCount { unsigned long long nodes, recs, exact; };


// Stack entry: a node index, or (bit 31) a leaf: first record << 2 | (count - 1).
#define LEAF_BIT 0x80000000u
__device__ __forceinline__ uint32_t child_entry(uint32_t child_base, uint32_t prim_base, uint2 meta, int i) {
    uint32_t m = byte_of(meta, i);
    if ((m >> 5) == FNODE_INNER) return child_base + (m & 31u);
    return LEAF_BIT | ((prim_base + (m & 31u)) << 2) | ((m >> 5) - 1u);
}

#define CSWAP(a, b) { uint32_t lo_ = min(a, b); b = max(a, b); a = lo_; }

// A traversal stack in local memory.  (Keeping the top entries in shared memory measured
// slower on B200: the L1 serves this stack well, and shared memory takes L1 capacity.)
template <class E>
struct LocalStack {
    E loc[FTB_STACK];
    __device__ __forceinline__ void put(int i, E v) { loc[i] = v; }
    __device__ __forceinline__ E get(int i) const { return loc[i]; }
};

// Closest-hit walk of one wide BVH.  Children of a node are visited near to far (leaves and
// inner nodes alike, keys sorted by an 8-input network in registers); entries farther than
// the current hit are culled when popped.  The loop is "while-while": a lane steps through
// inner nodes until it holds a leaf, so the lanes of a warp run the expensive leaf tests
// together rather than interleaved with node steps.  leaf(first, count, tmax_f) tests a
// leaf's records and returns the (possibly lowered) fp32 bound on t.
template <bool COUNT, class Stack, class Leaf>
__device__ __forceinline__ float walk_closest(const FNode* __restrict__ nodes, const RayF& F, float tmin_f,
                                              float tmax_f, Stack& st, Leaf& leaf, int32_t* status, TravCount& cnt,
                                              uint32_t root = 0) {
    int sp = 0;
    uint32_t cur = root;
    bool live = true;
    while (live) {
        while (!(cur & LEAF_BIT)) {
            float t[8];
            uint4 hdr;
            node_children(nodes, cur, F, tmin_f, tmax_f, t, hdr);
            if (COUNT) cnt.nodes++;
            uint32_t k[8];
#pragma unroll
            for (int i = 0; i < 8; ++i)
                k[i] = (t[i] == __int_as_float(0x7f800000)) ? 0xffffffffu
                                                           : ((__float_as_uint(t[i]) & ~7u) | (uint32_t)i);
            CSWAP(k[0], k[2]); CSWAP(k[1], k[3]); CSWAP(k[4], k[6]); CSWAP(k[5], k[7]);
            CSWAP(k[0], k[4]); CSWAP(k[1], k[5]); CSWAP(k[2], k[6]); CSWAP(k[3], k[7]);
            CSWAP(k[0], k[1]); CSWAP(k[2], k[3]); CSWAP(k[4], k[5]); CSWAP(k[6], k[7]);
            CSWAP(k[2], k[4]); CSWAP(k[3], k[5]);
            CSWAP(k[1], k[4]); CSWAP(k[3], k[6]);
            CSWAP(k[1], k[2]); CSWAP(k[3], k[4]); CSWAP(k[5], k[6]);
            const uint32_t child_base = hdr.x, prim_base = hdr.y;
            const uint2 meta = make_uint2(hdr.z, hdr.w);
#pragma unroll
            for (int i = 7; i >= 1; --i) {
                if (k[i] != 0xffffffffu) {
                    if (sp >= FTB_STACK) { atomicOr(status, ST_STACK_OVERFLOW); return tmax_f; }
                    st.put(sp, make_uint2(child_entry(child_base, prim_base, meta, (int)(k[i] & 7u)), k[i] & ~7u));
                    ++sp;
                }
            }
            if (k[0] != 0xffffffffu) {
                cur = child_entry(child_base, prim_base, meta, (int)(k[0] & 7u));
                continue;
            }
            bool found = false;
            while (sp > 0) {
                --sp;
                const uint2 v = st.get(sp);
                if (__uint_as_float(v.y) <= tmax_f * T_CULL) { cur = v.x; found = true; break; }
            }
            if (!found) { live = false; break; }
        }
        if (!live) break;
        tmax_f = leaf((int)((cur & ~LEAF_BIT) >> 2), (int)(cur & 3u) + 1, tmax_f);
        bool found = false;
        while (sp > 0) {
            --sp;
            const uint2 v = st.get(sp);
            if (__uint_as_float(v.y) <= tmax_f * T_CULL) { cur = v.x; found = true; break; }
        }
        if (!found) break;
    }
    return tmax_f;
}

// Any-hit walk: order does not change the answer, so children are taken in slot order,
// leaves first; leaf(first, count) returns true on a hit, which ends the walk.
template <bool COUNT, class Stack, class Leaf>
__device__ __forceinline__ bool walk_any(const FNode* __restrict__ nodes, const RayF& F, float tmin_f, float tmax_f,
                                         Stack& st, Leaf& leaf, int32_t* status, TravCount& cnt,
                                         uint32_t root = 0) {
    int sp = 0;
    uint32_t cur = root;
    bool live = true;
    while (live) {
        while (!(cur & LEAF_BIT)) {
            float t[8];
            uint4 hdr;
            node_children(nodes, cur, F, tmin_f, tmax_f, t, hdr);
            if (COUNT) cnt.nodes++;
            const uint2 meta = make_uint2(hdr.z, hdr.w);
            uint32_t hit = 0, imask = 0;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                if (t[i] != __int_as_float(0x7f800000)) hit |= 1u << i;
                if ((byte_of(meta, i) >> 5) == FNODE_INNER) imask |= 1u << i;
            }
            const uint32_t child_base = hdr.x, prim_base = hdr.y;
            uint32_t order = (hit & ~imask) | ((hit & imask) << 8);
            bool have_next = false;
            uint32_t next = 0;
            while (order) {
                int b = __ffs(order) - 1;
                order &= order - 1;
                uint32_t e = child_entry(child_base, prim_base, meta, b & 7);
                if (!have_next) { next = e; have_next = true; continue; }
                if (sp >= FTB_STACK) { atomicOr(status, ST_STACK_OVERFLOW); return false; }
                st.put(sp++, e);
            }
            if (have_next) { cur = next; continue; }
            if (sp == 0) { live = false; break; }
            cur = st.get(--sp);
        }
        if (!live) break;
        if (leaf((int)((cur & ~LEAF_BIT) >> 2), (int)(cur & 3u) + 1)) return true;
        if (sp == 0) break;
        cur = st.get(--sp);
    }
    return false;
}

// Affine::apply / applyDir (linalg.h:105-114) of a 12-double map (3x3 row-major, then t)
__device__ __forceinline__ D3 xf_point(const double* m, D3 p) {
    return mk(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[9],
              m[3] * p.x + m[4] * p.y + m[5] * p.z + m[10],
              m[6] * p.x + m[7] * p.y + m[8] * p.z + m[11]);
}
__device__ __forceinline__ D3 xf_dir(const double* m, D3 v) {
    return mk(m[0] * v.x + m[1] * v.y + m[2] * v.z,
              m[3] * v.x + m[4] * v.y + m[5] * v.z,
              m[6] * v.x + m[7] * v.y + m[8] * v.z);
}
// Affine::applyNormal of toWorld (linalg.h:161-167): toWorld.inverse() is toLocal, read
// transposed.
__device__ __forceinline__ D3 xf_normal(const double* il, D3 n) {
    return mk(il[0] * n.x + il[3] * n.y + il[6] * n.z,
              il[1] * n.x + il[4] * n.y + il[7] * n.z,
              il[2] * n.x + il[5] * n.y + il[8] * n.z);
}
__device__ __forceinline__ int rec_inst(const PrimRec& r) { return (int)__double_as_longlong(r.d[0]); }

// The world ray mapped into an instance's local space (Scene::closestHit instance leaf,
// scene.h:2226-2228): local t equals world t, the direction is not renormalized.
struct LocalRay { D3 o, d; };
__device__ __forceinline__ LocalRay to_local(const DevInst& I, D3 o, D3 d) {
    LocalRay L;
    L.o = xf_point(I.xl, o);
    L.d = xf_dir(I.xl, d);
    return L;
}

// The next double above a positive t (DBL_MAX -> +inf): record tests given this bound accept
// t <= best, so that an exact tie can be settled by primitive index.
__device__ __forceinline__ double next_up(double t) { return __longlong_as_double(__double_as_longlong(t) + 1); }

// Exact ties in t go to the lower primitive index (world index first, then the index within
// the BLAS).  The reference takes the first tied primitive its own hierarchy happens to
// test; with the index rule a closest hit does not depend on the hierarchy at all, and the
// oracle applies the same rule.
struct BestHit { int prim, sub_prim; };

// Blas::intersectLocal (scene.h:1017-1026): nearest BLAS triangle with t <= best_t that wins
// against the current best (ties by index); updates best_t / tmax_f / bh and returns the BLAS
// record, or -1.  `inst_prim` is the instance's world primitive index.
template <bool COUNT>
__device__ __noinline__ int blas_closest(const DevInst& I, D3 wo, D3 wd, double tmin, double& best_t,
                                         float& tmax_f, int inst_prim, BestHit& bh, int32_t* status,
                                         TravCount& cnt) {
    const LocalRay L = to_local(I, wo, wd);
    const Shear sh = make_shear(L.d);
    const RayF F = make_rayf(L.o, L.d);
    const PrimRec* __restrict__ recs = I.recs;
    int best = -1;
    auto leaf = [&](int first, int count, float tm) -> float {
        for (int k = 0; k < count; ++k) {
            if (COUNT) { cnt.recs++; cnt.exact++; }
            PrimRec r;
            load_rec(recs, first + k, r);
            double t;
            if (tri_test(sh, L.o, r.d, tmin, next_up(best_t), t, nullptr) &&
                (t < best_t || inst_prim < bh.prim || (inst_prim == bh.prim && r.prim < bh.sub_prim))) {
                best_t = t; best = first + k; tm = __double2float_ru(t);
                bh.prim = inst_prim; bh.sub_prim = r.prim;
            }
        }
        return tm;
    };
    LocalStack<uint2> st;
    tmax_f = walk_closest<COUNT>(I.nodes, F, __double2float_rd(tmin), tmax_f, st, leaf, status, cnt);
    return best;
}

// Blas::occludedLocal (scene.h:1027-1033)
template <bool COUNT>
__device__ __noinline__ bool blas_any(const DevInst& I, D3 wo, D3 wd, double tmin, double seg, float tmax_f,
                                      int32_t* status, TravCount& cnt) {
    const LocalRay L = to_local(I, wo, wd);
    const Shear sh = make_shear(L.d);
    const RayF F = make_rayf(L.o, L.d);
    const PrimRec* __restrict__ recs = I.recs;
    auto leaf = [&](int first, int count) -> bool {
        for (int k = 0; k < count; ++k) {
            if (COUNT) { cnt.recs++; cnt.exact++; }
            PrimRec r;
            load_rec(recs, first + k, r);
            double t;
            if (tri_test(sh, L.o, r.d, tmin, seg, t, nullptr)) return true;
        }
        return false;
    };
    LocalStack<uint32_t> st;
    return walk_any<COUNT>(I.nodes, F, __double2float_rd(tmin), tmax_f, st, leaf, status, cnt);
}

// Closest hit (Scene::closestHit, scene.h:2194-2242): returns the world record (or -1) and
// t; for an instance record, *sub receives the BLAS record.  INST selects the variant that
// can meet instance records (scenes with instances); the plain variant has no such branch.
template <bool COUNT, bool INST, bool SHAPES>
__device__ int traverse_closest(const DevScene& sc, const RayCtx& R, double tmin, double& best_t, int* sub,
                                int32_t* status, TravCount& cnt) {
    const RayF F = make_rayf(R.o, R.d);
    best_t = DBL_MAX;
    int best = -1;
    BestHit bh{INT_MAX, INT_MAX};
    const PrimRec* __restrict__ recs = sc.recs;
    auto leaf = [&](int first, int count, float tm) -> float {
        for (int k = 0; k < count; ++k) {
            if (COUNT) cnt.recs++;
            PrimRec r;
            load_rec(recs, first + k, r);
            if (INST && rec_type(r) == REC_INST) {
                int s = blas_closest<COUNT>(sc.inst[rec_inst(r)], R.o, R.d, tmin, best_t, tm, r.prim, bh, status, cnt);
                if (s >= 0) { best = first + k; *sub = s; }
                continue;
            }
            if (COUNT) cnt.exact++;
            double t;
            // t <= best_t from the test; a tie goes to the lower index
            if (rec_test<SHAPES>(R, r, tmin, next_up(best_t), t) && (t < best_t || r.prim < bh.prim)) {
                best_t = t; best = first + k; tm = __double2float_ru(t);
                bh.prim = r.prim; bh.sub_prim = INT_MAX;
            }
        }
        return tm;
    };
    LocalStack<uint2> st;
    const float tm = walk_closest<COUNT>(sc.nodes, F, __double2float_rd(tmin), FLT_MAX, st, leaf, status, cnt);
    if (SHAPES && sc.root2 > 0)   // the curves' hierarchy, under the bound the first walk left
        walk_closest<COUNT>(sc.nodes, F, __double2float_rd(tmin), tm, st, leaf, status, cnt, (uint32_t)sc.root2);
    return best;
}

// Any hit with t in [tmin, seg) (Scene::occluded, scene.h:2249-2271).
template <bool COUNT, bool INST, bool SHAPES>
__device__ bool traverse_any(const DevScene& sc, const RayCtx& R, double tmin, double seg, int32_t* status,
                             TravCount& cnt) {
    const RayF F = make_rayf(R.o, R.d);
    const float tmin_f = __double2float_rd(tmin), tmax_f = __double2float_ru(seg);
    const PrimRec* __restrict__ recs = sc.recs;
    auto leaf = [&](int first, int count) -> bool {
        for (int k = 0; k < count; ++k) {
            if (COUNT) cnt.recs++;
            PrimRec r;
            load_rec(recs, first + k, r);
            if (INST && rec_type(r) == REC_INST) {
                if (blas_any<COUNT>(sc.inst[rec_inst(r)], R.o, R.d, tmin, seg, tmax_f, status, cnt)) return true;
                continue;
            }
            if (COUNT) cnt.exact++;
            double t;
            if (rec_test<SHAPES>(R, r, tmin, seg, t)) return true;
        }
        return false;
    };
    LocalStack<uint32_t> st;
    // a scene with two hierarchies keeps a top node over both in its last three nodes
    const uint32_t root = (SHAPES && sc.root2 > 0) ? (uint32_t)(sc.n_nodes - 3) : 0u;
    return walk_any<COUNT>(sc.nodes, F, tmin_f, tmax_f, st, leaf, status, cnt, root);
}

// Hit on BLAS record `sub` of instance I, in world terms: the local hit's attributes
// (intersectTri on the local ray) mapped like Scene::instanceHitToWorld (scene.h:2139-2162).
__device__ void instance_hit(const DevInst& I, int sub, D3 ro, D3 rd, Hit& h) {
    const LocalRay L = to_local(I, ro, rd);
    RayCtx R;
    R.o = L.o; R.d = L.d;
    R.sh = make_shear(L.d);
    PrimRec br;
    load_rec(I.recs, sub, br);
    hit_attributes<false>(I.tri_n, R, br, h);   // BLAS records are triangles
    h.p = ro + rd * h.t;                        // world t == local t
    D3 wn = normalize(xf_normal(I.xl, h.n));
    D3 wng = normalize(xf_normal(I.xl, h.ng));
    h.ng = wng;
    h.n = (dot(rd, wn) < 0.0) ? wn : neg(wn);
    if (I.mat_override >= 0) h.mat = I.mat_override;
}

__device__ __forceinline__ RayCtx make_ray(D3 o, D3 d) {
    RayCtx R;
    R.o = o; R.d = d;
    R.sh = make_shear(d);
    R.cr = make_curve_ray(d);
    return R;
}

// ------------------------------------------------------------------ media --------------
__device__ __forceinline__ double med_sigma_t(const DevScene& sc, const DevMed& m, double lam) {
    double v = spec_eval(sc, m.sa, lam) + spec_eval(sc, m.ss, lam);
    return v > 0.0 ? v : 0.0;
}
__device__ __forceinline__ double med_albedo(const DevScene& sc, const DevMed& m, double lam) {
    double s = spec_eval(sc, m.ss, lam); s = s > 0.0 ? s : 0.0;
    double a = spec_eval(sc, m.sa, lam);
    double t = s + (a > 0.0 ? a : 0.0);
    return t > 0.0 ? s / t : 0.0;
}
// Medium::clipToBounds (scene.h:655-685)
__device__ bool clip_to_bounds(const DevMed& m, D3 o, D3 d, double t0, double t1, double& ta, double& tb) {
    if (m.bound == FTB_BOUND_NONE) { ta = t0; tb = t1; return t1 > t0; }
    if (m.bound == FTB_BOUND_SPHERE) {
        D3 oc = o - ld3(m.center);
        double A = dot(d, d);
        double B = 2.0 * dot(oc, d);
        double C = dot(oc, oc) - m.radius * m.radius;
        double disc = B * B - 4.0 * A * C;
        if (disc <= 0.0 || A <= 0.0) return false;
        double sd = sqrt(disc);
        double s0 = (-B - sd) / (2.0 * A), s1 = (-B + sd) / (2.0 * A);
        double lo = t0 > s0 ? t0 : s0, hi = t1 < s1 ? t1 : s1;
        if (lo > hi) return false;
        ta = lo; tb = hi; return tb > ta;
    }
    double lo = t0, hi = t1;
    for (int a = 0; a < 3; ++a) {
        double oa = comp(o, a), da = comp(d, a);
        double mn = m.bmin[a], mx = m.bmax[a];
        if (fabs(da) < 1e-12) { if (oa < mn || oa > mx) return false; continue; }
        double inv = 1.0 / da;
        double s0 = (mn - oa) * inv, s1 = (mx - oa) * inv;
        if (s0 > s1) { double t = s0; s0 = s1; s1 = t; }
        lo = (lo < s0) ? s0 : lo;
        hi = (s1 < hi) ? s1 : hi;
        if (lo > hi) return false;
    }
    ta = lo; tb = hi; return tb > ta;
}
// sampleMediaCollision, homogeneous (render.h:377-398, 444-458)
__device__ bool sample_media_collision(const DevScene& sc, D3 o, D3 d, double dmax, double lam, Pcg& rng,
                                       double& thit, int& which) {
    double best = dmax; int w = -1;
    for (int i = 0; i < sc.n_med; ++i) {
        const DevMed& m = sc.med[i];
        double st = med_sigma_t(sc, m, lam);
        if (st <= 0.0) continue;
        double ta, tb;
        if (!clip_to_bounds(m, o, d, 0.0, dmax, ta, tb)) continue;
        double t = ta - log(1.0 - uniform(rng)) / st;
        if (t < tb && t < best) { best = t; w = i; }
    }
    if (w < 0) return false;
    thit = best; which = w; return true;
}
// mediaTransmittance, homogeneous (render.h:403-421, 461-469)
__device__ double media_transmittance(const DevScene& sc, D3 o, D3 d, double dist, double lam) {
    double tr = 1.0;
    for (int i = 0; i < sc.n_med; ++i) {
        const DevMed& m = sc.med[i];
        double st = med_sigma_t(sc, m, lam);
        double mt = 1.0;
        if (st > 0.0) {
            double ta, tb;
            if (clip_to_bounds(m, o, d, 0.0, dist, ta, tb)) mt = exp(-st * (tb - ta));
        }
        tr *= mt;
        if (tr <= 0.0) break;
    }
    return tr;
}

// ------------------------------------------------------------------ camera -------------
// Camera::project, rectilinear (camera.h:137-151)
__device__ __forceinline__ bool cam_project(const DevCam& c, D3 p, int& px, int& py, double& cos_cam,
                                            double& dist2) {
    D3 d = p - ld3(c.eye);
    double cz = dot(d, ld3(c.w));
    if (cz <= 1e-9) return false;
    double cx = dot(d, ld3(c.u)), cy = dot(d, ld3(c.v));
    double ix = (cx / cz) / c.thx - 0.0;
    double iy = (cy / cz) / c.thy;
    if (ix < -1 || ix >= 1 || iy < -1 || iy >= 1) return false;
    px = (int)((ix * 0.5 + 0.5) * c.rx);
    py = (int)((iy * 0.5 + 0.5) * c.ry);
    dist2 = dot(d, d);
    cos_cam = cz / sqrt(dist2);
    return true;
}
__device__ __forceinline__ double cam_pixel_solid_angle(const DevCam& c, double cos_cam) {
    double ipa = 4.0 * c.thx * c.thy;
    double ppa = ipa / ((double)c.rx * (double)c.ry);
    return ppa * cos_cam * cos_cam * cos_cam;
}

// geometry.h:174-242
__device__ __forceinline__ D3 oriented_geo_n(const Hit& h) { return (dot(h.ng, h.n) >= 0.0) ? h.ng : neg(h.ng); }
__device__ __forceinline__ double shading_adjoint_corr(D3 wi, D3 wo, D3 ns, D3 ng) {
    double denom = fabs(dot(wi, ng)) * fabs(dot(wo, ns));
    if (denom <= 1e-8) return 1.0;
    double num = fabs(dot(wi, ns)) * fabs(dot(wo, ng));
    return num / denom;
}
__device__ __forceinline__ double shadow_terminator_g(D3 wi, D3 ns, D3 ng) {
    double cos_ng_ns = dot(ng, ns);
    if (cos_ng_ns >= 1.0 - 1e-7) return (dot(ng, wi) > 0.0) ? 1.0 : 0.0;
    double cos_ng_wi = dot(ng, wi);
    if (cos_ng_wi <= 0.0) return 0.0;
    double denom = dot(ns, wi) * cos_ng_ns;
    if (denom <= 1e-8) return 1.0;
    double g = cos_ng_wi / denom;
    if (g >= 1.0) return 1.0;
    return g * g * (1.0 - g) + g;
}

// ------------------------------------------------------------------ shadow queue -------
__device__ __forceinline__ int agg_inc(int32_t* ctr) {
    cg::coalesced_group g = cg::coalesced_threads();
    int base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(ctr, (int)g.size());
    return g.shfl(base, 0) + (int)g.thread_rank();
}

// A queue of paths is two-ended: paths outside every dielectric grow from entry 0 up
// (count q[0]), paths inside one -- or leaving a curve, among the strands -- grow from entry
// W-1 down (count q[1]), so each end holds paths of similar traversal cost (inside a closed
// mesh a ray crosses it; outside most rays meet a wall after a few nodes) and warps diverge
// less.  Queue position p < q[0] is entry
// p; position q[0] + k is entry W-1-k.
__device__ __forceinline__ int queue_len(const int32_t* q) { return q[0] + q[1]; }

// Dynamic work distribution over a queue: a warp takes the next 32 positions from a
// per-launch counter in Wave::counts whenever it is done, so warps that drew short paths
// take more and a launch ends with fewer idle SMs than a fixed grid-stride split.  Every
// lane of the warp calls warp_fetch; the loop ends for the whole warp at once.
__device__ __forceinline__ int warp_fetch(int32_t* ctr) {
    int base = 0;
    if ((threadIdx.x & 31) == 0) base = atomicAdd(ctr, 32);
    return __shfl_sync(0xffffffffu, base, 0);
}
#define FTB_FOR_WARP_CHUNKS(var, n, ctr)                                                      \
    for (int var##_base = warp_fetch(ctr); var##_base < (n); var##_base = warp_fetch(ctr))   \
        if (const int var = var##_base + (int)(threadIdx.x & 31); var < (n))
__device__ __forceinline__ int queue_entry(const Wave& w, int front, int p) {
    return p < front ? p : w.W - 1 - (p - front);
}

// A one-wavelength connection: the film increments cieX/Y/Z(lambda) * contribution in the
// order Film::add forms them (scene_film.h:12), from the matching functions evaluated once
// per path at emission.
__device__ __forceinline__ void push_shadow(const Wave& w, const Frame& f, int job, int view, D3 o, D3 d,
                                            double tmax, double val, const double* cie, int pix) {
    int i = agg_inc(&w.counts[kShadowCount]);
    if (i >= w.S) { atomicOr(f.status, ST_QUEUE_OVERFLOW); return; }
    w.sox[i] = o.x; w.soy[i] = o.y; w.soz[i] = o.z;
    w.sdx[i] = d.x; w.sdy[i] = d.y; w.sdz[i] = d.z;
    w.smax[i] = tmax; w.spix[i] = pix;
    w.sxyz[i] = cie[0] * val; w.sxyz[w.S + i] = cie[1] * val; w.sxyz[2 * (size_t)w.S + i] = cie[2] * val;
    w.sjob[i] = job; w.sview[i] = view;
}

// The views a job's vertices connect to: its own camera, or every view of a multi-camera job.
__device__ __forceinline__ int view_count(const DevJob& J) { return J.n_views > 1 ? J.n_views : 1; }
__device__ __forceinline__ const DevCam& view_cam(const DevJob& J, int v) {
    return J.n_views > 1 ? J.views[v].cam : J.cam;
}
__device__ __forceinline__ int64_t* view_film(const DevJob& J, int v) {
    return J.n_views > 1 ? J.views[v].film : J.film;
}

// connectGeom + connect, model B (render.h:499-559); the occlusion test is deferred to
// k_shadow, the rest of the contribution is formed here in the reference's order.
template <bool MEDIA>
__device__ void connect_surface(const DevScene& sc, const DevJob& J, const Wave& w, const Frame& f, int job,
                                D3 p, D3 n, D3 ng, D3 wi, double lam, const double* cie, double beta, double rho) {
    for (int v = 0; v < view_count(J); ++v) {
        const DevCam& cam = view_cam(J, v);
        D3 to_cam = ld3(cam.eye) - p;
        double dist = len(to_cam);
        D3 wdir = to_cam / dist;
        double cos_surf = dot(n, wdir);
        if (cos_surf <= 0) continue;
        double stg = shadow_terminator_g(wdir, n, ng);
        if (stg <= 0.0) continue;
        int px, py; double cos_cam, dist2;
        if (!cam_project(cam, p, px, py, cos_cam, dist2)) continue;
        double omega = cam_pixel_solid_angle(cam, cos_cam);
        double corr = shading_adjoint_corr(wi, wdir, n, ng);
        double denom = dist2 * omega;
        double fr = rho / PI_D;
        double contrib = beta * fr * cos_surf * corr / denom * stg;
        if (MEDIA && sc.n_med > 0) contrib *= media_transmittance(sc, p, wdir, dist, lam);
        push_shadow(w, f, job, v, p + ng * 1e-6, wdir, dist - 2e-6, contrib, cie, py * cam.rx + px);
    }
}
// connectVolume (render.h:584-600)
__device__ void connect_volume(const DevScene& sc, const DevJob& J, const Wave& w, const Frame& f, int job,
                               const DevMed& m, D3 p, D3 win, double lam, const double* cie, double beta) {
    for (int v = 0; v < view_count(J); ++v) {
        const DevCam& cam = view_cam(J, v);
        D3 to_cam = ld3(cam.eye) - p;
        double dist = len(to_cam);
        D3 wdir = to_cam / dist;
        int px, py; double cos_cam, dist2;
        if (!cam_project(cam, p, px, py, cos_cam, dist2)) continue;
        double ph = hg_phase(dot(win, wdir), m.g);
        double alb = med_albedo(sc, m, lam);
        double omega = cam_pixel_solid_angle(cam, cos_cam);
        double contrib = beta * alb * ph / (dist2 * omega);
        contrib *= media_transmittance(sc, p, wdir, dist, lam);
        push_shadow(w, f, job, v, p + wdir * 1e-6, wdir, dist - 2e-6, contrib, cie, py * cam.rx + px);
    }
}

// ------------------------------------------------------------------ planar mirrors -----
// A mirror connection in the shadow queue (marked by a negative pixel, ~pixel): vertex p,
// the direction wP toward the eye's mirror image and the distance dP to the mirror point in
// the origin / direction / max fields, view | plane << 16, the wavelength, the vertex factor
// beta * (weight * shape) and cieX/Y/Z(lambda) in place of the film increments -- the
// mirror's reflectance is known only once k_shadow has seen which mirror the eye meets.
__device__ __forceinline__ void push_mirror(const Wave& w, const Frame& f, int job, int view, int plane, D3 p, D3 wP,
                                            double dP, double a, double lam, const double* cie, int pix) {
    int i = agg_inc(&w.counts[kShadowCount]);
    if (i >= w.S) { atomicOr(f.status, ST_QUEUE_OVERFLOW); return; }
    w.sox[i] = p.x; w.soy[i] = p.y; w.soz[i] = p.z;
    w.sdx[i] = wP.x; w.sdy[i] = wP.y; w.sdz[i] = wP.z;
    w.smax[i] = dP; w.spix[i] = ~pix;
    w.sval[i] = a; w.slam[i] = lam;
    w.sxyz[i] = cie[0]; w.sxyz[w.S + i] = cie[1]; w.sxyz[2 * (size_t)w.S + i] = cie[2];
    w.sjob[i] = job; w.sview[i] = view | (plane << 16);
}

// connectSpecularPlane's geometry (render.h:1334-1366) for one plane and view: the vertex and
// the eye on the same side of the plane, the path unfolded through the eye's mirror image,
// the vertex factor (SpecVtx::shape, render.h:897-901), the mirror point inside the plane's
// box and in the image.  false when the connection is culled; else the direction wP to the
// mirrored eye, the distance dP to the mirror, `shape` and the pixel.  `volume`: a medium
// scatter with incoming direction nw and HG g; otherwise a surface with normal nw.
__device__ __forceinline__ bool mirror_geometry(const DevPlane& mp, const DevCam& cam, D3 p, bool volume, D3 nw,
                                                double g, D3& wP, double& dP, double& shape, int& pix) {
    const D3 pn = ld3(mp.n);
    const D3 eye = ld3(cam.eye);
    const double se = dot(pn, eye) - mp.d;
    const double sp = dot(pn, p) - mp.d;
    if (!(se * sp > 0.0)) return false;
    const D3 eye_m = eye - pn * (2.0 * se);
    wP = eye_m - p;
    const double D = len(wP);
    if (D < 1e-9) return false;
    wP = wP * (1.0 / D);
    if (volume) {
        shape = hg_phase(dot(nw, wP), g);
    } else {
        const double cs = dot(nw, wP);
        shape = cs <= 0.0 ? -1.0 : cs / PI_D;
    }
    if (shape < 0.0) return false;
    const double denom = dot(pn, wP);
    if (fabs(denom) < 1e-12) return false;
    dP = (mp.d - dot(pn, p)) / denom;
    if (dP <= 1e-7 || dP >= D - 1e-7) return false;
    const D3 R = p + wP * dP;
    if (R.x < mp.lo[0] || R.x > mp.hi[0] || R.y < mp.lo[1] || R.y > mp.hi[1] || R.z < mp.lo[2] || R.z > mp.hi[2])
        return false;
    int px, py; double cos_cam, dist2e;
    if (!cam_project(cam, R, px, py, cos_cam, dist2e)) return false;
    if (cam_pixel_solid_angle(cam, cos_cam) <= 0.0) return false;
    pix = py * cam.rx + px;
    return true;
}

// camSpecularSplatAll / camSpecularSplatVolumeAll (render.h:1515-1585) over the planar
// mirrors: a mirror record for k_shadow per plane and view that the geometry lets through.
// `weight`: the vertex's albedo.
__device__ __noinline__ void connect_mirrors(const DevScene& sc, const DevJob& J, const Wave& w, const Frame& f,
                                             int job, D3 p, bool volume, D3 nw, double g, double lam,
                                             const double* cie, double beta, double weight) {
    for (int k = 0; k < sc.n_planes; ++k) {
        for (int v = 0; v < view_count(J); ++v) {
            D3 wP; double dP, shape; int pix;
            if (!mirror_geometry(sc.planes[k], view_cam(J, v), p, volume, nw, g, wP, dP, shape, pix)) continue;
            push_mirror(w, f, job, v, k, p, wP, dP, beta * (weight * shape), lam, cie, pix);
        }
    }
}

// The same for a bundle's live wavelengths (camSpecularSplatAllHero, render.h:1570-1576): a
// record carries (lambda_i, beta_i x (rho_i x shape)) per wavelength, as the bundle's camera
// connections do; k_shadow_hero evaluates the mirror's reflectance per wavelength.
__device__ __noinline__ void connect_mirrors_hero(const DevScene& sc, const DevJob& J, const Wave& w, const Frame& f,
                                                  int job, D3 p, D3 n, const double* lam, const double* beta,
                                                  const double* rho, int nup) {
    for (int k = 0; k < sc.n_planes; ++k) {
        for (int v = 0; v < view_count(J); ++v) {
            D3 wP; double dP, shape; int pix;
            if (!mirror_geometry(sc.planes[k], view_cam(J, v), p, false, n, 0.0, wP, dP, shape, pix)) continue;
            const int i = agg_inc(&w.counts[kShadowCount]);
            if (i >= w.S) { atomicOr(f.status, ST_QUEUE_OVERFLOW); continue; }
            w.sox[i] = p.x; w.soy[i] = p.y; w.soz[i] = p.z;
            w.sdx[i] = wP.x; w.sdy[i] = wP.y; w.sdz[i] = wP.z;
            w.smax[i] = dP; w.spix[i] = ~pix; w.sjob[i] = job; w.sview[i] = v | (k << 16);
            w.slam[i] = lam[0]; w.sval[i] = beta[0] * (rho[0] * shape);
            for (int q = 1; q < nup; ++q) {
                w.xlam[(size_t)(q - 1) * w.S + i] = lam[q];
                w.xval[(size_t)(q - 1) * w.S + i] = beta[q] * (rho[q] * shape);
            }
            w.snup[i] = nup;
        }
    }
}

// isPlanarMirrorMat (scene.h:356-360)
__device__ __forceinline__ bool planar_mirror(const DevMat& m) {
    return m.type == FTB_MAT_MIRROR || m.type == FTB_MAT_HALF_MIRROR ||
           (m.type == FTB_MAT_GLOSSY && m.roughness <= 0.0);
}

// ------------------------------------------------------------------ tallies ------------
__device__ __forceinline__ long long to_fixed(double v, double scale_inv, int32_t* status) {
    double s = v * scale_inv;
    if (!(fabs(s) < 4.611686018427388e18)) {   // 2^62
        atomicOr(status, ST_FILM_SATURATED);
        return 0;
    }
    return __double2ll_rn(s);
}

// Sum a per-thread value over the block and add it to a global tally once per block.
__device__ void block_tally(unsigned long long* dst, long long v) {
    __shared__ long long red[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
        long long s = lane < nw ? red[lane] : 0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0 && s != 0) atomicAdd(dst, (unsigned long long)s);
    }
}

enum { T_EMIT = 0, T_ABS = 1, T_SENSOR = 2, T_ESC = 3, T_RES = 4 };

// Per-thread energy tallies.  A single-job launch reduces them over the block once at the
// end of the kernel.  In a multi-job launch a thread moves its sums into a per-block table
// in shared memory (one row of five per job of the table) whenever the job of the path it
// books changes -- often, in a streaming pass, where the paths of neighbouring jobs share
// the queues -- and the block adds the table's nonzero entries to the jobs' tallies once
// at the end, so the global atomics per launch do not grow with the job changes.
struct TallyAcc {
    int job;
    bool multi;
    long long v[5];
};
__device__ __forceinline__ unsigned long long* tally_table() {
    __shared__ unsigned long long tab[kWaveJobs * 5];
    return tab;
}
// Called by every thread of the block at the start of the kernel.
__device__ __forceinline__ void tally_init(TallyAcc& a, bool multi, int n_jobs) {
    a.job = 0;
    a.multi = multi;
#pragma unroll
    for (int k = 0; k < 5; ++k) a.v[k] = 0;
    if (multi) {
        unsigned long long* tab = tally_table();
        for (int e = threadIdx.x; e < n_jobs * 5; e += blockDim.x) tab[e] = 0ull;
        __syncthreads();
    }
}
__device__ __forceinline__ void tally_flush(TallyAcc& a) {
    unsigned long long* row = tally_table() + 5 * a.job;
#pragma unroll
    for (int k = 0; k < 5; ++k)
        if (a.v[k]) { atomicAdd(row + k, (unsigned long long)a.v[k]); a.v[k] = 0; }
}
__device__ __forceinline__ void tally_add(TallyAcc& a, const DevJob* jobs, bool multi, int job, int k,
                                          long long x) {
    if (multi && job != a.job) { tally_flush(a); a.job = job; }
    a.v[k] += x;
}
__device__ void block_tally(unsigned long long* dst, long long v);
// Called by every thread of the block at the end of the kernel.
__device__ __forceinline__ void tally_finish(TallyAcc& a, const DevJob* jobs, bool multi, int n_jobs = 1) {
    if (multi) {
        tally_flush(a);
        __syncthreads();
        const unsigned long long* tab = tally_table();
        for (int e = threadIdx.x; e < n_jobs * 5; e += blockDim.x)
            if (tab[e]) atomicAdd(jobs[e / 5].tally + e % 5, tab[e]);
        return;
    }
    unsigned long long* t = jobs[0].tally;
#pragma unroll
    for (int k = 0; k < 5; ++k) block_tally(t + k, a.v[k]);
}

__device__ __forceinline__ uint64_t fnv_i32(uint64_t h, int32_t v) {
    uint32_t u = (uint32_t)v;
#pragma unroll
    for (int i = 0; i < 4; ++i) { h ^= (u >> (8 * i)) & 0xffu; h *= 1099511628211ULL; }
    return h;
}

// Per-path instrumentation (parity tests only).
__device__ __forceinline__ void log_finish(const Wave& w, const PathState& ps, int i, int fate, double beta) {
    if (!w.logs) return;
    ftb_photon_log& L = w.logs[ps.pid[i] - (uint64_t)w.log_base];
    L.n_hits = ps.lnh[i];
    L.fate = fate;
    L.prim_hash = ps.lhash[i];
    L.beta = beta;
    for (int k = 0; k < 8; ++k) L.prims[k] = ps.lprims[k * w.W + i];
}
// The log of a photon that ends at emission (it never enters a queue).
__device__ __forceinline__ void log_emitted(const Wave& w, uint64_t photon, int fate, double beta) {
    if (!w.logs) return;
    ftb_photon_log& L = w.logs[photon - (uint64_t)w.log_base];
    L.n_hits = 0;
    L.fate = fate;
    L.prim_hash = 1469598103934665603ULL;
    L.beta = beta;
    for (int k = 0; k < 8; ++k) L.prims[k] = -2;
}
__device__ __forceinline__ void log_start(const Wave& w, const PathState& ps, int i, uint64_t photon) {
    if (!w.logs) return;
    ps.pid[i] = photon;
    ps.lhash[i] = 1469598103934665603ULL; ps.lnh[i] = 0;
    for (int q = 0; q < 8; ++q) ps.lprims[q * w.W + i] = -2;
}
// A hit joins the log of path i (in place), before shading decides its fate.
template <bool INST>
__device__ __forceinline__ void log_hit(const Wave& w, const PathState& ps, int i, const DevScene& sc, int rec) {
    if (!w.logs) return;
    const int nh = ps.lnh[i];
    const int prim = rec >= 0 ? sc.recs[rec].prim : -1;
    uint64_t hsh = fnv_i32(ps.lhash[i], prim);
    if (INST && rec >= 0 && rec_type(sc.recs[rec]) == REC_INST)   // and the BLAS triangle
        hsh = fnv_i32(hsh, sc.inst[rec_inst(sc.recs[rec])].recs[w.hit_sub[i]].prim);
    ps.lhash[i] = hsh;
    if (nh < 8) ps.lprims[nh * w.W + i] = prim;
    ps.lnh[i] = nh + 1;
}
// A surviving path's log moves with it.
__device__ __forceinline__ void log_move(const Wave& w, const PathState& in, int i, const PathState& out, int o) {
    if (!w.logs) return;
    out.pid[o] = in.pid[i];
    out.lhash[o] = in.lhash[i];
    out.lnh[o] = in.lnh[i];
    for (int q = 0; q < 8; ++q) out.lprims[q * w.W + o] = in.lprims[q * w.W + i];
}

// Photon sources of the emission kernels.  A wave emits photon photon0 + (t - slot0) of the
// table range holding t, for t < params[1]; a streaming pass's refill emits stream indices
// next .. next+F-1, F = the free places (slots less the survivors already queued, at most the
// photons left), each mapped to its range's photon.
struct PhotonSource {
    int64_t n;           // photons this launch emits
    int64_t next;        // streaming: first stream index
    int32_t have;        // streaming: survivors already in the output queue
};
template <bool STREAM>
__device__ __forceinline__ PhotonSource photon_source(const Wave& w, const int32_t* out_count) {
    PhotonSource p;
    if (STREAM) {
        const int64_t total = reinterpret_cast<const int64_t*>(w.params)[1];
        p.next = w.ctl->next;
        p.have = out_count[0];   // the refill appends through ctl->taken, so this stays put
        const int64_t room = (int64_t)w.params[1] - p.have - out_count[1], left = total - p.next;
        p.n = left < room ? left : room;
    } else {
        p.n = w.params[1];
        p.next = 0;
        p.have = 0;
    }
    return p;
}
// Job and photon index of the t-th photon of this launch.
template <bool STREAM>
__device__ __forceinline__ int photon_job(const DevJob* __restrict__ jobs, int n_jobs, const PhotonSource& p,
                                          int64_t t, uint64_t& photon) {
    int j = 0;
    if (STREAM) {
        const int64_t g = p.next + t;
        if (n_jobs > 1) {
            int lo = 0, hi = n_jobs - 1;
            while (lo < hi) { int mid = (lo + hi + 1) / 2; if (jobs[mid].g0 <= g) lo = mid; else hi = mid - 1; }
            j = lo;
        }
        photon = jobs[j].photon0 + (uint64_t)(g - jobs[j].g0);
    } else {
        const int slot = (int)t;
        if (n_jobs > 1) {
            int lo = 0, hi = n_jobs - 1;
            while (lo < hi) { int mid = (lo + hi + 1) / 2; if (jobs[mid].slot0 <= slot) lo = mid; else hi = mid - 1; }
            j = lo;
        }
        photon = jobs[j].photon0 + (uint64_t)(slot - jobs[j].slot0);
    }
    return j;
}
// Queue position of a photon that survives emission, with its job, bounce count and log set.
template <bool STREAM>
__device__ __forceinline__ int photon_enqueue(const Wave& w, const PathState& out, int32_t* out_count,
                                              const PhotonSource& p, int j, bool multi, uint64_t photon) {
    const int o = STREAM ? p.have + agg_inc(&w.ctl->taken) : agg_inc(out_count);
    out.nbounce[o] = 0;
    if (multi) out.job[o] = j;
    log_start(w, out, o, photon);
    return o;
}

// ------------------------------------------------------------------ emission -----------
// Scene::selectEmitter (scene.h:1851-1857): no draw with one emitter.
__device__ __forceinline__ int select_emitter(const DevScene& sc, Pcg& rng) {
    if (sc.n_emit <= 1) return 0;
    double u = uniform(rng);
    int lo = 0, hi = sc.n_emit - 1;
    while (lo < hi) { int mid = (lo + hi) / 2; if (sc.emit_cdf[mid] < u) lo = mid + 1; else hi = mid; }
    return lo;
}
// Emitter::samplePoint (scene.h:815-880) and the emission direction (render.h:1938-1941)
__device__ __forceinline__ void emit_sample(const DevEmit& em, Pcg& rng, D3& origin, D3& emit_n, D3& dir) {
    double u1 = uniform(rng), u2 = uniform(rng);
    if (em.shape == FTB_EMIT_SPHERE) {
        double z = 1.0 - 2.0 * u1;
        double s = 1.0 - z * z;
        double r = sqrt(s > 0.0 ? s : 0.0);
        double phi = 2.0 * PI_D * u2;
        D3 d = mk(r * cos(phi), r * sin(phi), z);
        emit_n = d;
        origin = ld3(em.origin) + d * em.radius;
    } else {
        origin = ld3(em.origin) + ld3(em.u) * u1 + ld3(em.v) * u2;
        emit_n = ld3(em.normal);
    }
    dir = em.collimated ? ld3(em.beam) : cosine_hemisphere(emit_n, rng);
}
// EmissionSampler::sampleAt (spectrum.h:374-383)
__device__ __forceinline__ double sample_at(const DevEmit& em, double u, double& pdf) {
    int lo = 0, hi = em.n;
    while (lo + 1 < hi) { int mid = (lo + hi) / 2; if (em.cdf[mid] <= u) lo = mid; else hi = mid; }
    double c0 = em.cdf[lo], c1 = em.cdf[lo + 1];
    double frac = (c1 > c0) ? (u - c0) / (c1 - c0) : 0.5;
    pdf = (c1 - c0) / em.step;
    return LAMBDA_MIN + (lo + frac) * em.step;
}

// FTB_LAMBDA_UNIFORM_380_780 (no counterpart in the reference): lambda uniform over
// [380, 780) nm from the variate u, and the weight pdf_SPD(lambda) / (1/400 nm) with the
// emitter's binned SPD pdf, so the photon's power times the weight is unbiased for the band.
__device__ __forceinline__ double sample_uniform_band(const DevEmit& em, double u, double& weight) {
    const double lam = 380.0 + 400.0 * u;
    int b = (int)((lam - LAMBDA_MIN) / em.step);
    if (b < 0) b = 0;
    if (b > em.n - 1) b = em.n - 1;
    weight = (em.cdf[b + 1] - em.cdf[b]) / em.step * 400.0;
    return lam;
}

// ------------------------------------------------------------------ kernels ------------
template <bool MEDIA, bool STREAM, bool MIRROR>
__global__ void __launch_bounds__(128, FTB_EMIT_MINB) k_emit(Wave w, const DevJob* __restrict__ jobs, Frame f, PathState out,
                                              int32_t* out_count) {
    const int32_t n_jobs = w.params[0];
    const bool multi = n_jobs > 1;
    const PhotonSource src = photon_source<STREAM>(w, out_count);
    TallyAcc acc;
    tally_init(acc, multi, n_jobs);
    for (int64_t t = blockIdx.x * blockDim.x + threadIdx.x; t < src.n; t += gridDim.x * blockDim.x) {
        uint64_t k;
        const int j = photon_job<STREAM>(jobs, n_jobs, src, t, k);
        const DevJob& J = jobs[j];
        const DevScene& sc = J.sc;
        Pcg rng = seed_photon(k);
        if (sc.total_power <= 0.0 || sc.n_emit == 0) { log_emitted(w, k, 4, 0.0); continue; }
        const int ei = select_emitter(sc, rng);
        const DevEmit& em = sc.emit[ei];
        D3 origin, emit_n, dir;
        emit_sample(em, rng, origin, emit_n, dir);
        double pdf = 0.0, wl = 1.0;
        const double ul = uniform(rng);
        double lam;
        if (J.lambda_mode == FTB_LAMBDA_UNIFORM_380_780) {
            lam = sample_uniform_band(em, ul, wl);
            pdf = wl;
        } else {
            lam = sample_at(em, ul, pdf);
        }
        if (pdf <= 0) { log_emitted(w, k, 4, 0.0); continue; }
        double beta = (sc.n_emit == 1) ? em.power : sc.total_power;
        beta *= 1.0;
        if (J.lambda_mode == FTB_LAMBDA_UNIFORM_380_780) beta *= wl;
        tally_add(acc, jobs, multi, j, T_EMIT, to_fixed(beta, J.tally_scale_inv, f.status));
        const double cie[3] = {cie_x(lam), cie_y(lam), cie_z(lam)};
        connect_surface<MEDIA>(sc, J, w, f, j, origin, emit_n, emit_n, emit_n, lam, cie, beta, 1.0);
        if (MIRROR && sc.n_planes > 0) connect_mirrors(sc, J, w, f, j, origin, false, emit_n, 0.0, lam, cie, beta, 1.0);
        D3 ro = origin + dir * 1e-6;
        if (J.max_bounce <= 0) {
            tally_add(acc, jobs, multi, j, T_RES, to_fixed(beta, J.tally_scale_inv, f.status));
            log_emitted(w, k, 2, beta);
            continue;
        }
        const int o = photon_enqueue<STREAM>(w, out, out_count, src, j, multi, k);
        out.rng_s[o] = rng.s; out.rng_i[o] = rng.inc;
        out.ox[o] = ro.x; out.oy[o] = ro.y; out.oz[o] = ro.z;
        out.dx[o] = dir.x; out.dy[o] = dir.y; out.dz[o] = dir.z;
        out.lam[o] = lam; out.beta[o] = beta;
        out.cie[o] = cie[0]; out.cie[w.W + o] = cie[1]; out.cie[2 * (size_t)w.W + o] = cie[2];
        out.stk_n[o] = 0;
    }
    tally_finish(acc, jobs, multi, n_jobs);
}

__device__ void block_add3(unsigned long long* dst, unsigned long long a, unsigned long long b,
                           unsigned long long c) {
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0 && (a | b | c)) {
        atomicAdd(dst, a); atomicAdd(dst + 1, b); atomicAdd(dst + 2, c);
    }
}

__device__ void block_add1(unsigned long long* dst, unsigned long long a) {
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0 && a) atomicAdd(dst, a);
}


template <bool COUNT, bool INST, bool SHAPES>
__global__ void __launch_bounds__(128, FTB_TRAV_MINB) k_extend(Wave w, const DevJob* __restrict__ jobs,
                                                              PathState in, const int32_t* qcount,
                                                              const int32_t* __restrict__ order, Frame f) {
    const int32_t n_jobs = w.params[0];
    const int front = qcount[0], nq = queue_len(qcount);
    TravCount cnt{0, 0, 0};
    unsigned long long rays = 0;
    FTB_FOR_WARP_CHUNKS(q, nq, &w.counts[kFetchExtend]) {
        const int i = order ? order[q] : queue_entry(w, front, q);
        const DevScene& sc = jobs[n_jobs > 1 ? in.job[i] : 0].sc;
        RayCtx R = make_ray(mk(in.ox[i], in.oy[i], in.oz[i]), mk(in.dx[i], in.dy[i], in.dz[i]));
        double t;
        int sub = -1;
        int rec = traverse_closest<COUNT, INST, SHAPES>(sc, R, EPS_RAY, t, &sub, f.status, cnt);
        w.hit_t[i] = t;
        w.hit_rec[i] = rec;
        if (INST) w.hit_sub[i] = sub;
        if (COUNT) rays++;
    }
    if (COUNT) {
        block_add3(f.stats, rays, cnt.nodes, cnt.recs);
        block_add1(f.stats + 6, cnt.exact);
    }
}

// Optional reordering of a closest-hit queue by ray direction: pieces of kSortChunk entries
// are bucketed by an 8-bit direction key (an octahedral 16 x 16 grid in Morton order), so
// the lanes of a warp head the same way.  The order of rays does not change any result.
constexpr int kSortChunk = 1024;

__device__ __forceinline__ uint32_t direction_key(D3 d) {
    float x = (float)d.x, y = (float)d.y, z = (float)d.z;
    const float s = fabsf(x) + fabsf(y) + fabsf(z);
    x /= s; y /= s; z /= s;
    if (z < 0.0f) {   // fold the lower hemisphere onto the octahedron's outer triangles
        const float fx = (1.0f - fabsf(y)) * copysignf(1.0f, x);
        const float fy = (1.0f - fabsf(x)) * copysignf(1.0f, y);
        x = fx; y = fy;
    }
    uint32_t u = (uint32_t)min(15, max(0, (int)((x * 0.5f + 0.5f) * 16.0f)));
    uint32_t v = (uint32_t)min(15, max(0, (int)((y * 0.5f + 0.5f) * 16.0f)));
    u = (u | (u << 2)) & 0x33u; u = (u | (u << 1)) & 0x55u;   // 4-bit Morton interleave
    v = (v | (v << 2)) & 0x33u; v = (v | (v << 1)) & 0x55u;
    return u | (v << 1);
}

// Traversal order of a queue, each kSortChunk-position piece bucketed by direction key (one
// block per piece, counting sort in shared memory): order[q] is the entry of the path the
// closest-hit kernel's q-th lane takes, so a warp's 32 lanes head the same way.
__global__ void __launch_bounds__(128) k_sort_queue(Wave w, PathState in, const int32_t* qcount,
                                                    int32_t* order) {
    __shared__ int32_t hist[256];
    const int front = qcount[0], nq = queue_len(qcount);
    constexpr int kPer = kSortChunk / 128;
    for (int base = blockIdx.x * kSortChunk; base < nq; base += gridDim.x * kSortChunk) {
        for (int t = threadIdx.x; t < 256; t += 128) hist[t] = 0;
        __syncthreads();
        int pos[kPer], key[kPer], off[kPer];
#pragma unroll
        for (int r = 0; r < kPer; ++r) {
            const int p = base + r * 128 + threadIdx.x;
            const int i = p < nq ? queue_entry(w, front, p) : 0;
            pos[r] = p < nq ? i : -1;
            key[r] = pos[r] >= 0 ? (int)direction_key(mk(in.dx[i], in.dy[i], in.dz[i])) : 255;
            off[r] = pos[r] >= 0 ? atomicAdd(&hist[key[r]], 1) : 0;
        }
        __syncthreads();
        if (threadIdx.x < 32) {   // exclusive scan of the 256 bucket counts by one warp
            int v[8], run = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) { v[k] = hist[threadIdx.x * 8 + k]; run += v[k]; }
            int incl = run;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, incl, o);
                if ((int)threadIdx.x >= o) incl += y;
            }
            int acc = incl - run;
#pragma unroll
            for (int k = 0; k < 8; ++k) { hist[threadIdx.x * 8 + k] = acc; acc += v[k]; }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kPer; ++r)
            if (pos[r] >= 0) order[base + hist[key[r]] + off[r]] = pos[r];
        __syncthreads();   // before the next piece reuses the histogram
    }
}

struct Stk { int n; int2 e[kStkCap]; };
__device__ __forceinline__ int stk_top_pri(const Stk& s) {
    int bp = INT_MIN;
    for (int i = 0; i < s.n; ++i) if (s.e[i].y > bp) bp = s.e[i].y;
    return s.n ? bp : INT_MIN;
}
__device__ __forceinline__ int stk_top_mat(const Stk& s) {
    int bp = INT_MIN, bm = -1;
    for (int i = 0; i < s.n; ++i) if (s.e[i].y >= bp) { bp = s.e[i].y; bm = s.e[i].x; }
    return bm;
}
__device__ __forceinline__ void stk_push(Stk& s, int mi, int p, int32_t* status) {
    if (s.n < kStkCap) { s.e[s.n] = make_int2(mi, p); ++s.n; }
    else atomicOr(status, ST_MEDIUM_STACK);
}
__device__ __forceinline__ void stk_pop_mat(Stk& s, int mi) {
    for (int i = s.n - 1; i >= 0; --i)
        if (s.e[i].x == mi) {
            for (int j = i; j < s.n - 1; ++j) s.e[j] = s.e[j + 1];
            --s.n; return;
        }
}

__device__ __forceinline__ double mat_ior(const DevScene& sc, const DevMat& m, double lam) {
    return m.ior >= 0 ? spec_eval(sc, m.ior, lam) : 1.5;
}

// refractOrReflect, stochastic branch (render.h:2657-2697)
__device__ void refract_or_reflect(const DevScene& sc, const DevMat& m, const Hit& h, D3 d, double lam,
                                   Pcg& rng, bool& transmitted, double ext_ior, D3& o_out, D3& d_out) {
    double ngi = mat_ior(sc, m, lam);
    bool entering = dot(d, h.ng) < 0.0;
    D3 nl = entering ? h.ng : neg(h.ng);
    double n1 = entering ? ext_ior : ngi;
    double n2 = entering ? ngi : ext_ior;
    double eta = n1 / n2;
    double cos_i = -dot(d, nl);
    double sin2t = eta * eta * (1.0 - cos_i * cos_i);
    D3 out;
    bool refracted = false;
    if (sin2t > 1.0) out = reflect(d, nl);
    else {
        double cos_t = sqrt(1.0 - sin2t);
        double rs = (n1 * cos_i - n2 * cos_t) / (n1 * cos_i + n2 * cos_t);
        double rp = (n1 * cos_t - n2 * cos_i) / (n1 * cos_t + n2 * cos_i);
        double R = 0.5 * (rs * rs + rp * rp);
        if (uniform(rng) < R) out = reflect(d, nl);
        else { out = d * eta + nl * (eta * cos_i - cos_t); refracted = true; }
    }
    out = normalize(out);
    if (m.roughness > 1e-3) {
        D3 pert = sample_glossy(out, m.roughness, rng);
        bool ok = refracted ? (dot(pert, nl) < 0.0) : (dot(pert, nl) > 0.0);
        if (ok) out = pert;
    }
    transmitted = refracted;
    o_out = h.p + out * 1e-6;
    d_out = out;
}

// One bounce of Renderer::tracePhoton's loop body (render.h:2013-2238).
template <bool MEDIA, bool INST, bool SHAPES, bool MIRROR>
__global__ void __launch_bounds__(128, MEDIA ? FTB_SHADE_MEDIA_MINB : FTB_SHADE_MINB) k_shade(Wave w, const DevJob* __restrict__ jobs,
                                                               Frame f, PathState in, const int32_t* in_count,
                                                               PathState out, int32_t* out_count) {
    const int32_t n_jobs = w.params[0];
    const bool multi = n_jobs > 1;
    TallyAcc acc;
    tally_init(acc, multi, n_jobs);
    const int front = in_count[0], nq = queue_len(in_count);
    FTB_FOR_WARP_CHUNKS(q, nq, &w.counts[kFetchShade]) {
        const int i = queue_entry(w, front, q);
        const int j = multi ? in.job[i] : 0;
        const DevJob& J = jobs[j];
        const DevScene& sc = J.sc;
        Pcg rng; rng.s = in.rng_s[i]; rng.inc = in.rng_i[i];
        D3 ro = mk(in.ox[i], in.oy[i], in.oz[i]), rd = mk(in.dx[i], in.dy[i], in.dz[i]);
        double lam = in.lam[i], beta = in.beta[i];
        double cie[3];   // read by the paths that connect or survive
        bool have_cie = false;
        auto load_cie = [&]() {
            if (have_cie) return;
            cie[0] = in.cie[i]; cie[1] = in.cie[w.W + i]; cie[2] = in.cie[2 * (size_t)w.W + i];
            have_cie = true;
        };
        double ht = w.hit_t[i];
        int rec = w.hit_rec[i];
        Stk stk; stk.n = in.stk_n[i];
        for (int k = 0; k < stk.n; ++k) stk.e[k] = in.stk[k * w.W + i];
        log_hit<INST>(w, in, i, sc, rec);
        int fate = -1;   // -1 continue, 0 absorbed, 1 escaped
        bool costly = false;   // the next ray starts among curves: back end of the queue
        bool valid = rec >= 0;
        double d_surf = valid ? ht : 1e30;
        double d_event = d_surf;
        bool medium_event = false;
        int scatter_med = -1;
        D3 mp = mk(0, 0, 0);
        if (MEDIA && sc.n_med > 0) {
            double tm; int which;
            if (sample_media_collision(sc, ro, rd, d_surf, lam, rng, tm, which)) {
                d_event = tm; medium_event = true; scatter_med = which; mp = ro + rd * tm;
            }
        }
        {   // Beer-Lambert inside the current dielectric (render.h:2063-2066)
            int mi = stk_top_mat(stk);
            double a = (mi >= 0) ? spec_slot(sc, sc.mats[mi].absorb, lam, 0.0) : 0.0;
            if (a > 0.0) beta *= exp(-a * d_event);
        }
        D3 no = ro, nd = rd;
        if (medium_event) {   // render.h:2105-2115
            const DevMed& sm = sc.med[scatter_med];
            load_cie();
            connect_volume(sc, J, w, f, j, sm, mp, rd, lam, cie, beta);
            if (MIRROR && sc.n_planes > 0)
                connect_mirrors(sc, J, w, f, j, mp, true, rd, sm.g, lam, cie, beta, med_albedo(sc, sm, lam));
            if (uniform(rng) >= med_albedo(sc, sm, lam)) fate = 0;
            else { nd = sample_hg(rd, sm.g, rng); no = mp; }
        } else if (!valid) {
            fate = 1;
        } else {
            PrimRec r;
            load_rec(sc.recs, rec, r);
            if (SHAPES && rec_type(r) == REC_CURVE) costly = true;
            Hit h;
            if (INST && rec_type(r) == REC_INST) {
                instance_hit(sc.inst[rec_inst(r)], w.hit_sub[i], ro, rd, h);
                h.prim = r.prim;
            } else {
                RayCtx R = make_ray(ro, rd);
                hit_attributes<SHAPES>(sc.tri_n, R, r, h);
            }
            const DevMat& m = sc.mats[h.mat];
            switch (m.type) {
            case FTB_MAT_DIELECTRIC: {   // render.h:1612-1660
                bool entering = dot(rd, h.ng) < 0.0;
                int mi = h.mat, pr = m.priority;
                bool has_pri = pr != INT_MIN;
                bool transmitted = false;
                if (entering) {
                    int out_mat = stk_top_mat(stk), out_pri = stk_top_pri(stk);
                    bool ranked = has_pri && (stk.n == 0 || (out_mat >= 0 && sc.mats[out_mat].priority != INT_MIN));
                    if (ranked && stk.n != 0 && pr <= out_pri) {
                        stk_push(stk, mi, pr, f.status);
                        no = h.p + rd * 1e-6;
                    } else {
                        double ext = (ranked && out_mat >= 0) ? mat_ior(sc, sc.mats[out_mat], lam) : 1.0;
                        refract_or_reflect(sc, m, h, rd, lam, rng, transmitted, ext, no, nd);
                        if (transmitted) stk_push(stk, mi, pr, f.status);
                    }
                } else {
                    Stk after = stk;
                    stk_pop_mat(after, mi);
                    int new_mat = stk_top_mat(after), new_pri = stk_top_pri(after);
                    bool ranked = has_pri && (after.n == 0 || (new_mat >= 0 && sc.mats[new_mat].priority != INT_MIN));
                    if (ranked && new_mat >= 0 && pr <= new_pri) {
                        stk_pop_mat(stk, mi);
                        no = h.p + rd * 1e-6;
                    } else {
                        double ext = (ranked && new_mat >= 0) ? mat_ior(sc, sc.mats[new_mat], lam) : 1.0;
                        refract_or_reflect(sc, m, h, rd, lam, rng, transmitted, ext, no, nd);
                        if (transmitted) stk_pop_mat(stk, mi);
                    }
                }
                break;
            }
            case FTB_MAT_GLOSSY: {   // render.h:1725-1733
                double rr = clamp01(spec_slot(sc, m.reflect, lam, 0.5));
                if (uniform(rng) >= rr) { fate = 0; break; }
                D3 o = sample_glossy(reflect(rd, h.n), m.roughness, rng);
                if (dot(o, h.n) <= 0) { fate = 0; break; }
                no = h.p + h.n * 1e-6; nd = o;
                break;
            }
            case FTB_MAT_MIRROR: {   // render.h:1680-1688
                double rr = clamp01(spec_slot(sc, m.reflect, lam, 0.5));
                if (uniform(rng) >= rr) { fate = 0; break; }
                nd = reflect(rd, h.n);
                no = h.p + h.n * 1e-6;
                break;
            }
            case FTB_MAT_HALF_MIRROR: {   // render.h:1702-1711
                double rr = clamp01(spec_slot(sc, m.reflect, lam, 0.5));
                if (uniform(rng) < rr) {
                    nd = reflect(rd, h.n);
                    no = h.p + h.n * 1e-6;
                } else {
                    no = h.p + rd * 1e-6;
                }
                break;
            }
            case FTB_MAT_FILTER: {   // render.h:1711-1723
                double tt = clamp01(spec_slot(sc, m.transmit, lam, 0.0));
                if (uniform(rng) >= tt) { fate = 0; break; }
                no = h.p + rd * 1e-6;
                break;
            }
            case FTB_MAT_DIFFUSE_TRANSMIT: {   // render.h:2180-2212
                double rr = clamp01(spec_slot(sc, m.reflect, lam, 0.5));
                double rt = clamp01(spec_slot(sc, m.transmit, lam, 0.0));
                double sum = rr + rt;
                if (sum > 1.0) { rr /= sum; rt /= sum; sum = 1.0; }
                D3 ngo = oriented_geo_n(h);
                D3 wi = mk(-rd.x, -rd.y, -rd.z);
                load_cie();
                connect_surface<MEDIA>(sc, J, w, f, j, h.p, h.n, ngo, wi, lam, cie, beta, rr);
                connect_surface<MEDIA>(sc, J, w, f, j, h.p, neg(h.n), neg(ngo), wi, lam, cie, beta, rt);
                if (MIRROR && sc.n_planes > 0) {
                    connect_mirrors(sc, J, w, f, j, h.p, false, h.n, 0.0, lam, cie, beta, rr);
                    connect_mirrors(sc, J, w, f, j, h.p, false, neg(h.n), 0.0, lam, cie, beta, rt);
                }
                double u = uniform(rng);
                if (u < rr) {
                    D3 wo = cosine_hemisphere(h.n, rng);
                    beta *= shading_adjoint_corr(wi, wo, h.n, ngo);
                    no = h.p + h.n * 1e-6; nd = wo;
                } else if (u < sum) {
                    D3 wo = cosine_hemisphere(mk(-h.n.x, -h.n.y, -h.n.z), rng);
                    beta *= shading_adjoint_corr(wi, wo, h.n, ngo);
                    no = h.p - h.n * 1e-6; nd = wo;
                } else fate = 0;
                break;
            }
            default: {   // Diffuse (render.h:2215-2236)
                double rho = clamp01(spec_slot(sc, m.reflect, lam, 0.5));
                D3 ngo = oriented_geo_n(h);
                D3 wi = mk(-rd.x, -rd.y, -rd.z);
                load_cie();
                connect_surface<MEDIA>(sc, J, w, f, j, h.p, h.n, ngo, wi, lam, cie, beta, rho);
                if (MIRROR && sc.n_planes > 0) connect_mirrors(sc, J, w, f, j, h.p, false, h.n, 0.0, lam, cie, beta, rho);
                if (uniform(rng) >= rho) { fate = 0; break; }
                D3 wo = cosine_hemisphere(h.n, rng);
                beta *= shading_adjoint_corr(wi, wo, h.n, ngo);
                no = h.p + h.n * 1e-6; nd = wo;
                break;
            }
            }
        }
        if (fate == 0) {
            tally_add(acc, jobs, multi, j, T_ABS, to_fixed(beta, J.tally_scale_inv, f.status));
            log_finish(w, in, i, 0, beta);
            continue;
        }
        if (fate == 1) {
            tally_add(acc, jobs, multi, j, T_ESC, to_fixed(beta, J.tally_scale_inv, f.status));
            log_finish(w, in, i, 1, beta);
            continue;
        }
        const int32_t b = in.nbounce[i];
        if (b + 1 >= J.max_bounce) {
            tally_add(acc, jobs, multi, j, T_RES, to_fixed(beta, J.tally_scale_inv, f.status));
            log_finish(w, in, i, 2, beta);
            continue;
        }
        load_cie();
        const int o = (stk.n > 0 || costly) ? w.W - 1 - agg_inc(out_count + 1) : agg_inc(out_count);
        out.rng_s[o] = rng.s; out.rng_i[o] = rng.inc;
        out.ox[o] = no.x; out.oy[o] = no.y; out.oz[o] = no.z;
        out.dx[o] = nd.x; out.dy[o] = nd.y; out.dz[o] = nd.z;
        out.lam[o] = lam; out.beta[o] = beta;
        out.cie[o] = cie[0]; out.cie[w.W + o] = cie[1]; out.cie[2 * (size_t)w.W + o] = cie[2];
        out.stk_n[o] = stk.n;
        for (int k = 0; k < stk.n; ++k) out.stk[k * w.W + o] = stk.e[k];
        out.nbounce[o] = b + 1;
        if (multi) out.job[o] = j;
        log_move(w, in, i, out, o);
    }
    tally_finish(acc, jobs, multi, n_jobs);
}

__device__ __forceinline__ void splat(const DevJob& J, int view, int pix, double X, double Y, double Z,
                                      int32_t* status) {
    long long* px = reinterpret_cast<long long*>(view_film(J, view)) + 4 * (size_t)pix;
    atomicAdd(reinterpret_cast<unsigned long long*>(px), (unsigned long long)to_fixed(X, J.film_scale_inv, status));
    atomicAdd(reinterpret_cast<unsigned long long*>(px + 1), (unsigned long long)to_fixed(Y, J.film_scale_inv, status));
    atomicAdd(reinterpret_cast<unsigned long long*>(px + 2), (unsigned long long)to_fixed(Z, J.film_scale_inv, status));
    atomicAdd(reinterpret_cast<unsigned long long*>(px + 3), 1ull);
}

// A mirror record's tests, in connectSpecularPlane's order (render.h:1366-1379): the light
// leg p -> R, stopping short of the mirror, must be clear; a closest hit from the eye toward
// R must land on a planar mirror within 1e-4 (1 + dE) of R (mirrorSeenAt, render.h:
// 1294-1308).  On success: the mirror's material, the unfolded length D, the mirror point
// R, the leg R -> eye (wRE, dE) and the pixel's solid angle, recomputed from the record
// with the push's arithmetic.
struct MirrorSeen {
    int mat;
    double D, dE, omega;
    D3 R, wRE;
};
template <bool COUNT, bool INST, bool SHAPES>
__device__ __forceinline__ bool mirror_seen(const DevJob& J, const Wave& w, const Frame& f, int i, TravCount& cnt,
                                            MirrorSeen& ms) {
    const DevScene& sc = J.sc;
    const int view = w.sview[i] & 0xffff, plane = w.sview[i] >> 16;
    const DevPlane& mp = sc.planes[plane];
    const D3 pn = ld3(mp.n);
    const D3 p = mk(w.sox[i], w.soy[i], w.soz[i]), wP = mk(w.sdx[i], w.sdy[i], w.sdz[i]);
    const double dP = w.smax[i];
    {
        const RayCtx L = make_ray(p + wP * 1e-6, wP);
        if (traverse_any<COUNT, INST, SHAPES>(sc, L, EPS_RAY, (dP - 2e-6) - EPS_RAY, f.status, cnt)) return false;
    }
    const DevCam& cam = view_cam(J, view);
    const D3 eye = ld3(cam.eye);
    const double se = dot(pn, eye) - mp.d;
    const D3 eye_m = eye - pn * (2.0 * se);
    ms.D = len(eye_m - p);
    ms.R = p + wP * dP;
    ms.dE = ms.D - dP;
    ms.wRE = (eye - ms.R) * (1.0 / ms.dE);
    const D3 wE = neg(ms.wRE);
    double t;
    int sub = -1;
    const int rec = traverse_closest<COUNT, INST, SHAPES>(sc, make_ray(eye, wE), EPS_RAY, t, &sub, f.status, cnt);
    if (rec < 0) return false;
    if (fabs(t - ms.dE) > 1e-4 * (1.0 + ms.dE)) return false;
    PrimRec r;
    load_rec(sc.recs, rec, r);
    ms.mat = rec_mat(r);
    if (INST && rec_type(r) == REC_INST) {
        Hit h;
        instance_hit(sc.inst[rec_inst(r)], sub, eye, wE, h);
        ms.mat = h.mat;
    }
    if (ms.mat < 0 || ms.mat >= sc.n_mats || !planar_mirror(sc.mats[ms.mat])) return false;
    int px, py; double cos_cam, dist2e;
    cam_project(cam, ms.R, px, py, cos_cam, dist2e);
    ms.omega = cam_pixel_solid_angle(cam, cos_cam);
    return true;
}

// One-wavelength mirror record: splatMirrorLegs (render.h:1315-1331) with the reflectance of
// the mirror the eye sees: (beta * (weight * shape)) * refl / (D^2 Omega), times the two legs'
// transmittance in media.
template <bool COUNT, bool INST, bool SHAPES>
__device__ __noinline__ void mirror_splat(const DevJob& J, const Wave& w, const Frame& f, int i, TravCount& cnt) {
    MirrorSeen ms;
    if (!mirror_seen<COUNT, INST, SHAPES>(J, w, f, i, cnt, ms)) return;
    const DevScene& sc = J.sc;
    const double inv_d2_omega = 1.0 / (ms.D * ms.D * ms.omega);
    const double lam = w.slam[i];
    const double refl = clamp01(spec_slot(sc, sc.mats[ms.mat].reflect, lam, 0.5));
    double contrib = w.sval[i] * refl * inv_d2_omega;
    if (contrib <= 0.0) return;
    if (sc.n_med > 0) {
        const D3 p = mk(w.sox[i], w.soy[i], w.soz[i]), wP = mk(w.sdx[i], w.sdy[i], w.sdz[i]);
        contrib *= media_transmittance(sc, p, wP, w.smax[i], lam);
        contrib *= media_transmittance(sc, ms.R, ms.wRE, ms.dE, lam);
    }
    splat(J, w.sview[i] & 0xffff, ~w.spix[i], w.sxyz[i] * contrib, w.sxyz[w.S + i] * contrib,
          w.sxyz[2 * (size_t)w.S + i] * contrib, f.status);
}

// Camera connections: occlusion (Scene::occluded, default tmin 1e-6) then Film::add.
// MIRROR: the queue may also hold mirror connections (scenes with planar mirrors).
template <bool COUNT, bool INST, bool SHAPES, bool MIRROR>
__global__ void __launch_bounds__(128, FTB_TRAV_MINB) k_shadow(Wave w, const DevJob* __restrict__ jobs,
                                                              Frame f) {
    const int32_t n_jobs = w.params[0];
    int n = w.counts[kShadowCount];
    if (n > w.S) n = w.S;
    TravCount cnt{0, 0, 0};
    unsigned long long rays = 0;
    FTB_FOR_WARP_CHUNKS(i, n, &w.counts[kFetchShadow]) {
        const DevJob& J = jobs[n_jobs > 1 ? w.sjob[i] : 0];
        const DevScene& sc = J.sc;
        if (COUNT) rays++;
        if (MIRROR && w.spix[i] < 0) {
            mirror_splat<COUNT, INST, SHAPES>(J, w, f, i, cnt);
            continue;
        }
        D3 o = mk(w.sox[i], w.soy[i], w.soz[i]), d = mk(w.sdx[i], w.sdy[i], w.sdz[i]);
        double max_dist = w.smax[i];
        RayCtx R = make_ray(o, d);
        if (traverse_any<COUNT, INST, SHAPES>(sc, R, EPS_RAY, max_dist - EPS_RAY, f.status, cnt)) continue;
        splat(J, w.sview[i], w.spix[i], w.sxyz[i], w.sxyz[w.S + i], w.sxyz[2 * (size_t)w.S + i], f.status);
    }
    if (COUNT) {
        block_add3(f.stats + 3, rays, cnt.nodes, cnt.recs);
        block_add1(f.stats + 7, cnt.exact);
    }
}

// ------------------------------------------------------------------ hero bundles -------
// Hero-wavelength sampling (Renderer::tracePhotonHero / tracePhotonHeroLoop, render.h:
// 2252-2631; the policies of hero.h:28-70): a photon carries C wavelengths drawn from one
// stratified variate; the hero decides the geometry, analog Russian roulette uses the
// maximum over the live wavelengths with the bounded reweights booked as absorption, and a
// dielectric de-heroes (the hero goes on alone, its beta times C).  A camera connection
// tests occlusion once and splats every live wavelength.  The reference runs bundles only
// in scenes without media, and so does this path (the host sends such jobs to the scalar
// kernels).

__device__ __forceinline__ void push_shadow_hero(const Wave& w, const Frame& f, int job, int view, D3 o, D3 d,
                                                 double tmax, int nup, const double* lam, const double* val, int pix) {
    int i = agg_inc(&w.counts[kShadowCount]);
    if (i >= w.S) { atomicOr(f.status, ST_QUEUE_OVERFLOW); return; }
    w.sox[i] = o.x; w.soy[i] = o.y; w.soz[i] = o.z;
    w.sdx[i] = d.x; w.sdy[i] = d.y; w.sdz[i] = d.z;
    w.smax[i] = tmax; w.spix[i] = pix; w.sjob[i] = job; w.sview[i] = view;
    w.slam[i] = lam[0]; w.sval[i] = val[0];
    for (int k = 1; k < nup; ++k) {
        w.xlam[(size_t)(k - 1) * w.S + i] = lam[k];
        w.xval[(size_t)(k - 1) * w.S + i] = val[k];
    }
    w.snup[i] = nup;
}

// connectHero (render.h:564-577): one connectGeom, a contribution per live wavelength
__device__ void connect_surface_hero(const DevJob& J, const Wave& w, const Frame& f, int job, D3 p, D3 n,
                                     D3 ng, D3 wi, const double* lam, const double* beta, const double* rho,
                                     int nup) {
    for (int v = 0; v < view_count(J); ++v) {
        const DevCam& cam = view_cam(J, v);
        D3 to_cam = ld3(cam.eye) - p;
        double dist = len(to_cam);
        D3 wdir = to_cam / dist;
        double cos_surf = dot(n, wdir);
        if (cos_surf <= 0) continue;
        double stg = shadow_terminator_g(wdir, n, ng);
        if (stg <= 0.0) continue;
        int px, py; double cos_cam, dist2;
        if (!cam_project(cam, p, px, py, cos_cam, dist2)) continue;
        double omega = cam_pixel_solid_angle(cam, cos_cam);
        double corr = shading_adjoint_corr(wi, wdir, n, ng);
        double denom = dist2 * omega;
        double val[kHeroMax];
        for (int i = 0; i < nup; ++i) {
            double fr = rho[i] / PI_D;
            val[i] = beta[i] * fr * cos_surf * corr / denom * stg;
        }
        push_shadow_hero(w, f, job, v, p + ng * 1e-6, wdir, dist - 2e-6, nup, lam, val, py * cam.rx + px);
    }
}

__device__ __forceinline__ double sum_of(const double* a, int n) {   // activeSum (render.h:2324)
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += a[i];
    return s;
}
__device__ __forceinline__ double max_of(const double* a, int n) {   // hero::maxOf (hero.h:120-126)
    double m = a[0];
    for (int i = 1; i < n; ++i) if (a[i] > m) m = a[i];
    return m;
}

template <bool STREAM, bool MIRROR>
__global__ void __launch_bounds__(128, FTB_EMIT_MINB) k_emit_hero(Wave w, const DevJob* __restrict__ jobs, Frame f, PathState out,
                                                   int32_t* out_count) {
    const int32_t n_jobs = w.params[0];
    const bool multi = n_jobs > 1;
    const PhotonSource src = photon_source<STREAM>(w, out_count);
    TallyAcc acc;
    tally_init(acc, multi, n_jobs);
    for (int64_t t = blockIdx.x * blockDim.x + threadIdx.x; t < src.n; t += gridDim.x * blockDim.x) {
        uint64_t k;
        const int j = photon_job<STREAM>(jobs, n_jobs, src, t, k);
        const DevJob& J = jobs[j];
        const DevScene& sc = J.sc;
        const int C = J.hero_c;
        Pcg rng = seed_photon(k);
        if (sc.total_power <= 0.0 || sc.n_emit == 0) { log_emitted(w, k, 4, 0.0); continue; }
        const DevEmit& em = sc.emit[select_emitter(sc, rng)];
        D3 origin, emit_n, dir;
        emit_sample(em, rng, origin, emit_n, dir);
        // hero::sampleBundle (hero.h:100-113): one variate, strata u + i/C wrapped into [0,1)
        double lam[kHeroMax], beta[kHeroMax], one[kHeroMax], wl[kHeroMax];
        const bool band = J.lambda_mode == FTB_LAMBDA_UNIFORM_380_780;
        double u = uniform(rng), pdf;
        if (band) { lam[0] = sample_uniform_band(em, u, wl[0]); pdf = wl[0]; }
        else lam[0] = sample_at(em, u, pdf);
        if (pdf <= 0) { log_emitted(w, k, 4, 0.0); continue; }
        for (int i = 1; i < C; ++i) {
            double uu = u + (double)i / (double)C;
            if (uu >= 1.0) uu -= 1.0;
            double p2;
            if (band) lam[i] = sample_uniform_band(em, uu, wl[i]);
            else lam[i] = sample_at(em, uu, p2);
        }
        double base = (sc.n_emit == 1) ? em.power : sc.total_power;
        base *= 1.0;   // spotW
        for (int i = 0; i < C; ++i) {
            beta[i] = base / C;
            if (band) beta[i] *= wl[i];
            one[i] = 1.0;
        }
        tally_add(acc, jobs, multi, j, T_EMIT, to_fixed(sum_of(beta, C), J.tally_scale_inv, f.status));
        connect_surface_hero(J, w, f, j, origin, emit_n, emit_n, emit_n, lam, beta, one, C);
        if (MIRROR && sc.n_planes > 0) connect_mirrors_hero(sc, J, w, f, j, origin, emit_n, lam, beta, one, C);
        D3 ro = origin + dir * 1e-6;
        if (J.max_bounce <= 0) {
            tally_add(acc, jobs, multi, j, T_RES, to_fixed(sum_of(beta, C), J.tally_scale_inv, f.status));
            log_emitted(w, k, 2, beta[0]);
            continue;
        }
        const int o = photon_enqueue<STREAM>(w, out, out_count, src, j, multi, k);
        out.rng_s[o] = rng.s; out.rng_i[o] = rng.inc;
        out.ox[o] = ro.x; out.oy[o] = ro.y; out.oz[o] = ro.z;
        out.dx[o] = dir.x; out.dy[o] = dir.y; out.dz[o] = dir.z;
        for (int i = 0; i < C; ++i) {
            out.hlam[(size_t)i * w.W + o] = lam[i];
            out.hbeta[(size_t)i * w.W + o] = beta[i];
        }
        out.hlive[o] = C;
        out.stk_n[o] = 0;
    }
    tally_finish(acc, jobs, multi, n_jobs);
}

template <bool INST, bool SHAPES, bool MIRROR>
__global__ void __launch_bounds__(128, FTB_SHADE_MINB) k_shade_hero(Wave w, const DevJob* __restrict__ jobs,
                                                                    Frame f, PathState in, const int32_t* in_count,
                                                                    PathState out, int32_t* out_count) {
    const int32_t n_jobs = w.params[0];
    const bool multi = n_jobs > 1;
    TallyAcc acc;
    tally_init(acc, multi, n_jobs);
    const int front = in_count[0], nq = queue_len(in_count);
    FTB_FOR_WARP_CHUNKS(q, nq, &w.counts[kFetchShade]) {
        const int p = queue_entry(w, front, q);
        const int j = multi ? in.job[p] : 0;
        const DevJob& J = jobs[j];
        const DevScene& sc = J.sc;
        const int C = J.hero_c;
        Pcg rng; rng.s = in.rng_s[p]; rng.inc = in.rng_i[p];
        D3 ro = mk(in.ox[p], in.oy[p], in.oz[p]), rd = mk(in.dx[p], in.dy[p], in.dz[p]);
        int nup = in.hlive[p];
        double lam[kHeroMax], beta[kHeroMax];
        for (int k = 0; k < nup; ++k) {
            lam[k] = in.hlam[(size_t)k * w.W + p];
            beta[k] = in.hbeta[(size_t)k * w.W + p];
        }
        double ht = w.hit_t[p];
        int rec = w.hit_rec[p];
        Stk stk; stk.n = in.stk_n[p];
        for (int k = 0; k < stk.n; ++k) stk.e[k] = in.stk[k * w.W + p];
        log_hit<INST>(w, in, p, sc, rec);
        const bool valid = rec >= 0;
        const double d_event = valid ? ht : 1e30;
        {   // Beer-Lambert per live wavelength (render.h:2389-2398)
            int mi = stk_top_mat(stk);
            if (mi >= 0)
                for (int i = 0; i < nup; ++i) {
                    double a = spec_slot(sc, sc.mats[mi].absorb, lam[i], 0.0);
                    if (a > 0.0) beta[i] *= exp(-a * d_event);
                }
        }
        int fate = -1;   // -1 continue, 0 absorbed, 1 escaped
        bool costly = false;   // the next ray starts among curves: back end of the queue
        D3 no = ro, nd = rd;
        long long absorbed = 0;   // reweights booked as absorption (fixed point, per add)
        if (!valid) {
            fate = 1;
        } else {
            PrimRec r;
            load_rec(sc.recs, rec, r);
            if (SHAPES && rec_type(r) == REC_CURVE) costly = true;
            Hit h;
            if (INST && rec_type(r) == REC_INST) {
                instance_hit(sc.inst[rec_inst(r)], w.hit_sub[p], ro, rd, h);
                h.prim = r.prim;
            } else {
                RayCtx R = make_ray(ro, rd);
                hit_attributes<SHAPES>(sc.tri_n, R, r, h);
            }
            const DevMat& m = sc.mats[h.mat];
            switch (m.type) {
            case FTB_MAT_DIFFUSE_TRANSMIT: {   // render.h:2454-2503
                double rr[kHeroMax], rt[kHeroMax];
                for (int i = 0; i < nup; ++i) {
                    double a = clamp01(spec_slot(sc, m.reflect, lam[i], 0.5));
                    double b = clamp01(spec_slot(sc, m.transmit, lam[i], 0.0));
                    double s = a + b;
                    if (s > 1.0) { a /= s; b /= s; }
                    rr[i] = a; rt[i] = b;
                }
                D3 ngo = oriented_geo_n(h);
                D3 wi = mk(-rd.x, -rd.y, -rd.z);
                connect_surface_hero(J, w, f, j, h.p, h.n, ngo, wi, lam, beta, rr, nup);
                connect_surface_hero(J, w, f, j, h.p, neg(h.n), neg(ngo), wi, lam, beta, rt, nup);
                if (MIRROR && sc.n_planes > 0) {
                    connect_mirrors_hero(sc, J, w, f, j, h.p, h.n, lam, beta, rr, nup);
                    connect_mirrors_hero(sc, J, w, f, j, h.p, neg(h.n), lam, beta, rt, nup);
                }
                double q_r = max_of(rr, nup), q_t = max_of(rt, nup);
                double sum_h = q_r + q_t;
                if (nup > 1 && sum_h > 1.0) { q_r /= sum_h; q_t /= sum_h; sum_h = q_r + q_t; }
                double uu = uniform(rng);
                if (uu < q_r || uu < sum_h) {
                    const bool front = uu < q_r;
                    for (int i = 0; i < nup; ++i) {
                        double wgt = (front ? rr[i] : rt[i]) / (front ? q_r : q_t);
                        absorbed += to_fixed(beta[i] * (1.0 - wgt), J.tally_scale_inv, f.status);
                        beta[i] *= wgt;
                    }
                    D3 wo = cosine_hemisphere(front ? h.n : mk(-h.n.x, -h.n.y, -h.n.z), rng);
                    double corr = shading_adjoint_corr(wi, wo, h.n, ngo);
                    for (int i = 0; i < nup; ++i) beta[i] *= corr;
                    no = front ? h.p + h.n * 1e-6 : h.p - h.n * 1e-6;
                    nd = wo;
                } else {
                    fate = 0;
                }
                break;
            }
            case FTB_MAT_MIRROR:
            case FTB_MAT_FILTER:
            case FTB_MAT_GLOSSY: {   // achromatic lobes (render.h:2509-2537)
                double cc[kHeroMax];
                for (int i = 0; i < nup; ++i)
                    cc[i] = (m.type == FTB_MAT_FILTER) ? clamp01(spec_slot(sc, m.transmit, lam[i], 0.0))
                                                       : clamp01(spec_slot(sc, m.reflect, lam[i], 0.5));
                double q = max_of(cc, nup);
                if (uniform(rng) >= q) { fate = 0; break; }
                for (int i = 0; i < nup; ++i) {
                    double wgt = cc[i] / q;
                    absorbed += to_fixed(beta[i] * (1.0 - wgt), J.tally_scale_inv, f.status);
                    beta[i] *= wgt;
                }
                if (m.type == FTB_MAT_MIRROR) {
                    no = h.p + h.n * 1e-6; nd = reflect(rd, h.n);
                } else if (m.type == FTB_MAT_FILTER) {
                    no = h.p + rd * 1e-6;
                } else {
                    D3 o = sample_glossy(reflect(rd, h.n), m.roughness, rng);
                    if (dot(o, h.n) <= 0) { fate = 0; break; }
                    no = h.p + h.n * 1e-6; nd = o;
                }
                break;
            }
            case FTB_MAT_HALF_MIRROR: {   // de-hero, then the scalar half mirror (render.h:2546-2589, 1702-1711)
                if (nup > 1) { beta[0] *= (double)C; nup = 1; }
                const double rr = clamp01(spec_slot(sc, m.reflect, lam[0], 0.5));
                if (uniform(rng) < rr) {
                    nd = reflect(rd, h.n);
                    no = h.p + h.n * 1e-6;
                } else {
                    no = h.p + rd * 1e-6;
                }
                break;
            }
            case FTB_MAT_DIELECTRIC: {   // de-hero, then the scalar interaction (render.h:2539-2589)
                if (nup > 1) { beta[0] *= (double)C; nup = 1; }
                const double lam0 = lam[0];
                bool entering = dot(rd, h.ng) < 0.0;
                int mi = h.mat, pr = m.priority;
                bool has_pri = pr != INT_MIN;
                bool transmitted = false;
                if (entering) {
                    int out_mat = stk_top_mat(stk), out_pri = stk_top_pri(stk);
                    bool ranked = has_pri && (stk.n == 0 || (out_mat >= 0 && sc.mats[out_mat].priority != INT_MIN));
                    if (ranked && stk.n != 0 && pr <= out_pri) {
                        stk_push(stk, mi, pr, f.status);
                        no = h.p + rd * 1e-6;
                    } else {
                        double ext = (ranked && out_mat >= 0) ? mat_ior(sc, sc.mats[out_mat], lam0) : 1.0;
                        refract_or_reflect(sc, m, h, rd, lam0, rng, transmitted, ext, no, nd);
                        if (transmitted) stk_push(stk, mi, pr, f.status);
                    }
                } else {
                    Stk after = stk;
                    stk_pop_mat(after, mi);
                    int new_mat = stk_top_mat(after), new_pri = stk_top_pri(after);
                    bool ranked = has_pri && (after.n == 0 || (new_mat >= 0 && sc.mats[new_mat].priority != INT_MIN));
                    if (ranked && new_mat >= 0 && pr <= new_pri) {
                        stk_pop_mat(stk, mi);
                        no = h.p + rd * 1e-6;
                    } else {
                        double ext = (ranked && new_mat >= 0) ? mat_ior(sc, sc.mats[new_mat], lam0) : 1.0;
                        refract_or_reflect(sc, m, h, rd, lam0, rng, transmitted, ext, no, nd);
                        if (transmitted) stk_pop_mat(stk, mi);
                    }
                }
                break;
            }
            default: {   // Diffuse (render.h:2591-2625)
                double rho[kHeroMax];
                for (int i = 0; i < nup; ++i) rho[i] = clamp01(spec_slot(sc, m.reflect, lam[i], 0.5));
                D3 ngo = oriented_geo_n(h);
                D3 wi = mk(-rd.x, -rd.y, -rd.z);
                connect_surface_hero(J, w, f, j, h.p, h.n, ngo, wi, lam, beta, rho, nup);
                if (MIRROR && sc.n_planes > 0) connect_mirrors_hero(sc, J, w, f, j, h.p, h.n, lam, beta, rho, nup);
                double q = max_of(rho, nup);
                if (uniform(rng) >= q) { fate = 0; break; }
                for (int i = 0; i < nup; ++i) {
                    double wgt = rho[i] / q;
                    absorbed += to_fixed(beta[i] * (1.0 - wgt), J.tally_scale_inv, f.status);
                    beta[i] *= wgt;
                }
                D3 wo = cosine_hemisphere(h.n, rng);
                double corr = shading_adjoint_corr(wi, wo, h.n, ngo);
                for (int i = 0; i < nup; ++i) beta[i] *= corr;
                no = h.p + h.n * 1e-6; nd = wo;
                break;
            }
            }
        }
        if (absorbed) tally_add(acc, jobs, multi, j, T_ABS, absorbed);
        if (fate >= 0) {
            tally_add(acc, jobs, multi, j, fate == 0 ? T_ABS : T_ESC,
                      to_fixed(sum_of(beta, nup), J.tally_scale_inv, f.status));
            log_finish(w, in, p, fate, beta[0]);
            continue;
        }
        const int32_t b = in.nbounce[p];
        if (b + 1 >= J.max_bounce) {
            tally_add(acc, jobs, multi, j, T_RES, to_fixed(sum_of(beta, nup), J.tally_scale_inv, f.status));
            log_finish(w, in, p, 2, beta[0]);
            continue;
        }
        const int o = (stk.n > 0 || costly) ? w.W - 1 - agg_inc(out_count + 1) : agg_inc(out_count);
        out.rng_s[o] = rng.s; out.rng_i[o] = rng.inc;
        out.ox[o] = no.x; out.oy[o] = no.y; out.oz[o] = no.z;
        out.dx[o] = nd.x; out.dy[o] = nd.y; out.dz[o] = nd.z;
        for (int k = 0; k < nup; ++k) {
            out.hlam[(size_t)k * w.W + o] = lam[k];
            out.hbeta[(size_t)k * w.W + o] = beta[k];
        }
        out.hlive[o] = nup;
        out.stk_n[o] = stk.n;
        for (int k = 0; k < stk.n; ++k) out.stk[k * w.W + o] = stk.e[k];
        out.nbounce[o] = b + 1;
        if (multi) out.job[o] = j;
        log_move(w, in, p, out, o);
    }
    tally_finish(acc, jobs, multi, n_jobs);
}

// A bundle's mirror record: every live wavelength is its own splat with its own reflectance
// (splatMirrorLegs, render.h:1321-1330; bundles run without media); a wavelength whose
// contribution is not positive adds nothing, not even to the hit count.
template <bool COUNT, bool INST, bool SHAPES>
__device__ __noinline__ void mirror_splat_hero(const DevJob& J, const Wave& w, const Frame& f, int i, TravCount& cnt) {
    MirrorSeen ms;
    if (!mirror_seen<COUNT, INST, SHAPES>(J, w, f, i, cnt, ms)) return;
    const DevScene& sc = J.sc;
    const double inv_d2_omega = 1.0 / (ms.D * ms.D * ms.omega);
    const int nup = w.snup[i];
    long long sx = 0, sy = 0, sz = 0, hits = 0;
    for (int k = 0; k < nup; ++k) {
        const double lam = k == 0 ? w.slam[i] : w.xlam[(size_t)(k - 1) * w.S + i];
        const double a = k == 0 ? w.sval[i] : w.xval[(size_t)(k - 1) * w.S + i];
        const double refl = clamp01(spec_slot(sc, sc.mats[ms.mat].reflect, lam, 0.5));
        const double contrib = a * refl * inv_d2_omega;
        if (contrib <= 0.0) continue;
        sx += to_fixed(cie_x(lam) * contrib, J.film_scale_inv, f.status);
        sy += to_fixed(cie_y(lam) * contrib, J.film_scale_inv, f.status);
        sz += to_fixed(cie_z(lam) * contrib, J.film_scale_inv, f.status);
        ++hits;
    }
    if (!hits) return;
    long long* px = reinterpret_cast<long long*>(view_film(J, w.sview[i] & 0xffff)) + 4 * (size_t)~w.spix[i];
    atomicAdd(reinterpret_cast<unsigned long long*>(px), (unsigned long long)sx);
    atomicAdd(reinterpret_cast<unsigned long long*>(px + 1), (unsigned long long)sy);
    atomicAdd(reinterpret_cast<unsigned long long*>(px + 2), (unsigned long long)sz);
    atomicAdd(reinterpret_cast<unsigned long long*>(px + 3), (unsigned long long)hits);
}

// Connections of bundles: one occlusion test, then a splat per wavelength.  MIRROR: the queue
// may also hold mirror records (scenes with planar mirrors).
template <bool COUNT, bool INST, bool SHAPES, bool MIRROR>
__global__ void __launch_bounds__(128, FTB_TRAV_MINB) k_shadow_hero(Wave w, const DevJob* __restrict__ jobs,
                                                                   Frame f) {
    const int32_t n_jobs = w.params[0];
    int n = w.counts[kShadowCount];
    if (n > w.S) n = w.S;
    TravCount cnt{0, 0, 0};
    unsigned long long rays = 0;
    FTB_FOR_WARP_CHUNKS(i, n, &w.counts[kFetchShadow]) {
        const DevJob& J = jobs[n_jobs > 1 ? w.sjob[i] : 0];
        const DevScene& sc = J.sc;
        if (COUNT) rays++;
        if (MIRROR && w.spix[i] < 0) {
            mirror_splat_hero<COUNT, INST, SHAPES>(J, w, f, i, cnt);
            continue;
        }
        D3 o = mk(w.sox[i], w.soy[i], w.soz[i]), d = mk(w.sdx[i], w.sdy[i], w.sdz[i]);
        double max_dist = w.smax[i];
        RayCtx R = make_ray(o, d);
        if (traverse_any<COUNT, INST, SHAPES>(sc, R, EPS_RAY, max_dist - EPS_RAY, f.status, cnt)) continue;
        long long* px = reinterpret_cast<long long*>(view_film(J, w.sview[i])) + 4 * (size_t)w.spix[i];
        const int nup = w.snup[i];
        // every wavelength is one Film::add, each rounded to fixed point on its own; their
        // integer sum goes to the pixel in one atomic per channel (integer sums are exact)
        long long sx = 0, sy = 0, sz = 0;
        for (int k = 0; k < nup; ++k) {
            double lam = k == 0 ? w.slam[i] : w.xlam[(size_t)(k - 1) * w.S + i];
            double c = k == 0 ? w.sval[i] : w.xval[(size_t)(k - 1) * w.S + i];
            double X = cie_x(lam) * c, Y = cie_y(lam) * c, Z = cie_z(lam) * c;
            sx += to_fixed(X, J.film_scale_inv, f.status);
            sy += to_fixed(Y, J.film_scale_inv, f.status);
            sz += to_fixed(Z, J.film_scale_inv, f.status);
        }
        atomicAdd(reinterpret_cast<unsigned long long*>(px), (unsigned long long)sx);
        atomicAdd(reinterpret_cast<unsigned long long*>(px + 1), (unsigned long long)sy);
        atomicAdd(reinterpret_cast<unsigned long long*>(px + 2), (unsigned long long)sz);
        atomicAdd(reinterpret_cast<unsigned long long*>(px + 3), (unsigned long long)nup);
    }
    if (COUNT) {
        block_add3(f.stats + 3, rays, cnt.nodes, cnt.recs);
        block_add1(f.stats + 7, cnt.exact);
    }
}

// ------------------------------------------------------------------ host side ----------
void wave_carve(Wave& w, void* block, int32_t W, bool log, int32_t hero) {
    w = Wave{};
    w.W = W;
    w.S = kShadowPerSlot * W;
    w.hero = hero > 1 ? hero : 1;
    w.bytes = wave_bytes(W, log, hero);
    w.block = block;
    char* p = (char*)block;
    auto take = [&](size_t n) { void* r = p; p += wave_align(n); return r; };
    size_t wn = (size_t)W, sn = (size_t)w.S;
    for (PathState& ps : w.ps) {   // path_state_bytes order
        ps.rng_s = (uint64_t*)take(8 * wn); ps.rng_i = (uint64_t*)take(8 * wn);
        ps.ox = (double*)take(8 * wn); ps.oy = (double*)take(8 * wn); ps.oz = (double*)take(8 * wn);
        ps.dx = (double*)take(8 * wn); ps.dy = (double*)take(8 * wn); ps.dz = (double*)take(8 * wn);
        ps.lam = (double*)take(8 * wn); ps.beta = (double*)take(8 * wn); ps.cie = (double*)take(24 * wn);
        ps.stk_n = (int32_t*)take(4 * wn); ps.stk = (int2*)take(8 * wn * kStkCap);
        ps.nbounce = (int32_t*)take(4 * wn); ps.job = (int32_t*)take(4 * wn);
        if (hero > 1) {
            const size_t h = (size_t)hero;
            ps.hlam = (double*)take(8 * wn * h); ps.hbeta = (double*)take(8 * wn * h); ps.hlive = (int32_t*)take(4 * wn);
        }
        if (log) {
            ps.pid = (uint64_t*)take(8 * wn); ps.lhash = (uint64_t*)take(8 * wn);
            ps.lnh = (int32_t*)take(4 * wn); ps.lprims = (int32_t*)take(4 * wn * 8);
        }
    }
    w.hit_t = (double*)take(8 * wn); w.hit_rec = (int32_t*)take(4 * wn); w.hit_sub = (int32_t*)take(4 * wn);
    w.perm = (int32_t*)take(4 * wn);
    w.counts = (int32_t*)take(64);
    w.sjob = (int32_t*)take(4 * sn);
    w.jobs = (DevJob*)take(sizeof(DevJob) * kWaveJobs);
    w.params = (int32_t*)take(64);
    w.ctl = (StreamCtl*)take(64);
    w.sox = (double*)take(8 * sn); w.soy = (double*)take(8 * sn); w.soz = (double*)take(8 * sn);
    w.sdx = (double*)take(8 * sn); w.sdy = (double*)take(8 * sn); w.sdz = (double*)take(8 * sn);
    w.smax = (double*)take(8 * sn); w.sval = (double*)take(8 * sn); w.slam = (double*)take(8 * sn);
    w.sxyz = (double*)take(24 * sn);
    w.spix = (int32_t*)take(4 * sn);
    w.sview = (int32_t*)take(4 * sn);
    if (hero > 1) {
        const size_t h = (size_t)hero;
        w.xlam = (double*)take(8 * sn * (h - 1)); w.xval = (double*)take(8 * sn * (h - 1));
        w.snup = (int32_t*)take(4 * sn);
    }
}

cudaError_t wave_alloc(Wave& w, int32_t W, bool log, int32_t hero) {
    void* block = nullptr;
    cudaError_t e = cudaMalloc(&block, wave_bytes(W, log, hero));
    if (e != cudaSuccess) { w = Wave{}; return e; }
    wave_carve(w, block, W, log, hero);
    return cudaSuccess;
}

void wave_free(Wave& w) {
    if (w.block) cudaFree(w.block);
    w.block = nullptr;
}

// Streaming-pass bookkeeping: both queues and the connection queue empty, nothing handed out.
__global__ void k_stream_init(Wave w) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    StreamCtl& c = *w.ctl;
    c.next = 0; c.taken = 0; c.half = 0; c.more = 1;
    for (int k = 0; k < 16; ++k) w.counts[k] = 0;
}

// End of a half-iteration (one thread): the refill's photons are booked and its paths join
// the queue for the next half-iteration, the consumed queue and the connection queue are
// emptied, and whether work is left -- paths queued or photons not yet handed out -- goes to
// the progress word and, inside a graph, to the loop condition.  A pass that reaches its
// half-iteration cap with work left stops with ST_LOOP_CAP.
__global__ void k_stream_advance(Wave w, Frame f, int32_t* consumed, int32_t* next_q,
                                 cudaGraphConditionalHandle loop, int32_t set_loop) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    StreamCtl& c = *w.ctl;
    const int64_t total = reinterpret_cast<const int64_t*>(w.params)[1];
    const int64_t cap = reinterpret_cast<const int64_t*>(w.params)[2];
    const int32_t have = next_q[0];   // survivors at the front; the refill filled the room above them
    const int64_t room = (int64_t)w.params[1] - have - next_q[1], left = total - c.next;
    c.next += left < room ? left : room;
    next_q[0] = have + c.taken;
    c.taken = 0;
    c.half += 1;
    consumed[0] = 0;
    consumed[1] = 0;
    w.counts[kShadowCount] = 0;
    w.counts[kFetchExtend] = 0;
    w.counts[kFetchShade] = 0;
    w.counts[kFetchShadow] = 0;
    int32_t more = (queue_len(next_q) > 0 || c.next < total) ? 1 : 0;
    if (more && c.half >= cap) {
        atomicOr(f.status, ST_LOOP_CAP);
        more = 0;
    }
    c.more = more;
    if (set_loop) cudaGraphSetConditional(loop, (unsigned)more);
}

// Launchers of the traversal kernels' variants (template template arguments of Issue::trav).
template <bool C, bool I, bool S>
struct LaunchExtend {
    static void go(int grid, cudaStream_t st, Wave w, const DevJob* jobs, PathState in, const int32_t* c,
                   const int32_t* order, Frame f) {
        k_extend<C, I, S><<<grid, 128, 0, st>>>(w, jobs, in, c, order, f);
    }
};
template <bool C, bool I, bool S>
struct LaunchShadow {
    static void go(int grid, cudaStream_t st, Wave w, const DevJob* jobs, Frame f) {
        k_shadow<C, I, S, false><<<grid, 128, 0, st>>>(w, jobs, f);
    }
};
template <bool C, bool I, bool S>
struct LaunchShadowMirror {
    static void go(int grid, cudaStream_t st, Wave w, const DevJob* jobs, Frame f) {
        k_shadow<C, I, S, true><<<grid, 128, 0, st>>>(w, jobs, f);
    }
};
template <bool C, bool I, bool S>
struct LaunchShadowHero {
    static void go(int grid, cudaStream_t st, Wave w, const DevJob* jobs, Frame f) {
        k_shadow_hero<C, I, S, false><<<grid, 128, 0, st>>>(w, jobs, f);
    }
};
template <bool C, bool I, bool S>
struct LaunchShadowHeroMirror {
    static void go(int grid, cudaStream_t st, Wave w, const DevJob* jobs, Frame f) {
        k_shadow_hero<C, I, S, true><<<grid, 128, 0, st>>>(w, jobs, f);
    }
};

namespace {
// Kernel launches of one wave buffer with the variants its WaveKind selects.
struct Issue {
    Wave& w;
    const WaveKind& kind;
    const Frame& f;
    int grid;
    bool sorted;
    cudaStream_t st;
    LaunchSink* sink;
    static constexpr int T = 128;

    void mark(int k, bool end) { if (sink) sink->mark(k, end, st); }
    void emit(bool stream, const PathState& out, int32_t* co) {
        mark(K_EMIT, false);
        const DevJob* jobs = w.jobs;
#define FTB_EMIT_HERO(S) \
    (kind.mirrors ? k_emit_hero<S, true><<<grid, T, 0, st>>>(w, jobs, f, out, co) \
                  : k_emit_hero<S, false><<<grid, T, 0, st>>>(w, jobs, f, out, co))
#define FTB_EMIT(M, S) \
    (kind.mirrors ? k_emit<M, S, true><<<grid, T, 0, st>>>(w, jobs, f, out, co) \
                  : k_emit<M, S, false><<<grid, T, 0, st>>>(w, jobs, f, out, co))
        if (stream) {
            if (kind.bundles) FTB_EMIT_HERO(true);
            else if (kind.media) FTB_EMIT(true, true);
            else FTB_EMIT(false, true);
        } else {
            if (kind.bundles) FTB_EMIT_HERO(false);
            else if (kind.media) FTB_EMIT(true, false);
            else FTB_EMIT(false, false);
        }
#undef FTB_EMIT
#undef FTB_EMIT_HERO
        mark(K_EMIT, true);
    }
    template <template <bool, bool, bool> class K, class... A>
    void trav(A... args) {   // a traversal kernel with the counting / instance / shape variant
        const bool count = f.stats != nullptr, inst = kind.instances, shp = kind.shapes;
        if (count) {
            if (inst) { if (shp) K<true, true, true>::go(grid, st, args...); else K<true, true, false>::go(grid, st, args...); }
            else { if (shp) K<true, false, true>::go(grid, st, args...); else K<true, false, false>::go(grid, st, args...); }
        } else {
            if (inst) { if (shp) K<false, true, true>::go(grid, st, args...); else K<false, true, false>::go(grid, st, args...); }
            else { if (shp) K<false, false, true>::go(grid, st, args...); else K<false, false, false>::go(grid, st, args...); }
        }
    }
    void shadow() {
        mark(K_SHADOW, false);
        if (kind.bundles && kind.mirrors) trav<LaunchShadowHeroMirror>(w, (const DevJob*)w.jobs, f);
        else if (kind.bundles) trav<LaunchShadowHero>(w, (const DevJob*)w.jobs, f);
        else if (kind.mirrors) trav<LaunchShadowMirror>(w, (const DevJob*)w.jobs, f);
        else trav<LaunchShadow>(w, (const DevJob*)w.jobs, f);
        mark(K_SHADOW, true);
    }
    void extend(const PathState& in, int32_t* c) {
        mark(K_EXTEND, false);
        const int32_t* order = nullptr;
        if (sorted) {
            const int gs = std::max(1, std::min(grid, (w.W + kSortChunk - 1) / kSortChunk));
            k_sort_queue<<<gs, T, 0, st>>>(w, in, c, w.perm);
            order = w.perm;
        }
        trav<LaunchExtend>(w, (const DevJob*)w.jobs, in, (const int32_t*)c, order, f);
        mark(K_EXTEND, true);
    }
    void shade(const PathState& in, const int32_t* ci, const PathState& out, int32_t* co) {
        const bool inst = kind.instances, shp = kind.shapes;
        const DevJob* jobs = w.jobs;
        mark(K_SHADE, false);
#define FTB_SHADE(...) __VA_ARGS__<<<grid, T, 0, st>>>(w, jobs, f, in, ci, out, co)
        if (kind.bundles && kind.mirrors) {
            if (inst) { if (shp) FTB_SHADE(k_shade_hero<true, true, true>); else FTB_SHADE(k_shade_hero<true, false, true>); }
            else { if (shp) FTB_SHADE(k_shade_hero<false, true, true>); else FTB_SHADE(k_shade_hero<false, false, true>); }
        } else if (kind.bundles) {
            if (inst) { if (shp) FTB_SHADE(k_shade_hero<true, true, false>); else FTB_SHADE(k_shade_hero<true, false, false>); }
            else { if (shp) FTB_SHADE(k_shade_hero<false, true, false>); else FTB_SHADE(k_shade_hero<false, false, false>); }
        } else if (kind.mirrors) {
            if (kind.media) {
                if (inst) { if (shp) FTB_SHADE(k_shade<true, true, true, true>); else FTB_SHADE(k_shade<true, true, false, true>); }
                else { if (shp) FTB_SHADE(k_shade<true, false, true, true>); else FTB_SHADE(k_shade<true, false, false, true>); }
            } else {
                if (inst) { if (shp) FTB_SHADE(k_shade<false, true, true, true>); else FTB_SHADE(k_shade<false, true, false, true>); }
                else { if (shp) FTB_SHADE(k_shade<false, false, true, true>); else FTB_SHADE(k_shade<false, false, false, true>); }
            }
        } else if (kind.media) {
            if (inst) { if (shp) FTB_SHADE(k_shade<true, true, true, false>); else FTB_SHADE(k_shade<true, true, false, false>); }
            else { if (shp) FTB_SHADE(k_shade<true, false, true, false>); else FTB_SHADE(k_shade<true, false, false, false>); }
        } else {
            if (inst) { if (shp) FTB_SHADE(k_shade<false, true, true, false>); else FTB_SHADE(k_shade<false, true, false, false>); }
            else { if (shp) FTB_SHADE(k_shade<false, false, true, false>); else FTB_SHADE(k_shade<false, false, false, false>); }
        }
#undef FTB_SHADE
        mark(K_SHADE, true);
    }
};

// The launch sequence of one wave: emit, its connections, then per bounce closest hit,
// shading (survivors compacted into the other path buffer) and the connections it queued.
// Every launch reads the wave's job count and slot count from w.params, so the same
// sequence serves any table (and one captured graph serves every wave of its shape).
void issue_wave(Issue& I, int32_t max_bounce) {
    Wave& w = I.w;
    cudaStream_t st = I.st;
    cudaMemsetAsync(w.counts, 0, 64, st);
    I.emit(false, w.ps[0], queue_counts(w, 0));
    I.shadow();
    cudaMemsetAsync(&w.counts[kShadowCount], 0, 4 * kCountWords, st);
    for (int b = 0; b < max_bounce; ++b) {
        const int a = b & 1;
        I.extend(w.ps[a], queue_counts(w, a));
        cudaMemsetAsync(queue_counts(w, a ^ 1), 0, 8, st);
        I.shade(w.ps[a], queue_counts(w, a), w.ps[a ^ 1], queue_counts(w, a ^ 1));
        I.shadow();
        cudaMemsetAsync(&w.counts[kShadowCount], 0, 4 * kCountWords, st);
    }
}

// A streaming pass: the prologue fills the first queue (ps[0]) and traces its emission
// connections; a half-iteration traces queue `a` and leaves the next one in queue a ^ 1
// (the survivors of shading, then the refill).
void stream_prologue(Issue& I) {
    Wave& w = I.w;
    k_stream_init<<<1, 32, 0, I.st>>>(w);
    I.emit(true, w.ps[0], queue_counts(w, 0));
    I.shadow();
    k_stream_advance<<<1, 32, 0, I.st>>>(w, I.f, queue_counts(w, 1), queue_counts(w, 0), 0, 0);
}
void stream_half(Issue& I, int a, cudaGraphConditionalHandle loop, int32_t set_loop) {
    Wave& w = I.w;
    I.extend(w.ps[a], queue_counts(w, a));
    I.shade(w.ps[a], queue_counts(w, a), w.ps[a ^ 1], queue_counts(w, a ^ 1));
    I.emit(true, w.ps[a ^ 1], queue_counts(w, a ^ 1));
    I.shadow();
    k_stream_advance<<<1, 32, 0, I.st>>>(w, I.f, queue_counts(w, a), queue_counts(w, a ^ 1), loop, set_loop);
}
}  // namespace

struct WaveGraphs {
    struct Entry {
        int32_t max_bounce, grid;   // max_bounce -1: a streaming pass
        bool inst, hero, media, shapes, mirrors, sorted;
        int32_t* status;
        cudaGraphExec_t exec;
    };
    std::vector<Entry> entries;
    ~WaveGraphs() {
        for (auto& e : entries) cudaGraphExecDestroy(e.exec);
    }
    cudaGraphExec_t find(int32_t max_bounce, int32_t grid, const WaveKind& kind, bool sorted, int32_t* status) const {
        for (auto& e : entries)
            if (e.max_bounce == max_bounce && e.grid == grid && e.inst == kind.instances && e.hero == kind.bundles &&
                e.media == kind.media && e.shapes == kind.shapes && e.mirrors == kind.mirrors && e.sorted == sorted &&
                e.status == status)
                return e.exec;
        return nullptr;
    }
};

WaveGraphs* wave_graphs_create() { return new WaveGraphs(); }
void wave_graphs_destroy(WaveGraphs* g) { delete g; }

namespace {
int launch_grid(const Wave& w, int32_t sms, const LaunchShape& shape) {
    const int T = Issue::T;
    int grid = sms * std::max(1, shape.grid_mult);
    const int gw = (w.W + T - 1) / T;   // enough blocks to give every slot a thread
    if (gw < grid) grid = gw < 1 ? 1 : gw;
    return grid;
}
}  // namespace

cudaError_t launch_wave(Wave& w, int32_t max_bounce, const WaveKind& kind, const Frame& f, int32_t sms,
                        const LaunchShape& shape, cudaStream_t st, LaunchSink* sink, WaveGraphs* graphs) {
    if (kind.bundles && w.hero < 2) return cudaErrorInvalidValue;   // the buffer carries no bundles
    const int grid = launch_grid(w, sms, shape);
    // A graph bakes the kernel arguments: the wave's buffers and status word are fixed for the
    // life of its cache, but a log buffer changes per call, so logging waves launch directly.
    if (!(shape.graph && graphs) || sink || f.stats || w.logs) {
        Issue I{w, kind, f, grid, shape.sort_rays, st, sink};
        issue_wave(I, max_bounce);
        return cudaGetLastError();
    }
    if (cudaGraphExec_t ex = graphs->find(max_bounce, grid, kind, shape.sort_rays, f.status))
        return cudaGraphLaunch(ex, st);
    cudaGraph_t g = nullptr;
    cudaError_t err = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (err != cudaSuccess) return err;
    Issue I{w, kind, f, grid, shape.sort_rays, st, nullptr};
    issue_wave(I, max_bounce);
    err = cudaStreamEndCapture(st, &g);
    if (err != cudaSuccess) return err;
    WaveGraphs::Entry e{max_bounce, grid, kind.instances, kind.bundles, kind.media, kind.shapes, kind.mirrors,
                        shape.sort_rays, f.status, nullptr};
    err = cudaGraphInstantiate(&e.exec, g, 0);
    cudaGraphDestroy(g);
    if (err != cudaSuccess) return err;
    graphs->entries.push_back(e);
    return cudaGraphLaunch(e.exec, st);
}

cudaError_t launch_stream(Wave& w, const WaveKind& kind, const Frame& f, int32_t sms, const LaunchShape& shape,
                          cudaStream_t st, LaunchSink* sink, WaveGraphs* graphs) {
    if (kind.bundles && w.hero < 2) return cudaErrorInvalidValue;
    const int grid = launch_grid(w, sms, shape);
    if (!(shape.graph && graphs) || sink || f.stats || w.logs) {
        // host-driven: the graph's loop body (two half-iterations) at a time, the progress
        // word read after each, so the launches are the ones a graph replay makes
        Issue I{w, kind, f, grid, shape.sort_rays, st, sink};
        stream_prologue(I);
        for (;;) {
            stream_half(I, 0, 0, 0);
            stream_half(I, 1, 0, 0);
            cudaError_t e = cudaGetLastError();
            int32_t more = 0;
            if (e == cudaSuccess) e = cudaMemcpyAsync(&more, &w.ctl->more, sizeof more, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return e;
            if (!more) return cudaSuccess;
        }
    }
    if (cudaGraphExec_t ex = graphs->find(-1, grid, kind, shape.sort_rays, f.status)) return cudaGraphLaunch(ex, st);
    // prologue, then a conditional while node whose body is two half-iterations (the queues
    // swap roles between them); the last advance of the body sets the loop condition
    Issue I{w, kind, f, grid, shape.sort_rays, st, nullptr};
    cudaGraph_t g = nullptr;
    cudaError_t err = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (err != cudaSuccess) return err;
    stream_prologue(I);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t n_deps = 0;
    cudaGraphConditionalHandle loop = 0;
    cudaGraphNode_t node = nullptr;
    cudaGraphNodeParams p{};
    err = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &n_deps);
    if (err == cudaSuccess) err = cudaGraphConditionalHandleCreate(&loop, g, 1, cudaGraphCondAssignDefault);
    if (err == cudaSuccess) {
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = loop;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        err = cudaGraphAddNode(&node, g, deps, n_deps, &p);
    }
    if (err == cudaSuccess) err = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
    cudaGraph_t captured = nullptr;
    cudaError_t end = cudaStreamEndCapture(st, &captured);
    if (err == cudaSuccess) err = end;
    if (err != cudaSuccess) {
        if (captured) cudaGraphDestroy(captured);
        return err;
    }
    cudaGraph_t body = p.conditional.phGraph_out[0];
    err = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (err == cudaSuccess) {
        stream_half(I, 0, loop, 0);
        stream_half(I, 1, loop, 1);
        cudaGraph_t b2 = nullptr;
        err = cudaStreamEndCapture(st, &b2);
    }
    WaveGraphs::Entry e{-1, grid, kind.instances, kind.bundles, kind.media, kind.shapes, kind.mirrors,
                        shape.sort_rays, f.status, nullptr};
    if (err == cudaSuccess) err = cudaGraphInstantiate(&e.exec, captured, 0);
    cudaGraphDestroy(captured);
    if (err != cudaSuccess) return err;
    graphs->entries.push_back(e);
    return cudaGraphLaunch(e.exec, st);
}

}  // namespace ftb
