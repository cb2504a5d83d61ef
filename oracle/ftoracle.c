/*
 * ftoracle.c -- CPU ORACLE for parity tests.  TEST INFRASTRUCTURE ONLY (see ftoracle.h).
 *
 * Plain-C restatement of the reference forward light tracer, one wavelength per photon,
 * pinhole camera (model B).  Every function names the reference code it restates
 * (file:line relative to the reference's src/).  Arithmetic is written in the same order
 * as the reference's C++ so that, compiled without FMA contraction (the x86-64 baseline
 * has no FMA; the Makefile passes -ffp-contract=off anyway), it produces bit-identical
 * doubles.  Only the acceleration structure differs from the reference: closest-hit
 * results do not depend on it except for exact ties in t.
 */
#include "ftoracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static __thread char g_err[256];
const char* fto_last_error(void) { return g_err; }
static int fail(const char* m) { snprintf(g_err, sizeof g_err, "%s", m); return -1; }

/* ---------------------------------------------------------------- linalg.h:57-91 ---- */
typedef struct { double x, y, z; } V3;
static inline V3 v3(double x, double y, double z) { V3 r = {x, y, z}; return r; }
static inline V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 vmul(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 vdiv(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
static inline V3 vneg(V3 a) { return v3(-a.x, -a.y, -a.z); }
static inline double vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 vcross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline double vlen(V3 a) { return sqrt(vdot(a, a)); }
static inline V3 vnorm(V3 a) { return vdiv(a, vlen(a)); }
static inline double vget(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
/* reflect (linalg.h:82) */
static inline V3 vreflect(V3 d, V3 n) { return vsub(d, vmul(n, 2.0 * vdot(d, n))); }
/* onb, Duff et al. (linalg.h:85-91) */
static inline void onb(V3 n, V3* t, V3* b) {
    double sign = copysign(1.0, n.z);
    double a = -1.0 / (sign + n.z);
    double d = n.x * n.y * a;
    *t = v3(1.0 + sign * n.x * n.x * a, sign * d, -sign * n.x);
    *b = v3(d, sign + n.y * n.y * a, -n.y);
}

#define PI_D 3.141592653589793
#define LAMBDA_MIN 360.0
#define LAMBDA_MAX 830.0

/* ---------------------------------------------------------------- rng.h:6-52 -------- */
typedef struct { uint64_t state, inc; } Pcg;
static inline uint32_t pcg_next(Pcg* r) {
    uint64_t old = r->state;
    r->state = old * 6364136223846793005ULL + r->inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((~rot + 1u) & 31));
}
static inline void pcg_seed(Pcg* r, uint64_t seq, uint64_t s) {
    r->state = 0; r->inc = (seq << 1u) | 1u;
    pcg_next(r); r->state += s; pcg_next(r);
}
static inline double pcg_uniform(Pcg* r) { return (pcg_next(r) >> 8) * (1.0 / 16777216.0); }
static inline uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
static inline void seed_unit(Pcg* r, uint64_t k, uint64_t salt) {
    pcg_seed(r, mix64(k ^ salt), mix64(k + salt));
}
#define PHOTON_SALT 0x9E3779B97F4A7C15ULL /* main.cpp:11326 */

void fto_uniforms(uint64_t k, int count, double* out) {
    Pcg r; seed_unit(&r, k, PHOTON_SALT);
    for (int i = 0; i < count; ++i) out[i] = pcg_uniform(&r);
}

/* cosineHemisphere (rng.h:45-52) */
static V3 cosine_hemisphere(V3 n, Pcg* rng) {
    double u1 = pcg_uniform(rng), u2 = pcg_uniform(rng);
    double r = sqrt(u1);
    double phi = 6.283185307179586 * u2;
    double lx = r * cos(phi), ly = r * sin(phi), lz = sqrt(1.0 - u1);
    V3 t, b; onb(n, &t, &b);
    return vnorm(vadd(vadd(vmul(t, lx), vmul(b, ly)), vmul(n, lz)));
}

/* ------------------------------------------------------------- spectrum.h ----------- */
typedef struct {
    const ftb_spectrum* spec;
    const double* tw;
    const double* tv;
    int nspec;
} SpecSet;

/* blackbodyRadiance (spectrum.h:185-190) */
static double blackbody_radiance(double kelvin, double lambda_nm) {
    const double h = 6.62607015e-34, c = 2.99792458e8, kb = 1.380649e-23;
    double l = lambda_nm * 1e-9;
    double e = exp((h * c) / (l * kb * kelvin)) - 1.0;
    return (2.0 * h * c * c) / (pow(l, 5.0) * e);
}

static double spec_eval(const SpecSet* S, int idx, double w) {
    const ftb_spectrum* s = &S->spec[idx];
    switch (s->kind) {
    case FTB_SPEC_CONST: return s->p[0];                       /* spectrum.h:179 */
    case FTB_SPEC_TABLE: {                                     /* spectrum.h:264-281 */
        const double* x = S->tw + s->offset;
        const double* y = S->tv + s->offset;
        int n = s->n;
        if (n <= 0) return 0.0;
        if (w <= x[0]) return y[0];
        if (w >= x[n - 1]) return y[n - 1];
        size_t lo = 0, hi = (size_t)n - 1;
        while (lo + 1 < hi) {
            size_t mid = (lo + hi) / 2;
            if (x[mid] <= w) lo = mid; else hi = mid;
        }
        double w0 = x[lo], w1 = x[lo + 1], v0 = y[lo], v1 = y[lo + 1];
        double f = (w1 > w0) ? (w - w0) / (w1 - w0) : 0.0;
        return v0 + (v1 - v0) * f;
    }
    case FTB_SPEC_CAUCHY: {                                    /* spectrum.h:243-248 */
        double um = w * 1e-3;
        return s->p[0] + s->p[1] / (um * um);
    }
    case FTB_SPEC_SELLMEIER: {                                 /* spectrum.h:233-239 */
        double l2 = (w * 1e-3) * (w * 1e-3);
        double n2 = 1.0 + s->p[0] * l2 / (l2 - s->p[3]) + s->p[1] * l2 / (l2 - s->p[4]) +
                    s->p[2] * l2 / (l2 - s->p[5]);
        return sqrt(n2 > 1.0 ? n2 : 1.0);
    }
    case FTB_SPEC_BLACKBODY:                                   /* spectrum.h:192-195 */
        return blackbody_radiance(s->p[0], w) * s->p[1];
    default: return 0.0;
    }
}

static int spec_ok(const ftb_scene_desc* d, int idx) {
    if (idx < 0 || idx >= d->n_spectra) return 0;
    const ftb_spectrum* s = &d->spectra[idx];
    if (s->kind < 0 || s->kind > FTB_SPEC_BLACKBODY) return 0;
    if (s->kind == FTB_SPEC_TABLE) {
        if (s->n <= 0 || s->offset < 0 || s->offset + s->n > d->n_table) return 0;
        if (!d->table_w || !d->table_v) return 0;
    }
    return 1;
}

double fto_spectrum_eval(const ftb_scene_desc* d, int spec, double lambda_nm) {
    if (!d || !spec_ok(d, spec)) return NAN;
    SpecSet S = {d->spectra, d->table_w, d->table_v, d->n_spectra};
    return spec_eval(&S, spec, lambda_nm);
}

/* EmissionSampler::build (spectrum.h:357-369) */
static int emission_build(const SpecSet* S, int spec, double step, double* cdf, int cap,
                          double* integral) {
    int n = (int)((LAMBDA_MAX - LAMBDA_MIN) / step);
    if (n < 1 || n + 1 > cap) return -1;
    for (int i = 0; i <= n; ++i) cdf[i] = 0.0;
    double acc = 0.0;
    for (int i = 0; i < n; ++i) {
        double w = LAMBDA_MIN + (i + 0.5) * step;
        double v = spec_eval(S, spec, w);
        acc += (v > 0.0 ? v : 0.0) * step;   /* std::max(0.0, spd(w)) */
        cdf[i + 1] = acc;
    }
    *integral = acc;
    if (acc > 0) for (int i = 0; i <= n; ++i) cdf[i] /= acc;
    return n;
}

int fto_emission_cdf(const ftb_scene_desc* d, int spec, double step, double* cdf, int cap,
                     double* integral) {
    if (!d || !spec_ok(d, spec) || !(step > 0.0)) return fail("emission_cdf: bad input");
    SpecSet S = {d->spectra, d->table_w, d->table_v, d->n_spectra};
    return emission_build(&S, spec, step, cdf, cap, integral);
}

/* FTB_LAMBDA_UNIFORM_380_780 (no counterpart in the reference; the build's uniform-band
 * policy, restated here so the oracle checks it): lambda = 380 + 400 u, weight =
 * pdf_SPD(lambda) / (1/400 nm) from the emitter's binned CDF. */
static double emission_sample_band(const double* cdf, int n, double step, double u, double* weight) {
    double lam = 380.0 + 400.0 * u;
    int b = (int)((lam - LAMBDA_MIN) / step);
    if (b < 0) b = 0;
    if (b > n - 1) b = n - 1;
    *weight = (cdf[b + 1] - cdf[b]) / step * 400.0;
    return lam;
}

/* EmissionSampler::sampleAt (spectrum.h:374-383) */
static double emission_sample_at(const double* cdf, int n, double step, double u,
                                 double* pdf) {
    int lo = 0, hi = n;           /* cdf.size()-1 */
    while (lo + 1 < hi) {
        int mid = (lo + hi) / 2;
        if (cdf[mid] <= u) lo = mid; else hi = mid;
    }
    double c0 = cdf[lo], c1 = cdf[lo + 1];
    double frac = (c1 > c0) ? (u - c0) / (c1 - c0) : 0.5;
    double w = LAMBDA_MIN + (lo + frac) * step;
    double bin_prob = c1 - c0;
    *pdf = bin_prob / step;
    return w;
}

/* ------------------------------------------------------------- color.h:8-24 --------- */
static inline double gauss_piece(double x, double mu, double s1, double s2) {
    double t = (x - mu) * ((x < mu) ? s1 : s2);
    return exp(-0.5 * t * t);
}
static inline double cie_x(double w) {
    return 0.362 * gauss_piece(w, 442.0, 0.0624, 0.0374) +
           1.056 * gauss_piece(w, 599.8, 0.0264, 0.0323) -
           0.065 * gauss_piece(w, 501.1, 0.0490, 0.0382);
}
static inline double cie_y(double w) {
    return 0.821 * gauss_piece(w, 568.8, 0.0213, 0.0247) +
           0.286 * gauss_piece(w, 530.9, 0.0613, 0.0322);
}
static inline double cie_z(double w) {
    return 1.217 * gauss_piece(w, 437.0, 0.0845, 0.0278) +
           0.681 * gauss_piece(w, 459.0, 0.0385, 0.0725);
}

/* ------------------------------------------------------------- scene ---------------- */
enum { PT_TRI = 0, PT_SPH = 1, PT_CRV = 2 };

typedef struct {
    V3 v0, v1, v2, gn, n0, n1, n2;
    int mat;
} Tri;

typedef struct {
    V3 p0, p1;
    double r0, r1, u0, u1;
    int mat;
} Crv;

typedef struct {
    V3 lo, hi;
    int left, right, first, count;   /* count>0: leaf over order[first..first+count) */
} Node;

/* Affine (linalg.h:99-182): m row-major 3x3, then t */
typedef struct { double m[9]; V3 t; } Aff;

/* a binary BVH over primitives order[] (the oracle's own culling structure) */
typedef struct { Node* nodes; int n_nodes; int* order; } Tree;

/* Blas (scene.h:996-1033): triangles in local space with their own tree */
typedef struct {
    int64_t nt;
    Tri* tris;
    Tree tree;
    V3 lo, hi;          /* localBounds: union of the tri boxes padded by 1e-6 */
} Blas;

typedef struct {
    int blas, mat_override;
    Aff to_world, to_local;
} Inst;

typedef struct {
    int shape, collimated, n;
    double step, power;
    const double* cdf;
    V3 origin, u, v, normal, beam;
    double area, radius;
} Emit;

typedef struct {
    double g;
    int sa, ss, bound;
    V3 bmin, bmax, center;
    double radius;
} Med;

/* Scene::MirrorPlane (scene.h:1617-1623): unit normal n, dot(n, x) == d, padded AABB of the
 * member faces, their total area */
typedef struct MPlane {
    V3 n;
    double d;
    V3 lo, hi;
    double area;
    long long key[4];
} MPlane;

/* isPlanarMirrorMat (scene.h:356-360): Mirror, HalfMirror, Glossy with roughness <= 0 */
static int planar_mirror(const ftb_material* m) {
    return m->type == FTB_MAT_MIRROR || m->type == FTB_MAT_HALF_MIRROR ||
           (m->type == FTB_MAT_GLOSSY && m->roughness <= 0.0);
}

struct fto_ctx {
    int lambda_mode;   /* ftb_lambda_mode; set by fto_set_lambda_mode */
    int64_t ni;
    int n_blas;
    Blas* blas;
    Inst* inst;
    SpecSet S;
    ftb_spectrum* spec;
    double *tw, *tv;
    int n_mats;
    ftb_material* mats;
    int64_t nt, ns, nc, np;
    Tri* tris;
    double* sph;      /* 4 per sphere */
    int* sph_mat;
    Crv* crv;
    Tree world;       /* over tris, spheres, curves, instances */
    int n_emit;
    Emit* emit;
    double* cdf_store;
    double* emitter_cdf;   /* selection CDF (scene.h:1499-1513) */
    double total_power;
    int n_med;
    Med* med;
    int n_mp;              /* planar mirrors (Scene::buildMirrorPlanes, scene.h:1646-1720) */
    struct MPlane* mp;
};

double fto_total_power(const fto_ctx* c) { return c ? c->total_power : 0.0; }

int fto_set_lambda_mode(fto_ctx* c, int mode) {
    if (!c || (mode != FTB_LAMBDA_SPD && mode != FTB_LAMBDA_UNIFORM_380_780)) return fail("fto_set_lambda_mode: bad input");
    c->lambda_mode = mode;
    return 0;
}

/* ------------------------------------------------------------- geometry.h ----------- */
typedef struct { int kx, ky, kz; double Sx, Sy, Sz; } Shear;

/* makeTriShear (geometry.h:261-276) */
static Shear make_shear(V3 d) {
    Shear s;
    double ax = fabs(d.x), ay = fabs(d.y), az = fabs(d.z);
    if (ax >= ay && ax >= az) s.kz = 0;
    else if (ay >= az) s.kz = 1;
    else s.kz = 2;
    s.kx = s.kz + 1; if (s.kx == 3) s.kx = 0;
    s.ky = s.kx + 1; if (s.ky == 3) s.ky = 0;
    if (vget(d, s.kz) < 0.0) { int t = s.kx; s.kx = s.ky; s.ky = t; }
    s.Sx = vget(d, s.kx) / vget(d, s.kz);
    s.Sy = vget(d, s.ky) / vget(d, s.kz);
    s.Sz = 1.0 / vget(d, s.kz);
    return s;
}

static double ld_diff(double a, double b, double c, double d) {
    return (double)((long double)a * (long double)b - (long double)c * (long double)d);
}

typedef struct {
    double t;
    int valid, prim, mat, sub;
    V3 p, n, ng;
} Hit;

/* intersectTri (geometry.h:280-369).  `tbest` is hit.t; on accept the hit is filled. */
static int intersect_tri(const Shear* sh, V3 ro, V3 rd, const Tri* tri, double tmin,
                         double tbest, Hit* hit) {
    const int kx = sh->kx, ky = sh->ky, kz = sh->kz;
    V3 A = vsub(tri->v0, ro), B = vsub(tri->v1, ro), C = vsub(tri->v2, ro);
    double Ax = vget(A, kx) - sh->Sx * vget(A, kz), Ay = vget(A, ky) - sh->Sy * vget(A, kz);
    double Bx = vget(B, kx) - sh->Sx * vget(B, kz), By = vget(B, ky) - sh->Sy * vget(B, kz);
    double Cx = vget(C, kx) - sh->Sx * vget(C, kz), Cy = vget(C, ky) - sh->Sy * vget(C, kz);
    double U = Cx * By - Cy * Bx;
    double V = Ax * Cy - Ay * Cx;
    double W = Bx * Ay - By * Ax;
    if (U == 0.0 || V == 0.0 || W == 0.0) {
        if (U == 0.0) U = ld_diff(Cx, By, Cy, Bx);
        if (V == 0.0) V = ld_diff(Ax, Cy, Ay, Cx);
        if (W == 0.0) W = ld_diff(Bx, Ay, By, Ax);
    }
    if ((U < 0.0 || V < 0.0 || W < 0.0) && (U > 0.0 || V > 0.0 || W > 0.0)) return 0;
    double det = U + V + W;
    if (det == 0.0) return 0;
    double T = U * (sh->Sz * vget(A, kz)) + V * (sh->Sz * vget(B, kz)) + W * (sh->Sz * vget(C, kz));
    double invDet = 1.0 / det;
    double t = T * invDet;
    if (t < tmin || t >= tbest) return 0;
    if (!hit) return 1;
    double b0 = U * invDet, b1 = V * invDet, b2 = W * invDet;
    hit->t = t; hit->p = vadd(ro, vmul(rd, t)); hit->valid = 1; hit->mat = tri->mat;
    V3 ns = vadd(vadd(vmul(tri->n0, b0), vmul(tri->n1, b1)), vmul(tri->n2, b2));
    double nl = vdot(ns, ns);
    ns = (nl > 1e-18) ? vmul(ns, 1.0 / sqrt(nl)) : tri->gn;
    V3 gn = (vdot(tri->gn, ns) < 0.0) ? vneg(tri->gn) : tri->gn;
    int flipped = !(vdot(rd, gn) < 0.0);
    hit->ng = gn;
    hit->n = flipped ? vneg(ns) : ns;
    return 1;
}

/* intersectSphere (geometry.h:377-396) */
static int intersect_sphere(V3 ro, V3 rd, const double* s, int mat, double tmin,
                            double tbest, Hit* hit) {
    V3 c = v3(s[0], s[1], s[2]);
    double r = s[3];
    V3 oc = vsub(ro, c);
    double a = vdot(rd, rd);
    double b = 2.0 * vdot(oc, rd);
    double cc = vdot(oc, oc) - r * r;
    double disc = b * b - 4.0 * a * cc;
    if (disc < 0.0) return 0;
    double sq = sqrt(disc);
    double t = (-b - sq) / (2.0 * a);
    if (t < tmin) t = (-b + sq) / (2.0 * a);
    if (t < tmin || t >= tbest) return 0;
    if (!hit) return 1;
    hit->t = t; hit->p = vadd(ro, vmul(rd, t)); hit->valid = 1;
    V3 ng = vnorm(vsub(hit->p, c));
    hit->ng = ng;
    int flipped = !(vdot(rd, ng) < 0.0);
    hit->n = flipped ? vneg(ng) : ng;
    hit->mat = mat;
    return 1;
}

/* makeCurveRay (curve.h:126-135) */
typedef struct { V3 dn; double inv_len; } CurveRay;
static CurveRay make_curve_ray(V3 d) {
    CurveRay c; c.dn = v3(0, 0, 1); c.inv_len = 1.0;
    double l2 = vdot(d, d);
    if (l2 > 0.0) { double l = sqrt(l2); c.inv_len = 1.0 / l; c.dn = vmul(d, c.inv_len); }
    return c;
}

/* curveSegCrossings<double> + intersectCurveSeg (curve.h:199-334).  The offer callback is
 * restated inline as `offer_root`. */
typedef struct { double best_tn, best_y, shift, inv_len, tmin, tbest; int piece; } CurveAcc;
static inline void offer_root(CurveAcc* a, double tn, int w, double y) {
    if (tn >= a->best_tn) return;
    double t = (tn + a->shift) * a->inv_len;
    if (t < a->tmin || t >= a->tbest) return;
    a->best_tn = tn; a->piece = w; a->best_y = y;
}

static int intersect_curve(const CurveRay* cr, V3 ro, V3 rdr, const Crv* s, double tmin,
                           double tbest, Hit* hit) {
    V3 rd = cr->dn;
    double ro_[3] = {ro.x, ro.y, ro.z}, rd_[3] = {rd.x, rd.y, rd.z};
    double p0[3] = {s->p0.x, s->p0.y, s->p0.z}, p1[3] = {s->p1.x, s->p1.y, s->p1.z};
    double r0 = s->r0, r1 = s->r1;
    CurveAcc acc = {DBL_MAX, 0.0, 0.0, cr->inv_len, tmin, tbest, -1};
#define D3(a, b) (a[0] * b[0] + a[1] * b[1] + a[2] * b[2])
    double ba[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]};
    double m0 = D3(ba, ba);
    if (!(m0 > 0.0)) return 0;
    double toP0[3] = {p0[0] - ro_[0], p0[1] - ro_[1], p0[2] - ro_[2]};
    acc.shift = D3(toP0, rd_);
    double o[3] = {ro_[0] + rd_[0] * acc.shift, ro_[1] + rd_[1] * acc.shift,
                   ro_[2] + rd_[2] * acc.shift};
    double oa[3] = {o[0] - p0[0], o[1] - p0[1], o[2] - p0[2]};
    double ob[3] = {o[0] - p1[0], o[1] - p1[1], o[2] - p1[2]};
    double rr = r0 - r1;
    double m1 = D3(ba, oa), m2 = D3(ba, rd_), m3 = D3(rd_, oa), m5 = D3(oa, oa);
    double m6 = D3(ob, rd_), m7 = D3(ob, ob);
    double d2 = m0 - rr * rr;
#undef D3
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
            if (ya > 0.0 && ya < d2) offer_root(&acc, ta, 0, ya);
            if (yb > 0.0 && yb < d2) offer_root(&acc, tb, 0, yb);
        }
        double h1 = m3 * m3 - m5 + r0 * r0;
        if (h1 > 0.0) {
            double q = sqrt(h1), base = m1 - r0 * rr;
            double ta = -m3 - q, tb = -m3 + q;
            if (base + ta * m2 <= 0.0) offer_root(&acc, ta, 1, 0.0);
            if (base + tb * m2 <= 0.0) offer_root(&acc, tb, 1, 0.0);
        }
        double h2 = m6 * m6 - m7 + r1 * r1;
        if (h2 > 0.0) {
            double q = sqrt(h2), base = m1 - r0 * rr;
            double ta = -m6 - q, tb = -m6 + q;
            if (base + ta * m2 >= d2) offer_root(&acc, ta, 2, d2);
            if (base + tb * m2 >= d2) offer_root(&acc, tb, 2, d2);
        }
    } else {
        int use_p0 = (r0 >= r1);
        double rc = use_p0 ? r0 : r1;
        double mm = use_p0 ? m3 : m6;
        double mq = use_p0 ? m5 : m7;
        double hh = mm * mm - mq + rc * rc;
        if (hh > 0.0) {
            double q = sqrt(hh);
            offer_root(&acc, -mm - q, use_p0 ? 1 : 2, use_p0 ? 0.0 : d2);
            offer_root(&acc, -mm + q, use_p0 ? 1 : 2, use_p0 ? 0.0 : d2);
        }
    }
    if (acc.piece < 0) return 0;
    double t = (acc.best_tn + acc.shift) * cr->inv_len;
    if (!hit) return 1;
    hit->t = t; hit->valid = 1;
    V3 bav = vsub(s->p1, s->p0);
    V3 rov = vadd(ro, vmul(rd, acc.shift));
    V3 oav = vsub(rov, s->p0), obv = vsub(rov, s->p1);
    hit->p = vadd(ro, vmul(rdr, t));
    hit->mat = s->mat;
    V3 ng;
    if (acc.piece == 0) ng = vsub(vmul(vadd(oav, vmul(rd, acc.best_tn)), d2), vmul(bav, acc.best_y));
    else if (acc.piece == 1) ng = vadd(oav, vmul(rd, acc.best_tn));
    else ng = vadd(obv, vmul(rd, acc.best_tn));
    double nl = sqrt(vdot(ng, ng));
    ng = (nl > 1e-18) ? vmul(ng, 1.0 / nl) : vnorm(bav);
    hit->ng = ng;
    hit->n = (vdot(rdr, ng) < 0.0) ? ng : vneg(ng);
    return 1;
}

/* orientedGeoN (geometry.h:174-176) */
static inline V3 oriented_geo_n(const Hit* h) {
    return (vdot(h->ng, h->n) >= 0.0) ? h->ng : vneg(h->ng);
}
/* shadingAdjointCorr (geometry.h:200-206) */
static inline double shading_adjoint_corr(V3 wi, V3 wo, V3 ns, V3 ng) {
    double denom = fabs(vdot(wi, ng)) * fabs(vdot(wo, ns));
    if (denom <= 1e-8) return 1.0;
    double num = fabs(vdot(wi, ns)) * fabs(vdot(wo, ng));
    return num / denom;
}
/* shadowTerminatorG (geometry.h:225-242) */
static inline double shadow_terminator_g(V3 wi, V3 ns, V3 ng) {
    double cos_ng_ns = vdot(ng, ns);
    if (cos_ng_ns >= 1.0 - 1e-7) return (vdot(ng, wi) > 0.0) ? 1.0 : 0.0;
    double cos_ng_wi = vdot(ng, wi);
    if (cos_ng_wi <= 0.0) return 0.0;
    double denom = vdot(ns, wi) * cos_ng_ns;
    if (denom <= 1e-8) return 1.0;
    double g = cos_ng_wi / denom;
    if (g >= 1.0) return 1.0;
    return g * g * (1.0 - g) + g;
}

/* ------------------------------------------------------------- Affine (linalg.h) --- */
/* Affine::apply / applyDir (linalg.h:105-114) */
static inline V3 aff_apply(const Aff* a, V3 p) {
    return v3(a->m[0] * p.x + a->m[1] * p.y + a->m[2] * p.z + a->t.x,
              a->m[3] * p.x + a->m[4] * p.y + a->m[5] * p.z + a->t.y,
              a->m[6] * p.x + a->m[7] * p.y + a->m[8] * p.z + a->t.z);
}
static inline V3 aff_apply_dir(const Aff* a, V3 v) {
    return v3(a->m[0] * v.x + a->m[1] * v.y + a->m[2] * v.z,
              a->m[3] * v.x + a->m[4] * v.y + a->m[5] * v.z,
              a->m[6] * v.x + a->m[7] * v.y + a->m[8] * v.z);
}
/* Affine::inverse (linalg.h:129-144) */
static Aff aff_inverse(const Aff* x) {
    Aff r;
    memset(&r, 0, sizeof r);
    r.m[0] = r.m[4] = r.m[8] = 1.0;
    double a = x->m[0], b = x->m[1], c = x->m[2];
    double d = x->m[3], e = x->m[4], f = x->m[5];
    double g = x->m[6], h = x->m[7], i = x->m[8];
    double det = a * (e * i - f * h) - b * (d * i - f * g) + c * (d * h - e * g);
    if (fabs(det) < 1e-30) return r;
    double id = 1.0 / det;
    r.m[0] = (e * i - f * h) * id; r.m[1] = (c * h - b * i) * id; r.m[2] = (b * f - c * e) * id;
    r.m[3] = (f * g - d * i) * id; r.m[4] = (a * i - c * g) * id; r.m[5] = (c * d - a * f) * id;
    r.m[6] = (d * h - e * g) * id; r.m[7] = (b * g - a * h) * id; r.m[8] = (a * e - b * d) * id;
    r.t = v3(-(r.m[0] * x->t.x + r.m[1] * x->t.y + r.m[2] * x->t.z),
             -(r.m[3] * x->t.x + r.m[4] * x->t.y + r.m[5] * x->t.z),
             -(r.m[6] * x->t.x + r.m[7] * x->t.y + r.m[8] * x->t.z));
    return r;
}
/* Affine::applyNormal (linalg.h:161-167): (M^-1)^T n with M^-1 = inverse() */
static inline V3 aff_apply_normal(const Aff* inv, V3 n) {
    return v3(inv->m[0] * n.x + inv->m[3] * n.y + inv->m[6] * n.z,
              inv->m[1] * n.x + inv->m[4] * n.y + inv->m[7] * n.z,
              inv->m[2] * n.x + inv->m[5] * n.y + inv->m[8] * n.z);
}

/* ------------------------------------------------------------- BVH (oracle only) ---- */
/* A plain median-split binary BVH with boxes grown by a relative margin, so that its
 * culling never rejects a primitive the exact slab test would keep.  Closest-hit results
 * equal the reference's (bvh.h:181-224) except for exact ties in t. */
typedef struct { V3 lo, hi, c; int idx; } BPrim;

static void tri_box(const Tri* t, V3* lo, V3* hi) {
    *lo = v3(fmin(t->v0.x, fmin(t->v1.x, t->v2.x)), fmin(t->v0.y, fmin(t->v1.y, t->v2.y)),
             fmin(t->v0.z, fmin(t->v1.z, t->v2.z)));
    *hi = v3(fmax(t->v0.x, fmax(t->v1.x, t->v2.x)), fmax(t->v0.y, fmax(t->v1.y, t->v2.y)),
             fmax(t->v0.z, fmax(t->v1.z, t->v2.z)));
}

static void box_of(const fto_ctx* c, int p, V3* lo, V3* hi) {
    if (p < c->nt) {
        tri_box(&c->tris[p], lo, hi);
    } else if (p < c->nt + c->ns) {
        const double* s = &c->sph[(p - c->nt) * 4];
        *lo = v3(s[0] - s[3], s[1] - s[3], s[2] - s[3]);
        *hi = v3(s[0] + s[3], s[1] + s[3], s[2] + s[3]);
    } else if (p < c->nt + c->ns + c->nc) {
        const Crv* s = &c->crv[p - c->nt - c->ns];
        *lo = v3(fmin(s->p0.x - s->r0, s->p1.x - s->r1), fmin(s->p0.y - s->r0, s->p1.y - s->r1),
                 fmin(s->p0.z - s->r0, s->p1.z - s->r1));
        *hi = v3(fmax(s->p0.x + s->r0, s->p1.x + s->r1), fmax(s->p0.y + s->r0, s->p1.y + s->r1),
                 fmax(s->p0.z + s->r0, s->p1.z + s->r1));
    } else {   /* instance: the 8 transformed corners of the BLAS bounds (scene.h:2033-2040) */
        const Inst* in = &c->inst[p - c->nt - c->ns - c->nc];
        const Blas* b = &c->blas[in->blas];
        *lo = v3(DBL_MAX, DBL_MAX, DBL_MAX);
        *hi = v3(-DBL_MAX, -DBL_MAX, -DBL_MAX);
        for (int k = 0; k < 8; ++k) {
            V3 q = v3((k & 1) ? b->hi.x : b->lo.x, (k & 2) ? b->hi.y : b->lo.y, (k & 4) ? b->hi.z : b->lo.z);
            V3 w = aff_apply(&in->to_world, q);
            *lo = v3(fmin(lo->x, w.x), fmin(lo->y, w.y), fmin(lo->z, w.z));
            *hi = v3(fmax(hi->x, w.x), fmax(hi->y, w.y), fmax(hi->z, w.z));
        }
        double m = 1e-7 * (1.0 + fmax(fmax(fabs(lo->x), fabs(hi->x)),
                                      fmax(fmax(fabs(lo->y), fabs(hi->y)), fmax(fabs(lo->z), fabs(hi->z)))));
        *lo = v3(lo->x - m, lo->y - m, lo->z - m);
        *hi = v3(hi->x + m, hi->y + m, hi->z + m);
    }
}

static int g_sort_axis;
static int cmp_prim(const void* a, const void* b) {
    double x = vget(((const BPrim*)a)->c, g_sort_axis), y = vget(((const BPrim*)b)->c, g_sort_axis);
    return (x < y) ? -1 : (x > y) ? 1 : 0;
}

static int build_rec(Tree* T, BPrim* bp, int start, int end) {
    int ni = T->n_nodes++;
    Node* nd = &T->nodes[ni];
    V3 lo = v3(DBL_MAX, DBL_MAX, DBL_MAX), hi = v3(-DBL_MAX, -DBL_MAX, -DBL_MAX);
    V3 clo = lo, chi = hi;
    for (int i = start; i < end; ++i) {
        lo = v3(fmin(lo.x, bp[i].lo.x), fmin(lo.y, bp[i].lo.y), fmin(lo.z, bp[i].lo.z));
        hi = v3(fmax(hi.x, bp[i].hi.x), fmax(hi.y, bp[i].hi.y), fmax(hi.z, bp[i].hi.z));
        clo = v3(fmin(clo.x, bp[i].c.x), fmin(clo.y, bp[i].c.y), fmin(clo.z, bp[i].c.z));
        chi = v3(fmax(chi.x, bp[i].c.x), fmax(chi.y, bp[i].c.y), fmax(chi.z, bp[i].c.z));
    }
    /* grow by a relative margin: covers the rounding of the slab test below */
    double m = 1e-9 * (1.0 + fmax(fmax(fabs(lo.x), fabs(hi.x)),
                                  fmax(fmax(fabs(lo.y), fabs(hi.y)), fmax(fabs(lo.z), fabs(hi.z)))));
    nd->lo = v3(lo.x - m, lo.y - m, lo.z - m);
    nd->hi = v3(hi.x + m, hi.y + m, hi.z + m);
    int count = end - start;
    V3 ext = vsub(chi, clo);
    int axis = (ext.x >= ext.y && ext.x >= ext.z) ? 0 : (ext.y >= ext.z ? 1 : 2);
    if (count <= 4 || vget(ext, axis) <= 0.0) {
        nd->count = count; nd->first = start; nd->left = nd->right = -1;
        return ni;
    }
    g_sort_axis = axis;
    qsort(bp + start, (size_t)count, sizeof(BPrim), cmp_prim);
    int mid = (start + end) / 2;
    int l = build_rec(T, bp, start, mid);
    int r = build_rec(T, bp, mid, end);
    nd = &T->nodes[ni];
    nd->left = l; nd->right = r; nd->count = 0;
    return ni;
}

static void build_tree(Tree* T, BPrim* bp, int n) {
    T->n_nodes = 0;
    T->nodes = (Node*)malloc(sizeof(Node) * (size_t)(2 * n + 1));
    T->order = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (n > 0) build_rec(T, bp, 0, n);
    for (int i = 0; i < n; ++i) T->order[i] = bp[i].idx;
}

/* slab test in double against a grown box; NaN-safe like Aabb::hit (bvh.h:45-67) */
static inline int box_hit(const Node* n, V3 o, V3 inv, double tmin, double tmax, double* te_out) {
    double te = tmin, tx = tmax, t0, t1, tt;
    t0 = (n->lo.x - o.x) * inv.x; t1 = (n->hi.x - o.x) * inv.x;
    if (t0 > t1) { tt = t0; t0 = t1; t1 = tt; }
    te = t0 > te ? t0 : te; tx = t1 < tx ? t1 : tx;
    if (tx < te) return 0;
    t0 = (n->lo.y - o.y) * inv.y; t1 = (n->hi.y - o.y) * inv.y;
    if (t0 > t1) { tt = t0; t0 = t1; t1 = tt; }
    te = t0 > te ? t0 : te; tx = t1 < tx ? t1 : tx;
    if (tx < te) return 0;
    t0 = (n->lo.z - o.z) * inv.z; t1 = (n->hi.z - o.z) * inv.z;
    if (t0 > t1) { tt = t0; t0 = t1; t1 = tt; }
    te = t0 > te ? t0 : te; tx = t1 < tx ? t1 : tx;
    if (tx < te) return 0;
    *te_out = te;
    return 1;
}

/* Nearest primitive p of tree T with test(env, p, tbest, &t) accepted; returns p or -1.
 * Exact ties in t go to the lower primitive index.  The reference takes the first of the
 * tied primitives its own hierarchy happens to test (bvh.h:181-224, strict t < tBest), an
 * order no other hierarchy reproduces; with the index rule the result does not depend on
 * the hierarchy at all, so the oracle and the device (which applies the same rule) agree on
 * every tie, and differ from the reference only where the reference's order picked the
 * higher index. */
typedef int (*PrimTest)(const void* env, int p, double tbest, double* t);
static int tree_closest(const Tree* T, V3 ro, V3 rd, double tmin, double tbest, PrimTest test, const void* env,
                        double* t_out) {
    if (T->n_nodes == 0) return -1;
    V3 inv = v3(1.0 / rd.x, 1.0 / rd.y, 1.0 / rd.z);
    double best = tbest;
    int bestp = -1;
    int stack[128]; double tst[128]; int sp = 0;
    double te;
    if (!box_hit(&T->nodes[0], ro, inv, tmin, best, &te)) return -1;
    stack[sp] = 0; tst[sp] = te; ++sp;
    while (sp) {
        --sp;
        if (tst[sp] > best) continue;
        const Node* n = &T->nodes[stack[sp]];
        if (n->count > 0) {
            for (int i = 0; i < n->count; ++i) {
                int p = T->order[n->first + i];
                double t;
                /* accept t <= best, then keep the lower index on a tie */
                if (test(env, p, nextafter(best, INFINITY), &t) && (t < best || bestp < 0 || p < bestp)) {
                    best = t;
                    bestp = p;
                }
            }
        } else {
            double tl = 0.0, tr = 0.0;
            int hl = box_hit(&T->nodes[n->left], ro, inv, tmin, best, &tl);
            int hr = box_hit(&T->nodes[n->right], ro, inv, tmin, best, &tr);
            if (sp + 2 > 128) { fail("oracle BVH stack overflow"); return -1; }
            if (hl && hr) {
                if (tl <= tr) { stack[sp] = n->right; tst[sp++] = tr; stack[sp] = n->left; tst[sp++] = tl; }
                else { stack[sp] = n->left; tst[sp++] = tl; stack[sp] = n->right; tst[sp++] = tr; }
            } else if (hl) { stack[sp] = n->left; tst[sp++] = tl; }
            else if (hr) { stack[sp] = n->right; tst[sp++] = tr; }
        }
    }
    if (bestp >= 0) *t_out = best;
    return bestp;
}

/* Any primitive of tree T with test(env, p, seg, &t) accepted. */
static int tree_any(const Tree* T, V3 o, V3 d, double tmin, double seg, PrimTest test, const void* env) {
    if (T->n_nodes == 0) return 0;
    V3 inv = v3(1.0 / d.x, 1.0 / d.y, 1.0 / d.z);
    double te, t;
    if (!box_hit(&T->nodes[0], o, inv, tmin, seg, &te)) return 0;
    int stack[128]; int sp = 0; stack[sp++] = 0;
    while (sp) {
        const Node* n = &T->nodes[stack[--sp]];
        if (n->count > 0) {
            for (int i = 0; i < n->count; ++i)
                if (test(env, T->order[n->first + i], seg, &t)) return 1;
        } else {
            if (sp + 2 > 128) { fail("oracle BVH stack overflow"); return 0; }
            if (box_hit(&T->nodes[n->left], o, inv, tmin, seg, &te)) stack[sp++] = n->left;
            if (box_hit(&T->nodes[n->right], o, inv, tmin, seg, &te)) stack[sp++] = n->right;
        }
    }
    return 0;
}

/* A ray as the leaf tests see it. */
typedef struct {
    const fto_ctx* c;
    const Blas* b;     /* BLAS being walked (instance leaves) */
    V3 ro, rd;
    Shear sh;
    CurveRay cr;
    double tmin;
} RayEnv;

static int blas_test(const void* env, int p, double tbest, double* t) {
    const RayEnv* E = (const RayEnv*)env;
    Hit h;
    if (!intersect_tri(&E->sh, E->ro, E->rd, &E->b->tris[p], E->tmin, tbest, &h)) return 0;
    *t = h.t;
    return 1;
}

/* Blas::intersectLocal / occludedLocal through an instance (scene.h:1017-1033, 2226-2231):
 * the world ray mapped by toLocal; local t == world t. */
static int inst_local_ray(const fto_ctx* c, int ii, V3 ro, V3 rd, double tmin, RayEnv* E) {
    const Inst* in = &c->inst[ii];
    E->c = c;
    E->b = &c->blas[in->blas];
    E->ro = aff_apply(&in->to_local, ro);
    E->rd = aff_apply_dir(&in->to_local, rd);
    E->sh = make_shear(E->rd);
    E->tmin = tmin;
    return 1;
}

static int world_test(const void* env, int p, double tbest, double* t) {
    const RayEnv* E = (const RayEnv*)env;
    const fto_ctx* c = E->c;
    Hit h;
    if (p < c->nt) {
        if (!intersect_tri(&E->sh, E->ro, E->rd, &c->tris[p], E->tmin, tbest, &h)) return 0;
    } else if (p < c->nt + c->ns) {
        if (!intersect_sphere(E->ro, E->rd, &c->sph[(p - c->nt) * 4], c->sph_mat[p - c->nt], E->tmin, tbest, &h))
            return 0;
    } else if (p < c->nt + c->ns + c->nc) {
        if (!intersect_curve(&E->cr, E->ro, E->rd, &c->crv[p - c->nt - c->ns], E->tmin, tbest, &h)) return 0;
    } else {
        RayEnv L;
        inst_local_ray(c, (int)(p - c->nt - c->ns - c->nc), E->ro, E->rd, E->tmin, &L);
        return tree_closest(&L.b->tree, L.ro, L.rd, E->tmin, tbest, blas_test, &L, t) >= 0;
    }
    *t = h.t;
    return 1;
}

static int world_any(const void* env, int p, double seg, double* t) {
    const RayEnv* E = (const RayEnv*)env;
    const fto_ctx* c = E->c;
    if (p >= c->nt + c->ns + c->nc) {
        RayEnv L;
        inst_local_ray(c, (int)(p - c->nt - c->ns - c->nc), E->ro, E->rd, E->tmin, &L);
        return tree_any(&L.b->tree, L.ro, L.rd, E->tmin, seg, blas_test, &L);
    }
    return world_test(env, p, seg, t);
}

/* Scene::closestHit (scene.h:2194-2242): nearest accepted primitive, returns prim or -1.
 * For an instance, hit->sub is the BLAS triangle and the hit is mapped to the world like
 * Scene::instanceHitToWorld (scene.h:2107-2133). */
static int closest_hit(const fto_ctx* c, V3 ro, V3 rd, double tmin, Hit* hit) {
    hit->valid = 0; hit->t = DBL_MAX; hit->prim = -1; hit->sub = -1;
    RayEnv E;
    E.c = c; E.b = NULL; E.ro = ro; E.rd = rd; E.sh = make_shear(rd); E.cr = make_curve_ray(rd); E.tmin = tmin;
    double t;
    int bestp = tree_closest(&c->world, ro, rd, tmin, DBL_MAX, world_test, &E, &t);
    if (bestp < 0) return -1;
    if (bestp < c->nt) intersect_tri(&E.sh, ro, rd, &c->tris[bestp], tmin, DBL_MAX, hit);
    else if (bestp < c->nt + c->ns)
        intersect_sphere(ro, rd, &c->sph[(bestp - c->nt) * 4], c->sph_mat[bestp - c->nt], tmin, DBL_MAX, hit);
    else if (bestp < c->nt + c->ns + c->nc)
        intersect_curve(&E.cr, ro, rd, &c->crv[bestp - c->nt - c->ns], tmin, DBL_MAX, hit);
    else {
        int ii = (int)(bestp - c->nt - c->ns - c->nc);
        const Inst* in = &c->inst[ii];
        RayEnv L;
        inst_local_ray(c, ii, ro, rd, tmin, &L);
        double tl;
        int tri = tree_closest(&L.b->tree, L.ro, L.rd, tmin, DBL_MAX, blas_test, &L, &tl);
        Hit lh;
        intersect_tri(&L.sh, L.ro, L.rd, &L.b->tris[tri], tmin, DBL_MAX, &lh);
        lh.p = vadd(ro, vmul(rd, lh.t));
        V3 wn = vnorm(aff_apply_normal(&in->to_local, lh.n));
        V3 wng = vnorm(aff_apply_normal(&in->to_local, lh.ng));
        lh.ng = wng;
        lh.n = (vdot(rd, wn) < 0.0) ? wn : vneg(wn);
        if (in->mat_override >= 0) lh.mat = in->mat_override;
        *hit = lh;
        hit->sub = tri;
    }
    hit->prim = bestp;
    return bestp;
}

/* Scene::occluded (scene.h:2249-2271): any primitive with t in [tmin, maxDist-tmin) */
static int occluded(const fto_ctx* c, V3 o, V3 d, double max_dist, double tmin) {
    double seg = max_dist - tmin;
    RayEnv E;
    E.c = c; E.b = NULL; E.ro = o; E.rd = d; E.sh = make_shear(d); E.cr = make_curve_ray(d); E.tmin = tmin;
    return tree_any(&c->world, o, d, tmin, seg, world_any, &E);
}

int fto_closest_hit(const fto_ctx* c, const double o[3], const double d[3], double tmin,
                    double* t_out) {
    Hit h;
    int p = closest_hit(c, v3(o[0], o[1], o[2]), v3(d[0], d[1], d[2]), tmin, &h);
    if (t_out) *t_out = h.valid ? h.t : INFINITY;
    return p;
}
int fto_occluded(const fto_ctx* c, const double o[3], const double d[3], double max_dist,
                 double tmin) {
    return occluded(c, v3(o[0], o[1], o[2]), v3(d[0], d[1], d[2]), max_dist, tmin);
}

/* ------------------------------------------------------------- camera.h ------------- */
void fto_camera_look_at(const double eye[3], const double target[3], const double up[3],
                        double fov, int rx, int ry, ftb_camera* out) {
    V3 e = v3(eye[0], eye[1], eye[2]);
    V3 w = vnorm(vsub(v3(target[0], target[1], target[2]), e));
    V3 u = vnorm(vcross(w, v3(up[0], up[1], up[2])));
    V3 v = vcross(u, w);
    double thy = tan(0.5 * fov * 3.141592653589793 / 180.0);
    double thx = thy * (double)rx / (double)ry;
    memset(out, 0, sizeof *out);
    out->eye[0] = e.x; out->eye[1] = e.y; out->eye[2] = e.z;
    out->u[0] = u.x; out->u[1] = u.y; out->u[2] = u.z;
    out->v[0] = v.x; out->v[1] = v.y; out->v[2] = v.z;
    out->w[0] = w.x; out->w[1] = w.y; out->w[2] = w.z;
    out->tan_half_x = thx; out->tan_half_y = thy;
    out->res_x = rx; out->res_y = ry;
}

typedef struct {
    V3 eye, u, v, w;
    double thx, thy;
    int rx, ry;
} Cam;

/* Camera::project, rectilinear branch (camera.h:137-151) */
static int cam_project(const Cam* c, V3 p, int* px, int* py, double* cos_cam, double* dist2) {
    V3 d = vsub(p, c->eye);
    double cz = vdot(d, c->w);
    if (cz <= 1e-9) return 0;
    double cx = vdot(d, c->u), cy = vdot(d, c->v);
    double ix = (cx / cz) / c->thx - 0.0;   /* frustumShiftX == 0 */
    double iy = (cy / cz) / c->thy;
    if (ix < -1 || ix >= 1 || iy < -1 || iy >= 1) return 0;
    *px = (int)((ix * 0.5 + 0.5) * c->rx);
    *py = (int)((iy * 0.5 + 0.5) * c->ry);
    *dist2 = vdot(d, d);
    *cos_cam = cz / sqrt(*dist2);
    return 1;
}
/* pixelPlaneArea * cos^3 (camera.h:179-183, 229-240) */
static inline double cam_pixel_solid_angle(const Cam* c, double cos_cam) {
    double ipa = 4.0 * c->thx * c->thy;
    double ppa = ipa / ((double)c->rx * (double)c->ry);
    return ppa * cos_cam * cos_cam * cos_cam;
}

/* ------------------------------------------------------------- tracer --------------- */
typedef struct {
    double* xyz;
    double* hits;
    int rx, ry;
} Film;

static inline void film_add(Film* f, int px, int py, double x, double y, double z) {
    size_t i = (size_t)py * f->rx + px;
    f->xyz[3 * i] += x; f->xyz[3 * i + 1] += y; f->xyz[3 * i + 2] += z;
    f->hits[i] += 1.0;
}

typedef struct {
    const fto_ctx* c;
    const Cam* cam;
    Film* film;
    int64_t rays;
} Tr;

/* Medium::sigmaT / albedo (scene.h:565-572) */
static inline double med_sigma_t(const fto_ctx* c, const Med* m, double lam) {
    double v = spec_eval(&c->S, m->sa, lam) + spec_eval(&c->S, m->ss, lam);
    return v > 0.0 ? v : 0.0;
}
static inline double med_albedo(const fto_ctx* c, const Med* m, double lam) {
    double s = spec_eval(&c->S, m->ss, lam); s = s > 0.0 ? s : 0.0;
    double a = spec_eval(&c->S, m->sa, lam);
    double t = s + (a > 0.0 ? a : 0.0);
    return t > 0.0 ? s / t : 0.0;
}
/* Medium::clipToBounds (scene.h:655-685) */
static int clip_to_bounds(const Med* m, V3 o, V3 d, double t0, double t1, double* ta, double* tb) {
    if (m->bound == FTB_BOUND_NONE) { *ta = t0; *tb = t1; return t1 > t0; }
    if (m->bound == FTB_BOUND_SPHERE) {
        V3 oc = vsub(o, m->center);
        double A = vdot(d, d);
        double B = 2.0 * vdot(oc, d);
        double C = vdot(oc, oc) - m->radius * m->radius;
        double disc = B * B - 4.0 * A * C;
        if (disc <= 0.0 || A <= 0.0) return 0;
        double sd = sqrt(disc);
        double s0 = (-B - sd) / (2.0 * A), s1 = (-B + sd) / (2.0 * A);
        double lo = t0 > s0 ? t0 : s0, hi = t1 < s1 ? t1 : s1;   /* std::max / std::min */
        if (lo > hi) return 0;
        *ta = lo; *tb = hi; return *tb > *ta;
    }
    double lo = t0, hi = t1;
    for (int a = 0; a < 3; ++a) {
        double oa = vget(o, a), da = vget(d, a);
        double mn = vget(m->bmin, a), mx = vget(m->bmax, a);
        if (fabs(da) < 1e-12) { if (oa < mn || oa > mx) return 0; continue; }
        double inv = 1.0 / da;
        double s0 = (mn - oa) * inv, s1 = (mx - oa) * inv;
        if (s0 > s1) { double t = s0; s0 = s1; s1 = t; }
        lo = (lo < s0) ? s0 : lo;    /* std::max(lo, s0) */
        hi = (s1 < hi) ? s1 : hi;    /* std::min(hi, s1) */
        if (lo > hi) return 0;
    }
    *ta = lo; *tb = hi; return *tb > *ta;
}
/* Renderer::sampleMediaCollision, homogeneous media (render.h:377-398, 444-458) */
static int sample_media_collision(const Tr* T, V3 o, V3 d, double dmax, double lam, Pcg* rng,
                                  double* thit, int* which) {
    const fto_ctx* c = T->c;
    double best = dmax; int w = -1;
    for (int i = 0; i < c->n_med; ++i) {
        const Med* m = &c->med[i];
        double st = med_sigma_t(c, m, lam);
        if (st <= 0.0) continue;
        double ta, tb;
        if (!clip_to_bounds(m, o, d, 0.0, dmax, &ta, &tb)) continue;
        double t = ta - log(1.0 - pcg_uniform(rng)) / st;
        if (t < tb && t < best) { best = t; w = i; }
    }
    if (w < 0) return 0;
    *thit = best; *which = w; return 1;
}
/* Renderer::mediaTransmittance, homogeneous media (render.h:403-421, 461-469) */
static double media_transmittance(const Tr* T, V3 o, V3 d, double dist, double lam) {
    const fto_ctx* c = T->c;
    double tr = 1.0;
    for (int i = 0; i < c->n_med; ++i) {
        const Med* m = &c->med[i];
        double st = med_sigma_t(c, m, lam);
        double mt = 1.0;
        if (st > 0.0) {
            double ta, tb;
            if (clip_to_bounds(m, o, d, 0.0, dist, &ta, &tb)) mt = exp(-st * (tb - ta));
        }
        tr *= mt;
        if (tr <= 0.0) break;
    }
    return tr;
}
/* hgPhase / sampleHG (phase.h:18-40) */
static inline double hg_phase(double cos_t, double g) {
    double d = 1.0 + g * g - 2.0 * g * cos_t;
    if (d < 1e-9) d = 1e-9;
    return (1.0 - g * g) / (4.0 * PI_D * d * sqrt(d));
}
static V3 sample_hg(V3 wi, double g, Pcg* rng) {
    double u1 = pcg_uniform(rng), u2 = pcg_uniform(rng);
    double cos_t;
    if (fabs(g) < 1e-3) cos_t = 1.0 - 2.0 * u1;
    else {
        double sq = (1.0 - g * g) / (1.0 + g - 2.0 * g * u1);
        cos_t = (1.0 + g * g - sq * sq) / (2.0 * g);
    }
    double s = 1.0 - cos_t * cos_t;
    double sin_t = sqrt(s > 0.0 ? s : 0.0);
    double phi = 2.0 * PI_D * u2;
    V3 t, b; onb(wi, &t, &b);
    return vnorm(vadd(vadd(vmul(t, sin_t * cos(phi)), vmul(b, sin_t * sin(phi))), vmul(wi, cos_t)));
}

/* Renderer::connectGeom + connect, surface vertex, model B (render.h:499-559) */
static void connect_surface(Tr* T, V3 p, V3 n, V3 ng, V3 wi, double lam, double beta, double rho) {
    const Cam* cam = T->cam;
    V3 to_cam = vsub(cam->eye, p);
    double dist = vlen(to_cam);
    V3 wdir = vdiv(to_cam, dist);
    double cos_surf = vdot(n, wdir);
    if (cos_surf <= 0) return;
    double stg = shadow_terminator_g(wdir, n, ng);
    if (stg <= 0.0) return;
    int px, py; double cos_cam, dist2;
    if (!cam_project(cam, p, &px, &py, &cos_cam, &dist2)) return;
    T->rays++;
    if (occluded(T->c, vadd(p, vmul(ng, 1e-6)), wdir, dist - 2e-6, 1e-6)) return;
    double omega = cam_pixel_solid_angle(cam, cos_cam);
    double corr = shading_adjoint_corr(wi, wdir, n, ng);
    double denom = dist2 * omega;
    double f = rho / PI_D;
    double contrib = beta * f * cos_surf * corr / denom * stg;
    if (T->c->n_med > 0) contrib *= media_transmittance(T, p, wdir, dist, lam);
    film_add(T->film, px, py, cie_x(lam) * contrib, cie_y(lam) * contrib, cie_z(lam) * contrib);
}

/* Renderer::connectVolume (render.h:584-600) */
static void connect_volume(Tr* T, const Med* m, V3 p, V3 win, double lam, double beta) {
    const Cam* cam = T->cam;
    V3 to_cam = vsub(cam->eye, p);
    double dist = vlen(to_cam);
    V3 wdir = vdiv(to_cam, dist);
    int px, py; double cos_cam, dist2;
    if (!cam_project(cam, p, &px, &py, &cos_cam, &dist2)) return;
    T->rays++;
    if (occluded(T->c, vadd(p, vmul(wdir, 1e-6)), wdir, dist - 2e-6, 1e-6)) return;
    double ph = hg_phase(vdot(win, wdir), m->g);
    double alb = med_albedo(T->c, m, lam);
    double omega = cam_pixel_solid_angle(cam, cos_cam);
    double contrib = beta * alb * ph / (dist2 * omega);
    contrib *= media_transmittance(T, p, wdir, dist, lam);
    film_add(T->film, px, py, cie_x(lam) * contrib, cie_y(lam) * contrib, cie_z(lam) * contrib);
}

/* glossyDirUV / sampleGlossy (render.h:46-64) */
static V3 sample_glossy(V3 mdir, double roughness, Pcg* rng) {
    double u1 = pcg_uniform(rng), u2 = pcg_uniform(rng);
    if (u1 >= 1.0) return mdir;
    double rr = roughness < 1e-3 ? 1e-3 : roughness;
    double e = 2.0 / (rr * rr) - 2.0; if (e < 0) e = 0;
    double cos_t = pow(u1, 1.0 / (e + 1.0));
    double s = 1.0 - cos_t * cos_t;
    double sin_t = sqrt(s > 0.0 ? s : 0.0);
    double phi = 2.0 * PI_D * u2;
    V3 t, b; onb(mdir, &t, &b);
    return vnorm(vadd(vadd(vmul(t, sin_t * cos(phi)), vmul(b, sin_t * sin(phi))), vmul(mdir, cos_t)));
}

/* MediumStack (medium_stack.h:17-47) */
#define STK_CAP 32
typedef struct { int mat[STK_CAP], pri[STK_CAP], n; } Stack;
static int stk_top_pri(const Stack* s) {
    int bp = INT_MIN;
    for (int i = 0; i < s->n; ++i) if (s->pri[i] > bp) bp = s->pri[i];
    return s->n ? bp : INT_MIN;
}
static int stk_top_mat(const Stack* s) {
    int bp = INT_MIN, bm = -1;
    for (int i = 0; i < s->n; ++i) if (s->pri[i] >= bp) { bp = s->pri[i]; bm = s->mat[i]; }
    return bm;
}
static void stk_push(Stack* s, int mi, int p) {
    if (s->n < STK_CAP) { s->mat[s->n] = mi; s->pri[s->n] = p; ++s->n; }
}
static void stk_pop_mat(Stack* s, int mi) {
    for (int i = s->n - 1; i >= 0; --i)
        if (s->mat[i] == mi) {
            for (int j = i; j < s->n - 1; ++j) { s->mat[j] = s->mat[j + 1]; s->pri[j] = s->pri[j + 1]; }
            --s->n; return;
        }
}

static inline double mat_ior(const fto_ctx* c, const ftb_material* m, double lam) {
    return m->ior >= 0 ? spec_eval(&c->S, m->ior, lam) : 1.5;   /* iorConstant(1.5) default */
}
static inline double clamp01(double x) { return x < 0 ? 0 : (x > 1 ? 1 : x); }
static inline double slot(const fto_ctx* c, int s, double lam, double dflt) {
    return s >= 0 ? spec_eval(&c->S, s, lam) : dflt;
}

/* Renderer::SpecVtx (render.h:878-902): the vertex a specular connection starts from -- a
 * surface (normal np) or a volume scatter (incoming direction win, HG g); shape() is the
 * vertex's angular factor toward wP, negative when wP leaves the wrong side. */
typedef struct { int volume; V3 np, win; double g; } SpecVtx;
static double vtx_shape(const SpecVtx* vt, V3 wP) {
    if (vt->volume) return hg_phase(vdot(vt->win, wP), vt->g);
    double cs = vdot(vt->np, wP);
    return cs <= 0.0 ? -1.0 : cs / PI_D;
}

/* Renderer::connectSpecularPlane + mirrorSeenAt + splatMirrorLegs, one wavelength
 * (render.h:1294-1380): vertex p reaches the pinhole by one reflection in the plane of
 * mirror mp -- through the eye's mirror image -- if the reflection point R lies in the
 * plane's box and in the image, the light leg p -> R is clear, and a closest hit from the
 * eye toward R lands on a planar mirror at R; the splat carries that mirror's reflectance. */
static void connect_specular_plane(Tr* T, const MPlane* mp, V3 p, const SpecVtx* vt, const double* lam,
                                   const double* beta, const double* w, int nup) {
    const fto_ctx* c = T->c;
    const Cam* cam = T->cam;
    const V3 eye = cam->eye;
    const double se = vdot(mp->n, eye) - mp->d;
    const double sp = vdot(mp->n, p) - mp->d;
    if (!(se * sp > 0.0)) return;
    const V3 eye_m = vsub(eye, vmul(mp->n, 2.0 * se));
    V3 wP = vsub(eye_m, p);
    const double D = vlen(wP);
    if (D < 1e-9) return;
    wP = vmul(wP, 1.0 / D);
    const double shape = vtx_shape(vt, wP);
    if (shape < 0.0) return;
    const double denom = vdot(mp->n, wP);
    if (fabs(denom) < 1e-12) return;
    const double dP = (mp->d - vdot(mp->n, p)) / denom;
    if (dP <= 1e-7 || dP >= D - 1e-7) return;
    const V3 R = vadd(p, vmul(wP, dP));
    if (R.x < mp->lo.x || R.x > mp->hi.x || R.y < mp->lo.y || R.y > mp->hi.y || R.z < mp->lo.z || R.z > mp->hi.z)
        return;
    int px, py; double cos_cam, dist2e;
    if (!cam_project(cam, R, &px, &py, &cos_cam, &dist2e)) return;
    const double omega = cam_pixel_solid_angle(cam, cos_cam);
    if (omega <= 0.0) return;
    const double dE = D - dP;
    const V3 wRE = vmul(vsub(eye, R), 1.0 / dE);
    T->rays++;
    if (occluded(c, vadd(p, vmul(wP, 1e-6)), wP, dP - 2e-6, 1e-6)) return;
    Hit hm;
    T->rays++;
    closest_hit(c, eye, vneg(wRE), 1e-6, &hm);
    if (!hm.valid) return;
    if (fabs(hm.t - dE) > 1e-4 * (1.0 + dE)) return;
    if (hm.mat < 0 || hm.mat >= c->n_mats || !planar_mirror(&c->mats[hm.mat])) return;
    const double inv_d2_omega = 1.0 / (D * D * omega);
    for (int i = 0; i < nup; ++i) {   /* every live wavelength (splatMirrorLegs) */
        const double refl = clamp01(slot(c, c->mats[hm.mat].reflect, lam[i], 0.5));
        double contrib = beta[i] * (w[i] * shape) * refl * inv_d2_omega;
        if (contrib <= 0.0) continue;
        if (c->n_med > 0) {
            contrib *= media_transmittance(T, p, wP, dP, lam[i]);
            contrib *= media_transmittance(T, R, wRE, dE, lam[i]);
        }
        film_add(T->film, px, py, cie_x(lam[i]) * contrib, cie_y(lam[i]) * contrib, cie_z(lam[i]) * contrib);
    }
}
/* camSpecularSplatAllVtxN (render.h:1515-1550), planar mirrors only (scenes with dielectric
 * or mirror spheres are outside this path): the vertex's nup live wavelengths */
static void cam_specular_splat(Tr* T, V3 p, const SpecVtx* vt, const double* lam, const double* beta,
                               const double* w, int nup) {
    for (int k = 0; k < T->c->n_mp; ++k) connect_specular_plane(T, &T->c->mp[k], p, vt, lam, beta, w, nup);
}
/* camSpecularSplatAll / camSpecularSplatAllHero (render.h:1559-1576): a surface vertex */
static void cam_specular_surface_n(Tr* T, V3 p, V3 n, const double* lam, const double* beta, const double* rho,
                                   int nup) {
    if (T->c->n_mp == 0) return;
    SpecVtx vt; vt.volume = 0; vt.np = n; vt.win = v3(0, 0, 0); vt.g = 0.0;
    cam_specular_splat(T, p, &vt, lam, beta, rho, nup);
}
static void cam_specular_surface(Tr* T, V3 p, V3 n, double lam, double beta, double rho) {
    cam_specular_surface_n(T, p, n, &lam, &beta, &rho, 1);
}

/* Renderer::refractOrReflect (render.h:2657-2697), stochastic branch */
static void refract_or_reflect(const fto_ctx* c, const ftb_material* m, const Hit* h, V3 d,
                               double lam, Pcg* rng, int* transmitted, double ext_ior,
                               V3* o_out, V3* d_out) {
    double ngi = mat_ior(c, m, lam);
    int entering = vdot(d, h->ng) < 0.0;
    V3 nl = entering ? h->ng : vneg(h->ng);
    double n1 = entering ? ext_ior : ngi;
    double n2 = entering ? ngi : ext_ior;
    double eta = n1 / n2;
    double cos_i = -vdot(d, nl);
    double sin2t = eta * eta * (1.0 - cos_i * cos_i);
    V3 out; int refracted = 0;
    if (sin2t > 1.0) {
        out = vreflect(d, nl);
    } else {
        double cos_t = sqrt(1.0 - sin2t);
        double rs = (n1 * cos_i - n2 * cos_t) / (n1 * cos_i + n2 * cos_t);
        double rp = (n1 * cos_t - n2 * cos_i) / (n1 * cos_t + n2 * cos_i);
        double R = 0.5 * (rs * rs + rp * rp);
        if (pcg_uniform(rng) < R) out = vreflect(d, nl);
        else { out = vadd(vmul(d, eta), vmul(nl, eta * cos_i - cos_t)); refracted = 1; }
    }
    out = vnorm(out);
    double rough = m->roughness;
    if (rough > 1e-3) {
        V3 pert = sample_glossy(out, rough, rng);
        int ok = refracted ? (vdot(pert, nl) < 0.0) : (vdot(pert, nl) > 0.0);
        if (ok) out = pert;
    }
    *transmitted = refracted;
    *o_out = vadd(h->p, vmul(out, 1e-6));
    *d_out = out;
}

static inline uint64_t fnv_i32(uint64_t h, int32_t v) {
    uint32_t u = (uint32_t)v;
    for (int i = 0; i < 4; ++i) { h ^= (u >> (8 * i)) & 0xffu; h *= 1099511628211ULL; }
    return h;
}
#define FNV_BASIS 1469598103934665603ULL

enum { E_EMIT = 0, E_ABS = 1, E_SENSOR = 2, E_ESC = 3, E_RES = 4 };

/* Renderer::tracePhoton, single wavelength (render.h:1811-2240) for the supported
 * subset: area emitters (quad / sphere), Diffuse, DiffuseTransmit, Dielectric (priority
 * stack, interior absorption, frosting), Glossy, Filter, homogeneous HG media. */
static void trace_photon(Tr* T, Pcg* rng, int max_bounce, double* e, ftb_photon_log* log) {
    const fto_ctx* c = T->c;
    uint64_t hash = FNV_BASIS;
    int nh = 0;
    if (log) { memset(log, 0, sizeof *log); log->fate = 4; for (int i = 0; i < 8; ++i) log->prims[i] = -2; }
    double grand_total = c->total_power;
    if (grand_total <= 0.0) return;
    if (c->n_emit == 0) return;
    /* Scene::selectEmitter (scene.h:1851-1857) */
    int ei = 0;
    if (c->n_emit > 1) {
        double u = pcg_uniform(rng);
        int lo = 0, hi = c->n_emit - 1;
        while (lo < hi) { int mid = (lo + hi) / 2; if (c->emitter_cdf[mid] < u) lo = mid + 1; else hi = mid; }
        ei = lo;
    }
    const Emit* em = &c->emit[ei];
    double u1 = pcg_uniform(rng), u2 = pcg_uniform(rng);
    V3 origin, emit_n, dir;
    /* Emitter::samplePoint (scene.h:815-880) */
    if (em->shape == FTB_EMIT_SPHERE) {
        double z = 1.0 - 2.0 * u1;
        double s = 1.0 - z * z;
        double r = sqrt(s > 0.0 ? s : 0.0);
        double phi = 2.0 * PI_D * u2;
        V3 d = v3(r * cos(phi), r * sin(phi), z);
        emit_n = d;
        origin = vadd(em->origin, vmul(d, em->radius));
    } else {
        origin = vadd(vadd(em->origin, vmul(em->u, u1)), vmul(em->v, u2));
        emit_n = em->normal;
    }
    dir = em->collimated ? em->beam : cosine_hemisphere(emit_n, rng);
    double pdf_l = 0.0, wl = 1.0;
    double ul = pcg_uniform(rng), lam;
    if (c->lambda_mode == FTB_LAMBDA_UNIFORM_380_780) {
        lam = emission_sample_band(em->cdf, em->n, em->step, ul, &wl);
        pdf_l = wl;
    } else {
        lam = emission_sample_at(em->cdf, em->n, em->step, ul, &pdf_l);
    }
    if (pdf_l <= 0) return;
    double beta = (c->n_emit == 1) ? em->power : c->total_power;
    beta *= 1.0;   /* spotW */
    if (c->lambda_mode == FTB_LAMBDA_UNIFORM_380_780) beta *= wl;
    e[E_EMIT] += beta;
    connect_surface(T, origin, emit_n, emit_n, emit_n, lam, beta, 1.0);
    cam_specular_surface(T, origin, emit_n, lam, beta, 1.0);
    V3 ro = vadd(origin, vmul(dir, 1e-6)), rd = dir;
    Stack stk; stk.n = 0;
    int fate = 2;
    for (int bounce = 0; bounce < max_bounce; ++bounce) {
        Hit h;
        T->rays++;
        int prim = closest_hit(c, ro, rd, 1e-6, &h);
        hash = fnv_i32(hash, prim);
        if (prim >= c->nt + c->ns + c->nc) hash = fnv_i32(hash, h.sub);   /* BLAS triangle */
        if (nh < 8 && log) log->prims[nh] = prim;
        ++nh;
        double d_surf = h.valid ? h.t : 1e30;
        double d_event = d_surf;
        int medium_event = 0, scatter_med = -1;
        V3 mp = v3(0, 0, 0);
        if (c->n_med > 0) {
            double tm; int which;
            if (sample_media_collision(T, ro, rd, d_surf, lam, rng, &tm, &which)) {
                d_event = tm; medium_event = 1; scatter_med = which; mp = vadd(ro, vmul(rd, tm));
            }
        }
        {   /* Beer-Lambert inside the current dielectric (render.h:2063-2066) */
            int mi = stk_top_mat(&stk);
            double a = (mi >= 0) ? slot(c, c->mats[mi].absorb, lam, 0.0) : 0.0;
            if (a > 0.0) beta *= exp(-a * d_event);
        }
        if (medium_event) {   /* render.h:2105-2115 */
            const Med* sm = &c->med[scatter_med];
            connect_volume(T, sm, mp, rd, lam, beta);
            if (c->n_mp > 0) {   /* camSpecularSplatVolumeAll (render.h:1580-1585) */
                SpecVtx vt; vt.volume = 1; vt.np = v3(0, 0, 0); vt.win = rd; vt.g = sm->g;
                const double alb = med_albedo(c, sm, lam);
                cam_specular_splat(T, mp, &vt, &lam, &beta, &alb, 1);
            }
            if (pcg_uniform(rng) >= med_albedo(c, sm, lam)) { e[E_ABS] += beta; fate = 0; goto done; }
            V3 nd = sample_hg(rd, sm->g, rng);
            ro = mp; rd = nd;
            continue;
        }
        if (!h.valid) { e[E_ESC] += beta; fate = 1; goto done; }
        const ftb_material* m = &c->mats[h.mat];
        switch (m->type) {
        case FTB_MAT_DIELECTRIC: {   /* render.h:1612-1660 */
            int entering = vdot(rd, h.ng) < 0.0;
            int mi = h.mat, pr = m->priority;
            int has_pri = pr != INT_MIN;
            V3 no, nd; int transmitted = 0;
            if (entering) {
                int out_mat = stk_top_mat(&stk), out_pri = stk_top_pri(&stk);
                int ranked = has_pri && (stk.n == 0 || (out_mat >= 0 && c->mats[out_mat].priority != INT_MIN));
                if (ranked && stk.n != 0 && pr <= out_pri) {
                    stk_push(&stk, mi, pr);
                    ro = vadd(h.p, vmul(rd, 1e-6));
                    continue;
                }
                double ext = (ranked && out_mat >= 0) ? mat_ior(c, &c->mats[out_mat], lam) : 1.0;
                refract_or_reflect(c, m, &h, rd, lam, rng, &transmitted, ext, &no, &nd);
                ro = no; rd = nd;
                if (transmitted) stk_push(&stk, mi, pr);
            } else {
                Stack after = stk;
                stk_pop_mat(&after, mi);
                int new_mat = stk_top_mat(&after), new_pri = stk_top_pri(&after);
                int ranked = has_pri && (after.n == 0 || (new_mat >= 0 && c->mats[new_mat].priority != INT_MIN));
                if (ranked && new_mat >= 0 && pr <= new_pri) {
                    stk_pop_mat(&stk, mi);
                    ro = vadd(h.p, vmul(rd, 1e-6));
                    continue;
                }
                double ext = (ranked && new_mat >= 0) ? mat_ior(c, &c->mats[new_mat], lam) : 1.0;
                refract_or_reflect(c, m, &h, rd, lam, rng, &transmitted, ext, &no, &nd);
                ro = no; rd = nd;
                if (transmitted) stk_pop_mat(&stk, mi);
            }
            continue;
        }
        case FTB_MAT_GLOSSY: {   /* render.h:1725-1733 */
            double r = clamp01(slot(c, m->reflect, lam, 0.5));
            if (pcg_uniform(rng) >= r) { e[E_ABS] += beta; fate = 0; goto done; }
            V3 o = sample_glossy(vreflect(rd, h.n), m->roughness, rng);
            if (vdot(o, h.n) <= 0) { e[E_ABS] += beta; fate = 0; goto done; }
            ro = vadd(h.p, vmul(h.n, 1e-6)); rd = o;
            continue;
        }
        case FTB_MAT_MIRROR: {   /* render.h:1680-1688 */
            double r = clamp01(slot(c, m->reflect, lam, 0.5));
            if (pcg_uniform(rng) >= r) { e[E_ABS] += beta; fate = 0; goto done; }
            V3 o = vreflect(rd, h.n);
            ro = vadd(h.p, vmul(h.n, 1e-6)); rd = o;
            continue;
        }
        case FTB_MAT_HALF_MIRROR: {   /* render.h:1702-1711 */
            double r = clamp01(slot(c, m->reflect, lam, 0.5));
            if (pcg_uniform(rng) < r) {
                V3 o = vreflect(rd, h.n);
                ro = vadd(h.p, vmul(h.n, 1e-6)); rd = o;
            } else {
                ro = vadd(h.p, vmul(rd, 1e-6));
            }
            continue;
        }
        case FTB_MAT_FILTER: {   /* render.h:1711-1723 */
            double t = clamp01(slot(c, m->transmit, lam, 0.0));
            if (pcg_uniform(rng) >= t) { e[E_ABS] += beta; fate = 0; goto done; }
            ro = vadd(h.p, vmul(rd, 1e-6));
            continue;
        }
        case FTB_MAT_DIFFUSE_TRANSMIT: {   /* render.h:2180-2212 */
            double rr = clamp01(slot(c, m->reflect, lam, 0.5));
            double rt = clamp01(slot(c, m->transmit, lam, 0.0));
            double sum = rr + rt;
            if (sum > 1.0) { rr /= sum; rt /= sum; sum = 1.0; }
            V3 ngo = oriented_geo_n(&h);
            V3 wi = v3(-rd.x, -rd.y, -rd.z);
            connect_surface(T, h.p, h.n, ngo, wi, lam, beta, rr);
            connect_surface(T, h.p, vneg(h.n), vneg(ngo), wi, lam, beta, rt);
            cam_specular_surface(T, h.p, h.n, lam, beta, rr);
            cam_specular_surface(T, h.p, vneg(h.n), lam, beta, rt);
            double u = pcg_uniform(rng);
            if (u < rr) {
                V3 wo = cosine_hemisphere(h.n, rng);
                beta *= shading_adjoint_corr(wi, wo, h.n, ngo);
                ro = vadd(h.p, vmul(h.n, 1e-6)); rd = wo;
                continue;
            } else if (u < sum) {
                V3 wo = cosine_hemisphere(v3(-h.n.x, -h.n.y, -h.n.z), rng);
                beta *= shading_adjoint_corr(wi, wo, h.n, ngo);
                ro = vsub(h.p, vmul(h.n, 1e-6)); rd = wo;
                continue;
            }
            e[E_ABS] += beta; fate = 0; goto done;
        }
        case FTB_MAT_DIFFUSE:
        default: {   /* render.h:2215-2236 */
            double rho = clamp01(slot(c, m->reflect, lam, 0.5));
            V3 ngo = oriented_geo_n(&h);
            V3 wi = v3(-rd.x, -rd.y, -rd.z);
            connect_surface(T, h.p, h.n, ngo, wi, lam, beta, rho);
            cam_specular_surface(T, h.p, h.n, lam, beta, rho);
            if (pcg_uniform(rng) >= rho) { e[E_ABS] += beta; fate = 0; goto done; }
            V3 wo = cosine_hemisphere(h.n, rng);
            beta *= shading_adjoint_corr(wi, wo, h.n, ngo);
            ro = vadd(h.p, vmul(h.n, 1e-6)); rd = wo;
            continue;
        }
        }
    }
    e[E_RES] += beta;
    fate = 2;
done:
    if (log) { log->n_hits = nh; log->fate = fate; log->prim_hash = hash; log->beta = beta; }
}

/* ------------------------------------------------------------- setup ---------------- */
void fto_release(fto_ctx* c) {
    if (!c) return;
    free(c->mp);
    free(c->spec); free(c->tw); free(c->tv); free(c->mats); free(c->tris); free(c->sph);
    free(c->sph_mat); free(c->crv); free(c->world.nodes); free(c->world.order); free(c->emit);
    free(c->cdf_store); free(c->emitter_cdf); free(c->med);
    for (int b = 0; b < c->n_blas; ++b) {
        free(c->blas[b].tris); free(c->blas[b].tree.nodes); free(c->blas[b].tree.order);
    }
    free(c->blas); free(c->inst);
    free(c);
}

static V3 rd3(const double* p) { return v3(p[0], p[1], p[2]); }

/* Tri::finalize (geometry.h:51-55): geometric normal; missing shading normals take it */
static void finalize_tri(Tri* t, const double* v, const double* n, int mat) {
    t->v0 = rd3(v); t->v1 = rd3(v + 3); t->v2 = rd3(v + 6);
    t->mat = mat;
    t->gn = vnorm(vcross(vsub(t->v1, t->v0), vsub(t->v2, t->v0)));
    V3 z = v3(0, 0, 0);
    t->n0 = z; t->n1 = z; t->n2 = z;
    if (n) { t->n0 = rd3(n); t->n1 = rd3(n + 3); t->n2 = rd3(n + 6); }
    if (vdot(t->n0, t->n0) < 1e-12) t->n0 = t->gn;
    if (vdot(t->n1, t->n1) < 1e-12) t->n1 = t->gn;
    if (vdot(t->n2, t->n2) < 1e-12) t->n2 = t->gn;
}

static int cmp_plane_area(const void* a, const void* b) {
    const MPlane* x = (const MPlane*)a;
    const MPlane* y = (const MPlane*)b;
    if (x->area != y->area) return x->area < y->area ? 1 : -1;   /* larger area first */
    return (x->key[0] > y->key[0]) - (x->key[0] < y->key[0]);   /* then first seen */
}

/* Scene::buildMirrorPlanes (scene.h:1646-1720): the planar-mirror triangles grouped by
 * plane (unit normal flipped so its largest component is positive, offset d = dot(n, v0),
 * bucketed by the quantized (n, d) key in first-seen order), each plane's AABB over its
 * member vertices and total area; at most 64 planes (the largest by area; the reference's
 * sort is not stable, so a tie in area at the cut is ordered by first sighting here); the
 * boxes padded by 1e-6 (1 + diagonal). */
static void build_mirror_planes(fto_ctx* c) {
    c->n_mp = 0;
    c->mp = NULL;
    int cap = 0;
    for (int64_t i = 0; i < c->nt; ++i) {
        const Tri* t = &c->tris[i];
        if (t->mat < 0 || t->mat >= c->n_mats || !planar_mirror(&c->mats[t->mat])) continue;
        V3 n = t->gn;
        double nl = vlen(n);
        if (nl < 1e-12) continue;
        n = vmul(n, 1.0 / nl);
        const double sx = fabs(n.x), sy = fabs(n.y), sz = fabs(n.z);
        const double lead = (sx >= sy && sx >= sz) ? n.x : ((sy >= sz) ? n.y : n.z);
        if (lead < 0.0) n = v3(-n.x, -n.y, -n.z);
        double d = vdot(n, t->v0);
        const double q_pos = 1e5, q_dir = 1e6;
        long long key[4] = {llround(n.x * q_dir), llround(n.y * q_dir), llround(n.z * q_dir), llround(d * q_pos)};
        int idx = -1;
        for (int k = 0; k < c->n_mp && idx < 0; ++k)
            if (memcmp(c->mp[k].key, key, sizeof key) == 0) idx = k;
        if (idx < 0) {
            if (c->n_mp == cap) {
                cap = cap ? 2 * cap : 8;
                c->mp = (MPlane*)realloc(c->mp, sizeof(MPlane) * (size_t)cap);
            }
            idx = c->n_mp++;
            MPlane* m = &c->mp[idx];
            m->n = n; m->d = d; m->lo = t->v0; m->hi = t->v0; m->area = 0.0;
            memcpy(m->key, key, sizeof key);
        }
        MPlane* m = &c->mp[idx];
        const V3 vs[3] = {t->v0, t->v1, t->v2};
        for (int k = 0; k < 3; ++k) {   /* std::min(lo, v) / std::max(hi, v) */
            m->lo.x = vs[k].x < m->lo.x ? vs[k].x : m->lo.x; m->hi.x = m->hi.x < vs[k].x ? vs[k].x : m->hi.x;
            m->lo.y = vs[k].y < m->lo.y ? vs[k].y : m->lo.y; m->hi.y = m->hi.y < vs[k].y ? vs[k].y : m->hi.y;
            m->lo.z = vs[k].z < m->lo.z ? vs[k].z : m->lo.z; m->hi.z = m->hi.z < vs[k].z ? vs[k].z : m->hi.z;
        }
        m->area += 0.5 * vlen(vcross(vsub(t->v1, t->v0), vsub(t->v2, t->v0)));
    }
    if (c->n_mp > 64) {
        /* qsort is not stable: ties fall back to the first-seen index, kept in key[0] */
        for (int k = 0; k < c->n_mp; ++k) c->mp[k].key[0] = k;
        qsort(c->mp, (size_t)c->n_mp, sizeof(MPlane), cmp_plane_area);
        c->n_mp = 64;
    }
    for (int k = 0; k < c->n_mp; ++k) {
        MPlane* m = &c->mp[k];
        const double pad = 1e-6 * (1.0 + vlen(vsub(m->hi, m->lo)));
        m->lo = vsub(m->lo, v3(pad, pad, pad));
        m->hi = vadd(m->hi, v3(pad, pad, pad));
    }
}

int fto_mirror_planes(const fto_ctx* c, double* out, int cap) {
    if (!c) return -1;
    for (int k = 0; k < c->n_mp && k < cap; ++k) {
        const MPlane* m = &c->mp[k];
        double* o = out + 10 * k;
        o[0] = m->n.x; o[1] = m->n.y; o[2] = m->n.z; o[3] = m->d;
        o[4] = m->lo.x; o[5] = m->lo.y; o[6] = m->lo.z; o[7] = m->hi.x; o[8] = m->hi.y; o[9] = m->hi.z;
    }
    return c->n_mp;
}

fto_ctx* fto_prepare(const ftb_scene_desc* d) {
    if (!d) { fail("null desc"); return NULL; }
    fto_ctx* c = (fto_ctx*)calloc(1, sizeof(fto_ctx));
    if (!c) return NULL;
    /* spectra */
    c->spec = (ftb_spectrum*)malloc(sizeof(ftb_spectrum) * (size_t)(d->n_spectra > 0 ? d->n_spectra : 1));
    memcpy(c->spec, d->spectra, sizeof(ftb_spectrum) * (size_t)d->n_spectra);
    size_t nt = (size_t)(d->n_table > 0 ? d->n_table : 1);
    c->tw = (double*)calloc(nt, sizeof(double)); c->tv = (double*)calloc(nt, sizeof(double));
    if (d->n_table > 0) {
        memcpy(c->tw, d->table_w, sizeof(double) * (size_t)d->n_table);
        memcpy(c->tv, d->table_v, sizeof(double) * (size_t)d->n_table);
    }
    c->S.spec = c->spec; c->S.tw = c->tw; c->S.tv = c->tv; c->S.nspec = d->n_spectra;
    for (int i = 0; i < d->n_spectra; ++i)
        if (!spec_ok(d, i)) { fail("bad spectrum"); fto_release(c); return NULL; }
    /* materials */
    c->n_mats = d->n_mats;
    c->mats = (ftb_material*)malloc(sizeof(ftb_material) * (size_t)(d->n_mats > 0 ? d->n_mats : 1));
    memcpy(c->mats, d->mats, sizeof(ftb_material) * (size_t)d->n_mats);
    /* triangles: Tri::finalize (geometry.h:51-55) */
    c->nt = d->n_tris; c->ns = d->n_spheres; c->nc = d->n_curves;
    c->tris = (Tri*)malloc(sizeof(Tri) * (size_t)(c->nt > 0 ? c->nt : 1));
    for (int64_t i = 0; i < c->nt; ++i) {
        finalize_tri(&c->tris[i], d->tri_v + 9 * i, d->tri_n ? d->tri_n + 9 * i : NULL, d->tri_mat[i]);
        if (d->tri_mat[i] < 0 || d->tri_mat[i] >= d->n_mats) {
            fail("tri material out of range"); fto_release(c); return NULL;
        }
    }
    c->sph = (double*)malloc(sizeof(double) * 4 * (size_t)(c->ns > 0 ? c->ns : 1));
    c->sph_mat = (int*)malloc(sizeof(int) * (size_t)(c->ns > 0 ? c->ns : 1));
    if (c->ns) { memcpy(c->sph, d->sph, sizeof(double) * 4 * (size_t)c->ns);
                 for (int64_t i = 0; i < c->ns; ++i) c->sph_mat[i] = d->sph_mat[i]; }
    c->crv = (Crv*)malloc(sizeof(Crv) * (size_t)(c->nc > 0 ? c->nc : 1));
    for (int64_t i = 0; i < c->nc; ++i) {
        const double* s = d->curve + 10 * i;
        Crv* k = &c->crv[i];
        k->p0 = rd3(s); k->p1 = rd3(s + 3); k->r0 = s[6]; k->r1 = s[7];
        k->u0 = (double)(float)s[8]; k->u1 = (double)(float)s[9];
        k->mat = d->curve_mat[i];
    }
    /* BLAS assets (scene.h:996-1015) and instances (scene.h:1035-1063) */
    c->n_blas = d->n_blas > 0 ? d->n_blas : 0;
    c->ni = d->n_instances > 0 ? d->n_instances : 0;
    c->blas = (Blas*)calloc((size_t)(c->n_blas > 0 ? c->n_blas : 1), sizeof(Blas));
    c->inst = (Inst*)calloc((size_t)(c->ni > 0 ? c->ni : 1), sizeof(Inst));
    for (int b = 0; b < c->n_blas; ++b) {
        const ftb_blas_desc* bd = &d->blas[b];
        Blas* B = &c->blas[b];
        B->nt = bd->n_tris;
        B->tris = (Tri*)malloc(sizeof(Tri) * (size_t)(B->nt > 0 ? B->nt : 1));
        B->lo = v3(DBL_MAX, DBL_MAX, DBL_MAX);
        B->hi = v3(-DBL_MAX, -DBL_MAX, -DBL_MAX);
        BPrim* bp = (BPrim*)malloc(sizeof(BPrim) * (size_t)(B->nt > 0 ? B->nt : 1));
        for (int64_t i = 0; i < B->nt; ++i) {
            if (bd->tri_mat[i] < 0 || bd->tri_mat[i] >= d->n_mats) {
                fail("blas tri material out of range"); free(bp); fto_release(c); return NULL;
            }
            finalize_tri(&B->tris[i], bd->tri_v + 9 * i, bd->tri_n ? bd->tri_n + 9 * i : NULL, bd->tri_mat[i]);
            V3 lo, hi;
            tri_box(&B->tris[i], &lo, &hi);
            lo = v3(lo.x - 1e-6, lo.y - 1e-6, lo.z - 1e-6);
            hi = v3(hi.x + 1e-6, hi.y + 1e-6, hi.z + 1e-6);
            B->lo = v3(fmin(B->lo.x, lo.x), fmin(B->lo.y, lo.y), fmin(B->lo.z, lo.z));
            B->hi = v3(fmax(B->hi.x, hi.x), fmax(B->hi.y, hi.y), fmax(B->hi.z, hi.z));
            bp[i].lo = lo; bp[i].hi = hi; bp[i].c = vmul(vadd(lo, hi), 0.5); bp[i].idx = (int)i;
        }
        build_tree(&B->tree, bp, (int)B->nt);
        free(bp);
    }
    for (int64_t k = 0; k < c->ni; ++k) {
        const ftb_instance* id = &d->instances[k];
        if (id->blas < 0 || id->blas >= c->n_blas || id->mat_override >= d->n_mats) {
            fail("instance out of range"); fto_release(c); return NULL;
        }
        Inst* in = &c->inst[k];
        in->blas = id->blas;
        in->mat_override = id->mat_override;
        memcpy(in->to_world.m, id->to_world, sizeof(double) * 9);
        in->to_world.t = v3(id->to_world[9], id->to_world[10], id->to_world[11]);
        in->to_local = aff_inverse(&in->to_world);
    }
    c->np = c->nt + c->ns + c->nc + c->ni;
    /* world tree over tris, spheres, curves, instances */
    if (c->np > 0) {
        BPrim* bp = (BPrim*)malloc(sizeof(BPrim) * (size_t)c->np);
        for (int64_t i = 0; i < c->np; ++i) {
            box_of(c, (int)i, &bp[i].lo, &bp[i].hi);
            bp[i].c = vmul(vadd(bp[i].lo, bp[i].hi), 0.5);
            bp[i].idx = (int)i;
        }
        build_tree(&c->world, bp, (int)c->np);
        free(bp);
    }
    /* emitters + selection CDF (scene.h:1491-1513) */
    c->n_emit = d->n_emitters;
    c->emit = (Emit*)calloc((size_t)(c->n_emit > 0 ? c->n_emit : 1), sizeof(Emit));
    c->emitter_cdf = (double*)calloc((size_t)(c->n_emit > 0 ? c->n_emit : 1), sizeof(double));
    int64_t cdf_total = 0;
    for (int i = 0; i < c->n_emit; ++i) cdf_total += d->emitters[i].cdf_n + 1;
    c->cdf_store = (double*)malloc(sizeof(double) * (size_t)(cdf_total > 0 ? cdf_total : 1));
    int64_t off = 0;
    double tp = 0.0;
    for (int i = 0; i < c->n_emit; ++i) {
        const ftb_emitter* s = &d->emitters[i];
        Emit* k = &c->emit[i];
        k->shape = s->shape; k->collimated = s->collimated; k->n = s->cdf_n;
        k->step = s->step; k->power = s->power; k->area = s->area; k->radius = s->radius;
        k->origin = rd3(s->origin); k->u = rd3(s->u); k->v = rd3(s->v);
        k->normal = rd3(s->normal); k->beam = rd3(s->beam);
        memcpy(c->cdf_store + off, d->emitter_cdf + s->cdf_offset, sizeof(double) * (size_t)(s->cdf_n + 1));
        k->cdf = c->cdf_store + off;
        off += s->cdf_n + 1;
        tp += k->power;
        c->emitter_cdf[i] = tp;
    }
    c->total_power = tp;
    if (tp > 0) for (int i = 0; i < c->n_emit; ++i) c->emitter_cdf[i] /= tp;
    /* media */
    c->n_med = d->n_media;
    c->med = (Med*)calloc((size_t)(c->n_med > 0 ? c->n_med : 1), sizeof(Med));
    for (int i = 0; i < c->n_med; ++i) {
        const ftb_medium* s = &d->media[i];
        Med* m = &c->med[i];
        m->g = s->g; m->sa = s->sigma_a; m->ss = s->sigma_s; m->bound = s->bound;
        m->bmin = rd3(s->bmin); m->bmax = rd3(s->bmax); m->center = rd3(s->center); m->radius = s->radius;
    }
    build_mirror_planes(c);
    return c;
}

/* ------------------------------------------------------------- hero wavelengths ----- */
#define HERO_MAX 8

/* connectHero (render.h:564-577): one connectGeom (render.h:499-536), then every live
 * wavelength splats with its own beta and reflectance.  Hero bundles never run with media. */
static void connect_surface_hero(Tr* T, V3 p, V3 n, V3 ng, V3 wi, const double* lam, const double* beta,
                                 const double* rho, int nup) {
    const Cam* cam = T->cam;
    V3 to_cam = vsub(cam->eye, p);
    double dist = vlen(to_cam);
    V3 wdir = vdiv(to_cam, dist);
    double cos_surf = vdot(n, wdir);
    if (cos_surf <= 0) return;
    double stg = shadow_terminator_g(wdir, n, ng);
    if (stg <= 0.0) return;
    int px, py; double cos_cam, dist2;
    if (!cam_project(cam, p, &px, &py, &cos_cam, &dist2)) return;
    T->rays++;
    if (occluded(T->c, vadd(p, vmul(ng, 1e-6)), wdir, dist - 2e-6, 1e-6)) return;
    double omega = cam_pixel_solid_angle(cam, cos_cam);
    double corr = shading_adjoint_corr(wi, wdir, n, ng);
    double denom = dist2 * omega;
    for (int i = 0; i < nup; ++i) {
        double f = rho[i] / PI_D;
        double contrib = beta[i] * f * cos_surf * corr / denom * stg;
        film_add(T->film, px, py, cie_x(lam[i]) * contrib, cie_y(lam[i]) * contrib, cie_z(lam[i]) * contrib);
    }
}

/* the energy of the live wavelengths (activeSum, render.h:2324-2325) */
static inline double active_sum(const double* beta, int n) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += beta[i];
    return s;
}

static inline double max_of(const double* a, int n) {   /* hero::maxOf (hero.h:120-126) */
    double m = a[0];
    for (int i = 1; i < n; ++i) if (a[i] > m) m = a[i];
    return m;
}

/* Renderer::tracePhotonHero + tracePhotonHeroLoop (render.h:2252-2631) for the materials on
 * this path: C wavelengths per photon (hero.h sampleBundle), geometry decided by the hero,
 * analog RR on the max over live wavelengths with bounded reweights booked as absorption,
 * and a dielectric de-heroes (the hero continues alone, boosted x C). */
static void trace_photon_hero(Tr* T, Pcg* rng, int max_bounce, int C, double* e, ftb_photon_log* log) {
    const fto_ctx* c = T->c;
    uint64_t hash = FNV_BASIS;
    int nh = 0;
    if (log) { memset(log, 0, sizeof *log); log->fate = 4; for (int i = 0; i < 8; ++i) log->prims[i] = -2; }
    if (c->total_power <= 0.0 || c->n_emit == 0) return;
    int ei = 0;
    if (c->n_emit > 1) {
        double u = pcg_uniform(rng);
        int lo = 0, hi = c->n_emit - 1;
        while (lo < hi) { int mid = (lo + hi) / 2; if (c->emitter_cdf[mid] < u) lo = mid + 1; else hi = mid; }
        ei = lo;
    }
    const Emit* em = &c->emit[ei];
    double u1 = pcg_uniform(rng), u2 = pcg_uniform(rng);
    V3 origin, emit_n, dir;
    if (em->shape == FTB_EMIT_SPHERE) {
        double z = 1.0 - 2.0 * u1;
        double s = 1.0 - z * z;
        double r = sqrt(s > 0.0 ? s : 0.0);
        double phi = 2.0 * PI_D * u2;
        V3 d = v3(r * cos(phi), r * sin(phi), z);
        emit_n = d;
        origin = vadd(em->origin, vmul(d, em->radius));
    } else {
        origin = vadd(vadd(em->origin, vmul(em->u, u1)), vmul(em->v, u2));
        emit_n = em->normal;
    }
    dir = em->collimated ? em->beam : cosine_hemisphere(emit_n, rng);
    /* hero::sampleBundle (hero.h:100-113): one variate, strata u + i/C wrapped */
    double lam[HERO_MAX], pdf[HERO_MAX], beta[HERO_MAX], wl[HERO_MAX];
    const int band = c->lambda_mode == FTB_LAMBDA_UNIFORM_380_780;
    double u = pcg_uniform(rng);
    pdf[0] = 0.0;
    if (band) { lam[0] = emission_sample_band(em->cdf, em->n, em->step, u, &wl[0]); pdf[0] = wl[0]; }
    else lam[0] = emission_sample_at(em->cdf, em->n, em->step, u, &pdf[0]);
    if (pdf[0] <= 0.0) return;
    for (int i = 1; i < C; ++i) {
        double uu = u + (double)i / (double)C;
        if (uu >= 1.0) uu -= 1.0;
        pdf[i] = 0.0;
        if (band) lam[i] = emission_sample_band(em->cdf, em->n, em->step, uu, &wl[i]);
        else lam[i] = emission_sample_at(em->cdf, em->n, em->step, uu, &pdf[i]);
    }
    double base = (c->n_emit == 1) ? em->power : c->total_power;
    base *= 1.0;   /* spotW */
    for (int i = 0; i < C; ++i) {
        beta[i] = base / C;
        if (band) beta[i] *= wl[i];
    }
    int sec_alive = C > 1;
    e[E_EMIT] += active_sum(beta, sec_alive ? C : 1);
    {
        double one[HERO_MAX];
        for (int i = 0; i < C; ++i) one[i] = 1.0;
        connect_surface_hero(T, origin, emit_n, emit_n, emit_n, lam, beta, one, C);
        cam_specular_surface_n(T, origin, emit_n, lam, beta, one, C);
    }
    V3 ro = vadd(origin, vmul(dir, 1e-6)), rd = dir;
    Stack stk; stk.n = 0;
    int fate = 2;
    for (int bounce = 0; bounce < max_bounce; ++bounce) {
        int nup = sec_alive ? C : 1;
        Hit h;
        T->rays++;
        int prim = closest_hit(c, ro, rd, 1e-6, &h);
        hash = fnv_i32(hash, prim);
        if (prim >= c->nt + c->ns + c->nc) hash = fnv_i32(hash, h.sub);
        if (nh < 8 && log) log->prims[nh] = prim;
        ++nh;
        double d_event = h.valid ? h.t : 1e30;
        {   /* Beer-Lambert per live wavelength (render.h:2389-2398) */
            int mi = stk_top_mat(&stk);
            if (mi >= 0)
                for (int i = 0; i < nup; ++i) {
                    double a = slot(c, c->mats[mi].absorb, lam[i], 0.0);
                    if (a > 0.0) beta[i] *= exp(-a * d_event);
                }
        }
        if (!h.valid) { e[E_ESC] += active_sum(beta, sec_alive ? C : 1); fate = 1; goto done; }
        const ftb_material* m = &c->mats[h.mat];
        switch (m->type) {
        case FTB_MAT_DIFFUSE_TRANSMIT: {   /* render.h:2454-2503 */
            double rho_r[HERO_MAX] = {0}, rho_t[HERO_MAX] = {0};
            for (int i = 0; i < nup; ++i) {
                double rr = clamp01(slot(c, m->reflect, lam[i], 0.5));
                double rt = clamp01(slot(c, m->transmit, lam[i], 0.0));
                double s = rr + rt;
                if (s > 1.0) { rr /= s; rt /= s; }
                rho_r[i] = rr; rho_t[i] = rt;
            }
            V3 ngo = oriented_geo_n(&h);
            V3 wi = v3(-rd.x, -rd.y, -rd.z);
            connect_surface_hero(T, h.p, h.n, ngo, wi, lam, beta, rho_r, nup);
            connect_surface_hero(T, h.p, vneg(h.n), vneg(ngo), wi, lam, beta, rho_t, nup);
            cam_specular_surface_n(T, h.p, h.n, lam, beta, rho_r, nup);
            cam_specular_surface_n(T, h.p, vneg(h.n), lam, beta, rho_t, nup);
            double q_r = max_of(rho_r, nup), q_t = max_of(rho_t, nup);
            double sum_h = q_r + q_t;
            if (nup > 1 && sum_h > 1.0) { q_r /= sum_h; q_t /= sum_h; sum_h = q_r + q_t; }
            double uu = pcg_uniform(rng);
            if (uu < q_r) {
                for (int i = 0; i < nup; ++i) {
                    double w = rho_r[i] / q_r;
                    e[E_ABS] += beta[i] * (1.0 - w);
                    beta[i] *= w;
                }
                V3 wo = cosine_hemisphere(h.n, rng);
                double corr = shading_adjoint_corr(wi, wo, h.n, ngo);
                for (int i = 0; i < nup; ++i) beta[i] *= corr;
                ro = vadd(h.p, vmul(h.n, 1e-6)); rd = wo;
                continue;
            } else if (uu < sum_h) {
                for (int i = 0; i < nup; ++i) {
                    double w = rho_t[i] / q_t;
                    e[E_ABS] += beta[i] * (1.0 - w);
                    beta[i] *= w;
                }
                V3 wo = cosine_hemisphere(v3(-h.n.x, -h.n.y, -h.n.z), rng);
                double corr = shading_adjoint_corr(wi, wo, h.n, ngo);
                for (int i = 0; i < nup; ++i) beta[i] *= corr;
                ro = vsub(h.p, vmul(h.n, 1e-6)); rd = wo;
                continue;
            }
            e[E_ABS] += active_sum(beta, sec_alive ? C : 1); fate = 0; goto done;
        }
        case FTB_MAT_MIRROR:
        case FTB_MAT_FILTER:
        case FTB_MAT_GLOSSY: {   /* achromatic lobes (render.h:2509-2537) */
            double cc[HERO_MAX] = {0};
            for (int i = 0; i < nup; ++i)
                cc[i] = (m->type == FTB_MAT_FILTER) ? clamp01(slot(c, m->transmit, lam[i], 0.0))
                                                     : clamp01(slot(c, m->reflect, lam[i], 0.5));
            double q = max_of(cc, nup);
            if (pcg_uniform(rng) >= q) { e[E_ABS] += active_sum(beta, sec_alive ? C : 1); fate = 0; goto done; }
            for (int i = 0; i < nup; ++i) {
                double w = cc[i] / q;
                e[E_ABS] += beta[i] * (1.0 - w);
                beta[i] *= w;
            }
            if (m->type == FTB_MAT_MIRROR) {
                ro = vadd(h.p, vmul(h.n, 1e-6)); rd = vreflect(rd, h.n);
            } else if (m->type == FTB_MAT_FILTER) {
                ro = vadd(h.p, vmul(rd, 1e-6));
            } else {
                V3 o = sample_glossy(vreflect(rd, h.n), m->roughness, rng);
                if (vdot(o, h.n) <= 0) { e[E_ABS] += active_sum(beta, sec_alive ? C : 1); fate = 0; goto done; }
                ro = vadd(h.p, vmul(h.n, 1e-6)); rd = o;
            }
            continue;
        }
        case FTB_MAT_HALF_MIRROR: {   /* de-hero, then the scalar half mirror (render.h:2546-2589, 1702-1711) */
            if (sec_alive) { beta[0] *= (double)C; sec_alive = 0; }
            double r = clamp01(slot(c, m->reflect, lam[0], 0.5));
            if (pcg_uniform(rng) < r) {
                V3 o = vreflect(rd, h.n);
                ro = vadd(h.p, vmul(h.n, 1e-6)); rd = o;
            } else {
                ro = vadd(h.p, vmul(rd, 1e-6));
            }
            continue;
        }
        case FTB_MAT_DIELECTRIC: {   /* de-hero, then the scalar interaction (render.h:2539-2589) */
            if (sec_alive) { beta[0] *= (double)C; sec_alive = 0; }
            const double lam0 = lam[0];
            int entering = vdot(rd, h.ng) < 0.0;
            int mi = h.mat, pr = m->priority;
            int has_pri = pr != INT_MIN;
            V3 no, nd; int transmitted = 0;
            if (entering) {
                int out_mat = stk_top_mat(&stk), out_pri = stk_top_pri(&stk);
                int ranked = has_pri && (stk.n == 0 || (out_mat >= 0 && c->mats[out_mat].priority != INT_MIN));
                if (ranked && stk.n != 0 && pr <= out_pri) {
                    stk_push(&stk, mi, pr);
                    ro = vadd(h.p, vmul(rd, 1e-6));
                    continue;
                }
                double ext = (ranked && out_mat >= 0) ? mat_ior(c, &c->mats[out_mat], lam0) : 1.0;
                refract_or_reflect(c, m, &h, rd, lam0, rng, &transmitted, ext, &no, &nd);
                ro = no; rd = nd;
                if (transmitted) stk_push(&stk, mi, pr);
            } else {
                Stack after = stk;
                stk_pop_mat(&after, mi);
                int new_mat = stk_top_mat(&after), new_pri = stk_top_pri(&after);
                int ranked = has_pri && (after.n == 0 || (new_mat >= 0 && c->mats[new_mat].priority != INT_MIN));
                if (ranked && new_mat >= 0 && pr <= new_pri) {
                    stk_pop_mat(&stk, mi);
                    ro = vadd(h.p, vmul(rd, 1e-6));
                    continue;
                }
                double ext = (ranked && new_mat >= 0) ? mat_ior(c, &c->mats[new_mat], lam0) : 1.0;
                refract_or_reflect(c, m, &h, rd, lam0, rng, &transmitted, ext, &no, &nd);
                ro = no; rd = nd;
                if (transmitted) stk_pop_mat(&stk, mi);
            }
            continue;
        }
        case FTB_MAT_DIFFUSE:
        default: {   /* render.h:2591-2625 */
            double rho[HERO_MAX] = {0};
            for (int i = 0; i < nup; ++i) rho[i] = clamp01(slot(c, m->reflect, lam[i], 0.5));
            V3 ngo = oriented_geo_n(&h);
            V3 wi = v3(-rd.x, -rd.y, -rd.z);
            connect_surface_hero(T, h.p, h.n, ngo, wi, lam, beta, rho, nup);
            cam_specular_surface_n(T, h.p, h.n, lam, beta, rho, nup);
            double q = max_of(rho, nup);
            if (pcg_uniform(rng) >= q) { e[E_ABS] += active_sum(beta, sec_alive ? C : 1); fate = 0; goto done; }
            for (int i = 0; i < nup; ++i) {
                double w = rho[i] / q;
                e[E_ABS] += beta[i] * (1.0 - w);
                beta[i] *= w;
            }
            V3 wo = cosine_hemisphere(h.n, rng);
            double corr = shading_adjoint_corr(wi, wo, h.n, ngo);
            for (int i = 0; i < nup; ++i) beta[i] *= corr;
            ro = vadd(h.p, vmul(h.n, 1e-6)); rd = wo;
            continue;
        }
        }
    }
    e[E_RES] += active_sum(beta, sec_alive ? C : 1);
    fate = 2;
done:
    if (log) { log->n_hits = nh; log->fate = fate; log->prim_hash = hash; log->beta = beta[0]; }
}

/* ------------------------------------------------------------- driver --------------- */
typedef struct {
    const fto_ctx* c;
    const Cam* cam;
    int64_t lo, hi;
    uint64_t seed_base;
    int max_bounce;
    int hero_c;   /* wavelengths per photon; 1 = the scalar tracer */
    double* xyz;
    double* hits;
    double e[5];
    ftb_photon_log* logs;
    int64_t* rays;
} Job;

static void* worker(void* arg) {
    Job* j = (Job*)arg;
    Film f = {j->xyz, j->hits, j->cam->rx, j->cam->ry};
    Tr T = {j->c, j->cam, &f, 0};
    Pcg rng;
    for (int64_t i = j->lo; i < j->hi; ++i) {
        seed_unit(&rng, j->seed_base + (uint64_t)i, PHOTON_SALT);
        T.rays = 0;
        if (j->hero_c > 1) trace_photon_hero(&T, &rng, j->max_bounce, j->hero_c, j->e, j->logs ? &j->logs[i] : NULL);
        else trace_photon(&T, &rng, j->max_bounce, j->e, j->logs ? &j->logs[i] : NULL);
        if (j->rays) j->rays[i] = T.rays;
    }
    return NULL;
}

int fto_trace(const fto_ctx* c, const ftb_camera* cam, int64_t n, uint64_t seed_base,
              int max_bounce, int hero_c, int threads, double* film_xyz, double* film_hits,
              double* energy, ftb_photon_log* logs, int64_t* rays) {
    if (!c || !cam || n < 0 || !film_xyz || !film_hits || !energy) return fail("fto_trace: bad input");
    /* -heroc is clamped to [1, kHeroMax] and hero sampling is off in scenes with media
     * (hero.h:81-86, main.cpp:11309-11312) */
    if (hero_c < 1) hero_c = 1;
    if (hero_c > HERO_MAX) hero_c = HERO_MAX;
    if (c->n_med > 0) hero_c = 1;
    if (threads < 1) threads = 1;
    Cam cm;
    cm.eye = rd3(cam->eye); cm.u = rd3(cam->u); cm.v = rd3(cam->v); cm.w = rd3(cam->w);
    cm.thx = cam->tan_half_x; cm.thy = cam->tan_half_y; cm.rx = cam->res_x; cm.ry = cam->res_y;
    size_t npix = (size_t)cm.rx * (size_t)cm.ry;
    Job* jobs = (Job*)calloc((size_t)threads, sizeof(Job));
    pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    for (int t = 0; t < threads; ++t) {
        Job* j = &jobs[t];
        j->c = c; j->cam = &cm; j->seed_base = seed_base; j->max_bounce = max_bounce; j->hero_c = hero_c;
        j->lo = n * t / threads; j->hi = n * (t + 1) / threads;
        j->logs = logs; j->rays = rays;
        if (threads == 1) { j->xyz = film_xyz; j->hits = film_hits; }
        else {
            j->xyz = (double*)calloc(npix * 3, sizeof(double));
            j->hits = (double*)calloc(npix, sizeof(double));
        }
    }
    if (threads == 1) worker(&jobs[0]);
    else {
        for (int t = 0; t < threads; ++t) pthread_create(&th[t], NULL, worker, &jobs[t]);
        for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
        /* Film::merge in thread order (scene_film.h:17-19, main.cpp:11334) */
        for (int t = 0; t < threads; ++t) {
            for (size_t i = 0; i < npix; ++i) {
                film_xyz[3 * i] += jobs[t].xyz[3 * i];
                film_xyz[3 * i + 1] += jobs[t].xyz[3 * i + 1];
                film_xyz[3 * i + 2] += jobs[t].xyz[3 * i + 2];
                film_hits[i] += jobs[t].hits[i];
            }
            free(jobs[t].xyz); free(jobs[t].hits);
        }
    }
    for (int t = 0; t < threads; ++t)
        for (int k = 0; k < 5; ++k) energy[k] += jobs[t].e[k];
    free(jobs); free(th);
    return 0;
}
