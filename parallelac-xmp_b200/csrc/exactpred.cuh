// exactpred.cuh -- decision-exact predicates (PAC_PRED_EXACT).
//
// In this mode every decision of the pipeline is the exact sign of a
// polynomial in the binary32 inputs as the pipeline holds them: centres
// (x, y, z), shifted radii r = r_raw + sol (rounded to binary32 once, as
// the reference stores them, LD:1085), weights w = r^2 taken exactly (not
// rounded to binary32), and alpha.  The reference asks the same questions
// with single-precision formulas whose rounding can flip near-ties; this
// mode does not reproduce those flips, it answers the questions exactly.
// The candidate sets and the 27-cell windows stay the reference's.
//
// Cascade.  Each polynomial is first evaluated in FP64 with a running bound
// on its absolute error (every operation adds |result| * 2^-53 and products
// propagate their operands' bounds).  If |value| exceeds the bound the sign
// is certain.  Otherwise the polynomial is evaluated again in 640-bit
// two's-complement integers, after writing every input as an integer
// multiple of one power of two chosen per call; that path is counted
// (pac_stats.exact_fallbacks).
//
// Polynomials, with u = p2 - p1, v = p3 - p1, s = p4 - p1, n = u x v and
// B_k = |p_k - p1|^2 + w1 - w_k (twice the offset of the radical plane of
// balls 1 and k along p_k - p1):
//   edge alpha      |u| > 0 and 4 |u|^2 (w1 + a) - B2^2 >= 0
//   triangle alpha  n != 0 and 4 (w1 + a) |n|^2 - (B2^2 |v|^2 - 2 B2 B3 (u.v) + B3^2 |u|^2) >= 0
//   tetrahedron     d = det(u, v, s) = 0 (kept, LD:577-580), or
//                   4 (w1 + a) d^2 - |B2 (v x s) + B3 (s x u) + B4 (u x v)|^2 >= 0
//   edge attached   (|q - p1|^2 - wq + w1) |u|^2 - B2 (u . (q - p1)) <= 0
//   tri attached    (|q - p1|^2 - wq + w1) |n|^2 - (q - p1) . (B2 (v x n) + B3 (n x u)) <= 0
//   orient3d        det(pa - pd, pb - pd, pc - pd)                     (PRED:2015-2054)
//   insphere_w      the lifted 4x4 determinant of PRED:4250-4367, w exact
// Each is the reference's test with its divisions multiplied out: the
// edge test is (foot power) <= alpha for the foot p1 + u B2 / (2|u|^2)
// (LD:173-189), the triangle and tetrahedron tests are (orthocentre power)
// <= alpha for the orthocentres p1 + (B2 (v x n) + B3 (n x u)) / (2|n|^2)
// and p1 + (B2 (v x s) + B3 (s x u) + B4 (u x v)) / (2 d) (LD:308-347,
// 531-591), and the attachment tests compare the power of ball q at that
// centre with the simplex's own (LD:825-829, 964-968, ties attach).
#pragma once
#include <cstdint>

#include "refarith.cuh"
#include "sos.cuh"

namespace pac {
namespace ex {

// ------------------------------------------------------------------ FP64 filter
struct EV {
    double v, e;  // value, bound on |value - exact|
};

constexpr double kU = 1.1102230246251565e-16;  // 2^-53
constexpr double kTiny = 1e-300;               // covers underflow of a product

__device__ __forceinline__ EV ev(float f) { return EV{(double)f, 0.0}; }
__device__ __forceinline__ EV operator+(const EV a, const EV b) {
    const double v = a.v + b.v;
    return EV{v, (a.e + b.e) + fabs(v) * kU};
}
__device__ __forceinline__ EV operator-(const EV a, const EV b) {
    const double v = a.v - b.v;
    return EV{v, (a.e + b.e) + fabs(v) * kU};
}
__device__ __forceinline__ EV operator*(const EV a, const EV b) {
    const double v = a.v * b.v;
    return EV{v, ((fabs(a.v) * b.e + fabs(b.v) * a.e) + a.e * b.e) + (fabs(v) * kU + kTiny)};
}
// +1 / -1 when certain, 0 when the filter cannot tell.  The bound itself is
// computed with rounding; the factor covers that (far fewer than 10^3 terms).
__device__ __forceinline__ int ev_sign(const EV a) {
    const double b = a.e * (1.0 + 1e-12);
    if (a.v > b) return 1;
    if (a.v < -b) return -1;
    return 0;
}

// ------------------------------------------------------------------ integers
struct BI {
    BigInt b;
};
__device__ __forceinline__ BI operator+(const BI &a, const BI &b) {
    BI r;
    bi_add(r.b, a.b, b.b);
    return r;
}
__device__ __forceinline__ BI operator-(const BI &a, const BI &b) {
    BI r;
    bi_sub(r.b, a.b, b.b);
    return r;
}
__device__ __forceinline__ BI operator*(const BI &a, const BI &b) {
    BI r;
    bi_mul(r.b, a.b, b.b);
    return r;
}

// ------------------------------------------------------------------ polynomials
template <class R>
struct P4 {
    R x, y, z, w;  // centre and weight
};
template <class R>
struct V3 {
    R x, y, z;
};
template <class R>
__device__ __forceinline__ V3<R> dif(const P4<R> &a, const P4<R> &b) {
    return V3<R>{a.x - b.x, a.y - b.y, a.z - b.z};
}
template <class R>
__device__ __forceinline__ R dot(const V3<R> &a, const V3<R> &b) {
    return (a.x * b.x + a.y * b.y) + a.z * b.z;
}
template <class R>
__device__ __forceinline__ V3<R> cross(const V3<R> &a, const V3<R> &b) {
    return V3<R>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R>
__device__ __forceinline__ V3<R> scale(const R &k, const V3<R> &a) {
    return V3<R>{k * a.x, k * a.y, k * a.z};
}
template <class R>
__device__ __forceinline__ V3<R> add3(const V3<R> &a, const V3<R> &b) {
    return V3<R>{a.x + b.x, a.y + b.y, a.z + b.z};
}

// Each functor maps points p[0..] (and alpha, and for the attachment tests
// the extra ball q = p[last]) to a polynomial whose sign is the decision.
struct FEdge {  // >= 0: alpha edge (given |u| > 0)
    static constexpr int kPts = 2;
    template <class R>
    __device__ R operator()(const P4<R> *p, const R &a) const {
        const V3<R> u = dif(p[1], p[0]);
        const R uu = dot(u, u);
        const R B2 = (uu + p[0].w) - p[1].w;
        const R four = uu + uu + uu + uu;
        return four * (p[0].w + a) - B2 * B2;
    }
};
struct FNormal2 {  // |n|^2 of a triangle: 0 iff collinear
    static constexpr int kPts = 3;
    template <class R>
    __device__ R operator()(const P4<R> *p, const R &) const {
        const V3<R> n = cross(dif(p[1], p[0]), dif(p[2], p[0]));
        return dot(n, n);
    }
};
struct FTri {  // >= 0: alpha triangle (given n != 0)
    static constexpr int kPts = 3;
    template <class R>
    __device__ R operator()(const P4<R> *p, const R &a) const {
        const V3<R> u = dif(p[1], p[0]), v = dif(p[2], p[0]);
        const V3<R> n = cross(u, v);
        const R uu = dot(u, u), vv = dot(v, v), uv = dot(u, v), nn = dot(n, n);
        const R B2 = (uu + p[0].w) - p[1].w, B3 = (vv + p[0].w) - p[2].w;
        const R wa = p[0].w + a;
        const R lhs = (wa + wa + wa + wa) * nn;
        const R t = B2 * B3;
        return lhs - (((B2 * B2) * vv - (t + t) * uv) + (B3 * B3) * uu);
    }
};
struct FDet {  // det(u, v, s) of a tetrahedron
    static constexpr int kPts = 4;
    template <class R>
    __device__ R operator()(const P4<R> *p, const R &) const {
        return dot(dif(p[1], p[0]), cross(dif(p[2], p[0]), dif(p[3], p[0])));
    }
};
struct FTet {  // >= 0: alpha tetrahedron (given det != 0)
    static constexpr int kPts = 4;
    template <class R>
    __device__ R operator()(const P4<R> *p, const R &a) const {
        const V3<R> u = dif(p[1], p[0]), v = dif(p[2], p[0]), s = dif(p[3], p[0]);
        const V3<R> vs = cross(v, s), su = cross(s, u), uv = cross(u, v);
        const R d = dot(u, vs);
        const R B2 = (dot(u, u) + p[0].w) - p[1].w;
        const R B3 = (dot(v, v) + p[0].w) - p[2].w;
        const R B4 = (dot(s, s) + p[0].w) - p[3].w;
        const V3<R> c = add3(add3(scale(B2, vs), scale(B3, su)), scale(B4, uv));
        const R wa = p[0].w + a;
        return ((wa + wa + wa + wa) * d) * d - dot(c, c);
    }
};
struct FEdgeAttach {  // <= 0: ball p[2] attaches edge (p[0], p[1])
    static constexpr int kPts = 3;
    template <class R>
    __device__ R operator()(const P4<R> *p, const R &) const {
        const V3<R> u = dif(p[1], p[0]), q = dif(p[2], p[0]);
        const R uu = dot(u, u);
        const R B2 = (uu + p[0].w) - p[1].w;
        return ((dot(q, q) - p[2].w) + p[0].w) * uu - B2 * dot(u, q);
    }
};
struct FTriAttach {  // <= 0: ball p[3] attaches triangle (p[0], p[1], p[2])
    static constexpr int kPts = 4;
    template <class R>
    __device__ R operator()(const P4<R> *p, const R &) const {
        const V3<R> u = dif(p[1], p[0]), v = dif(p[2], p[0]), q = dif(p[3], p[0]);
        const V3<R> n = cross(u, v);
        const R B2 = (dot(u, u) + p[0].w) - p[1].w, B3 = (dot(v, v) + p[0].w) - p[2].w;
        const V3<R> c = add3(scale(B2, cross(v, n)), scale(B3, cross(n, u)));
        return ((dot(q, q) - p[3].w) + p[0].w) * dot(n, n) - dot(q, c);
    }
};
struct FOrient {  // orient3d(pa, pb, pc, pd): rows pa - pd, pb - pd, pc - pd
    static constexpr int kPts = 4;
    template <class R>
    __device__ R operator()(const P4<R> *p, const R &) const {
        const V3<R> a = dif(p[0], p[3]), b = dif(p[1], p[3]), c = dif(p[2], p[3]);
        return dot(c, cross(a, b));
    }
};
struct FInsphere {  // insphere_w(pa, pb, pc, pd, pe) of PRED:4250-4367
    static constexpr int kPts = 5;
    template <class R>
    __device__ R operator()(const P4<R> *p, const R &) const {
        V3<R> d[4];
        R lw[4];
        for (int i = 0; i < 4; i++) {
            d[i] = dif(p[i], p[4]);
            lw[i] = dot(d[i], d[i]) - (p[i].w - p[4].w);
        }
        const R ab = d[0].x * d[1].y - d[1].x * d[0].y;
        const R bc = d[1].x * d[2].y - d[2].x * d[1].y;
        const R cd = d[2].x * d[3].y - d[3].x * d[2].y;
        const R da = d[3].x * d[0].y - d[0].x * d[3].y;
        const R ac = d[0].x * d[2].y - d[2].x * d[0].y;
        const R bd = d[1].x * d[3].y - d[3].x * d[1].y;
        const R abc = (d[0].z * bc - d[1].z * ac) + d[2].z * ab;
        const R bcd = (d[1].z * cd - d[2].z * bd) + d[3].z * bc;
        const R cda = (d[2].z * da + d[3].z * ac) + d[0].z * cd;
        const R dab = (d[3].z * ab + d[0].z * bd) + d[1].z * da;
        return (lw[3] * abc - lw[2] * dab) + (lw[1] * cda - lw[0] * bcd);
    }
};

// ------------------------------------------------------------------ evaluation
// Exponent of the lowest and one past the highest mantissa bit of a float
// (value = m * 2^lo, |value| < 2^hi); false for zero.
__device__ __forceinline__ bool fexp(float f, int &lo, int &hi) {
    const uint32_t u = __float_as_uint(f);
    if (!(u & 0x7fffffffu)) return false;
    const uint32_t ex = (u >> 23) & 0xffu;
    lo = ex ? (int)ex - 150 : -149;
    hi = lo + 24;
    return true;
}

// Exact sign by integers.  *range is set when the inputs span more bits
// than the 640-bit integers hold for a polynomial of weighted degree 8.
template <class F, int N>
__device__ __noinline__ int exact_sign(const F f, const Ball (&b)[N], float alpha, int *range) {
    int E = 0, H = -1000, lo, hi;
    for (int i = 0; i < N; i++) {
        const float c[4] = {b[i].x, b[i].y, b[i].z, b[i].r};
        for (int k = 0; k < 4; k++)
            if (fexp(c[k], lo, hi)) {
                E = min(E, lo);
                H = max(H, hi);
            }
    }
    if (fexp(alpha, lo, hi)) {  // alpha sits at scale 2E: halve its exponents
        E = min(E, lo >> 1);
        H = max(H, (hi + 1) >> 1);
    }
    if (8 * (H - E) + 24 > kLimbs * 32 - 1) {
        *range = 1;
        return 0;
    }
    P4<BI> p[N];
    for (int i = 0; i < N; i++) {
        bi_from_float(p[i].x.b, b[i].x, E);
        bi_from_float(p[i].y.b, b[i].y, E);
        bi_from_float(p[i].z.b, b[i].z, E);
        BI r;
        bi_from_float(r.b, b[i].r, E);
        p[i].w = r * r;
    }
    BI a;
    bi_from_float(a.b, alpha, 2 * E);
    return bi_sign(f(p, a).b);
}

// Per-thread counts of one kernel: filtered decisions, integer
// evaluations, and whether an input exceeded the integers' range.
struct Tally {
    uint32_t evals = 0;
    uint32_t fallbacks = 0;
    int range = 0;
};

// The cascade: FP64 filter, integers when it cannot decide.
template <class F, int N>
__device__ __forceinline__ int sign_of(const F f, const Ball (&b)[N], float alpha, Tally &t) {
    P4<EV> p[N];
#pragma unroll
    for (int i = 0; i < N; i++) {
        const EV r = ev(b[i].r);
        p[i] = P4<EV>{ev(b[i].x), ev(b[i].y), ev(b[i].z), r * r};
    }
    t.evals++;
    const int s = ev_sign(f(p, ev(alpha)));
    if (s) return s;
    t.fallbacks++;
    return exact_sign(f, b, alpha, &t.range);
}

// ------------------------------------------------------------------ decisions

__device__ __forceinline__ bool edge_alpha(const Ball a1, const Ball a2, float alpha, Tally &t) {
    if (a1.x == a2.x && a1.y == a2.y && a1.z == a2.z) return false;  // 0/0 in the reference
    const Ball b[2] = {a1, a2};
    return sign_of(FEdge{}, b, alpha, t) >= 0;
}

__device__ __forceinline__ bool tri_alpha(const Ball a1, const Ball a2, const Ball a3, float alpha,
                                          Tally &t) {
    const Ball b[3] = {a1, a2, a3};
    if (sign_of(FNormal2{}, b, alpha, t) == 0) return false;  // collinear
    return sign_of(FTri{}, b, alpha, t) >= 0;
}

// Returns the alpha decision; *flat is set when det = 0 (kept, no orthocentre).
__device__ __forceinline__ bool tet_alpha(const Ball a1, const Ball a2, const Ball a3,
                                          const Ball a4, float alpha, bool &flat, Tally &t) {
    const Ball b[4] = {a1, a2, a3, a4};
    flat = sign_of(FDet{}, b, alpha, t) == 0;
    if (flat) return true;
    return sign_of(FTet{}, b, alpha, t) >= 0;
}

__device__ __forceinline__ int orient_sign(const Ball a, const Ball b, const Ball c, const Ball d,
                                           Tally &t) {
    const Ball p[4] = {a, b, c, d};
    return sign_of(FOrient{}, p, 0.0f, t);
}

__device__ __forceinline__ int insphere_sign(const Ball a, const Ball b, const Ball c,
                                             const Ball d, const Ball e, Tally &t) {
    const Ball p[5] = {a, b, c, d, e};
    return sign_of(FInsphere{}, p, 0.0f, t);
}

__device__ __forceinline__ bool edge_attached(const Ball a1, const Ball a2, const Ball q,
                                              Tally &t) {
    const Ball p[3] = {a1, a2, q};
    return sign_of(FEdgeAttach{}, p, 0.0f, t) <= 0;
}

__device__ __forceinline__ bool tri_attached(const Ball a1, const Ball a2, const Ball a3,
                                             const Ball q, Tally &t) {
    const Ball p[4] = {a1, a2, a3, q};
    return sign_of(FTriAttach{}, p, 0.0f, t) <= 0;
}

// ------------------------------------------------------------------ window centres
// FP64 centres for the window lookups (the decisions above do not use them).
__device__ __forceinline__ float3 edge_centre(const Ball a1, const Ball a2) {
    const double ux = (double)a2.x - a1.x, uy = (double)a2.y - a1.y, uz = (double)a2.z - a1.z;
    const double uu = ux * ux + uy * uy + uz * uz;
    const double w1 = (double)a1.r * a1.r, w2 = (double)a2.r * a2.r;
    const double t = (uu + w1 - w2) / (2.0 * uu);
    return make_float3((float)(a1.x + t * ux), (float)(a1.y + t * uy), (float)(a1.z + t * uz));
}

__device__ __forceinline__ float3 tri_centre(const Ball a1, const Ball a2, const Ball a3) {
    const double ux = (double)a2.x - a1.x, uy = (double)a2.y - a1.y, uz = (double)a2.z - a1.z;
    const double vx = (double)a3.x - a1.x, vy = (double)a3.y - a1.y, vz = (double)a3.z - a1.z;
    const double nx = uy * vz - uz * vy, ny = uz * vx - ux * vz, nz = ux * vy - uy * vx;
    const double w1 = (double)a1.r * a1.r;
    const double B2 = ux * ux + uy * uy + uz * uz + w1 - (double)a2.r * a2.r;
    const double B3 = vx * vx + vy * vy + vz * vz + w1 - (double)a3.r * a3.r;
    // B2 (v x n) + B3 (n x u), over 2 |n|^2
    const double cx = B2 * (vy * nz - vz * ny) + B3 * (ny * uz - nz * uy);
    const double cy = B2 * (vz * nx - vx * nz) + B3 * (nz * ux - nx * uz);
    const double cz = B2 * (vx * ny - vy * nx) + B3 * (nx * uy - ny * ux);
    const double k = 1.0 / (2.0 * (nx * nx + ny * ny + nz * nz));
    return make_float3((float)(a1.x + cx * k), (float)(a1.y + cy * k), (float)(a1.z + cz * k));
}

__device__ __forceinline__ float3 tet_centre(const Ball a1, const Ball a2, const Ball a3,
                                             const Ball a4) {
    const double ux = (double)a2.x - a1.x, uy = (double)a2.y - a1.y, uz = (double)a2.z - a1.z;
    const double vx = (double)a3.x - a1.x, vy = (double)a3.y - a1.y, vz = (double)a3.z - a1.z;
    const double sx = (double)a4.x - a1.x, sy = (double)a4.y - a1.y, sz = (double)a4.z - a1.z;
    const double w1 = (double)a1.r * a1.r;
    const double B2 = ux * ux + uy * uy + uz * uz + w1 - (double)a2.r * a2.r;
    const double B3 = vx * vx + vy * vy + vz * vz + w1 - (double)a3.r * a3.r;
    const double B4 = sx * sx + sy * sy + sz * sz + w1 - (double)a4.r * a4.r;
    const double vsx = vy * sz - vz * sy, vsy = vz * sx - vx * sz, vsz = vx * sy - vy * sx;
    const double sux = sy * uz - sz * uy, suy = sz * ux - sx * uz, suz = sx * uy - sy * ux;
    const double uvx = uy * vz - uz * vy, uvy = uz * vx - ux * vz, uvz = ux * vy - uy * vx;
    const double d = ux * vsx + uy * vsy + uz * vsz;
    const double k = 1.0 / (2.0 * d);
    return make_float3((float)(a1.x + (B2 * vsx + B3 * sux + B4 * uvx) * k),
                       (float)(a1.y + (B2 * vsy + B3 * suy + B4 * uvy) * k),
                       (float)(a1.z + (B2 * vsz + B3 * suz + B4 * uvz) * k));
}

}  // namespace ex
}  // namespace pac
