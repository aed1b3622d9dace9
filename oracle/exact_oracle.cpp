// exact_oracle.cpp -- decision-exact predicates of the restatement (the
// ORC_EXACT mode of pac_oracle.c).
//
// TEST INFRASTRUCTURE ONLY: part of the checker library (liboracle.so),
// never linked by the product.
//
// Every predicate is the exact sign of a polynomial in binary32 inputs:
// ball centres, shifted radii r, weights r^2 taken exactly, alpha.  The
// polynomials are the reference's tests with their divisions multiplied
// out (u = p2-p1, v = p3-p1, s = p4-p1, n = u x v,
// B_k = |p_k - p1|^2 + w1 - w_k):
//   edge alpha      |u| > 0 and 4|u|^2 (w1+a) - B2^2 >= 0           (LD:173-189)
//   triangle alpha  n != 0 and 4(w1+a)|n|^2
//                     - (B2^2 |v|^2 - 2 B2 B3 (u.v) + B3^2 |u|^2) >= 0   (LD:308-347)
//   tetrahedron     det(u,v,s) = 0 (kept, LD:577-580), or
//                   4(w1+a) det^2 - |B2 (v x s) + B3 (s x u) + B4 (u x v)|^2 >= 0
//   attached        (|q-p1|^2 - wq + w1) N - (q-p1).C <= 0 with
//                   (N, C) = (|u|^2, B2 u) for an edge and
//                   (|n|^2, B2 (v x n) + B3 (n x u)) for a triangle  (LD:825-829, 964-968)
//   orient3d, insphere_w: the determinants of PRED:2015-2054, 4250-4367.
//
// Evaluation: first in x87 extended precision (64-bit significand) beside
// the same polynomial over absolute values (a bound on every partial sum);
// the sign is taken when |value| > 2^-50 * bound, far above the rounding
// error of the < 64 operations involved.  Otherwise the polynomial is
// evaluated again over arbitrary-precision integers (sign + magnitude
// limbs), after writing each input as an integer multiple of one power of
// two.  The engine uses a different filter (FP64 with a running error
// bound) and fixed-width two's-complement integers, so the two checks are
// independent of each other.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// ---------------------------------------------------------------- filter
struct LM {
    long double v, m;  // value, bound on |partial sums|
};
LM operator+(const LM &a, const LM &b) { return LM{a.v + b.v, a.m + b.m}; }
LM operator-(const LM &a, const LM &b) { return LM{a.v - b.v, a.m + b.m}; }
LM operator*(const LM &a, const LM &b) { return LM{a.v * b.v, a.m * b.m}; }

int lm_sign(const LM &a) {
    const long double t = a.m * 0x1p-50L;
    if (a.v > t) return 1;
    if (a.v < -t) return -1;
    return 0;
}

// ---------------------------------------------------------------- integers
struct Z {
    std::vector<uint32_t> mag;  // little-endian limbs, no leading zeros
    bool neg = false;
};
void trim(Z &a) {
    while (!a.mag.empty() && !a.mag.back()) a.mag.pop_back();
    if (a.mag.empty()) a.neg = false;
}
int cmp_mag(const Z &a, const Z &b) {
    if (a.mag.size() != b.mag.size()) return a.mag.size() < b.mag.size() ? -1 : 1;
    for (size_t i = a.mag.size(); i-- > 0;)
        if (a.mag[i] != b.mag[i]) return a.mag[i] < b.mag[i] ? -1 : 1;
    return 0;
}
Z add_mag(const Z &a, const Z &b) {
    Z r;
    size_t n = std::max(a.mag.size(), b.mag.size());
    r.mag.resize(n + 1);
    uint64_t c = 0;
    for (size_t i = 0; i < n; i++) {
        uint64_t t = c + (i < a.mag.size() ? a.mag[i] : 0) + (i < b.mag.size() ? b.mag[i] : 0);
        r.mag[i] = (uint32_t)t;
        c = t >> 32;
    }
    r.mag[n] = (uint32_t)c;
    trim(r);
    return r;
}
Z sub_mag(const Z &a, const Z &b) {  // |a| >= |b|
    Z r;
    r.mag.resize(a.mag.size());
    int64_t br = 0;
    for (size_t i = 0; i < a.mag.size(); i++) {
        int64_t t = (int64_t)a.mag[i] - (i < b.mag.size() ? b.mag[i] : 0) - br;
        br = t < 0;
        r.mag[i] = (uint32_t)(t + (br << 32));
    }
    trim(r);
    return r;
}
Z operator+(const Z &a, const Z &b) {
    if (a.neg == b.neg) {
        Z r = add_mag(a, b);
        r.neg = a.neg && !r.mag.empty();
        return r;
    }
    if (cmp_mag(a, b) >= 0) {
        Z r = sub_mag(a, b);
        r.neg = a.neg && !r.mag.empty();
        return r;
    }
    Z r = sub_mag(b, a);
    r.neg = b.neg && !r.mag.empty();
    return r;
}
Z operator-(const Z &a, const Z &b) {
    Z nb = b;
    if (!nb.mag.empty()) nb.neg = !nb.neg;
    return a + nb;
}
Z operator*(const Z &a, const Z &b) {
    Z r;
    if (a.mag.empty() || b.mag.empty()) return r;
    r.mag.assign(a.mag.size() + b.mag.size(), 0);
    for (size_t i = 0; i < a.mag.size(); i++) {
        uint64_t c = 0;
        for (size_t j = 0; j < b.mag.size(); j++) {
            uint64_t t = (uint64_t)a.mag[i] * b.mag[j] + r.mag[i + j] + c;
            r.mag[i + j] = (uint32_t)t;
            c = t >> 32;
        }
        r.mag[i + b.mag.size()] = (uint32_t)c;
    }
    r.neg = a.neg != b.neg;
    trim(r);
    return r;
}
int z_sign(const Z &a) { return a.mag.empty() ? 0 : (a.neg ? -1 : 1); }

// binary32 -> integer multiple of 2^scale (the float must be one)
Z z_from(float f, int scale) {
    Z r;
    uint32_t u;
    std::memcpy(&u, &f, 4);
    uint32_t ex = (u >> 23) & 0xff, fr = u & 0x7fffff;
    uint64_t m = ex ? (fr | 0x800000u) : fr;
    int e = ex ? (int)ex - 150 : -149;
    if (!m) return r;
    int sh = e - scale;  // >= 0 by the choice of scale
    r.mag.assign((size_t)(sh / 32) + 3, 0);
    r.mag[sh / 32] = (uint32_t)(m << (sh % 32));
    r.mag[sh / 32 + 1] = (uint32_t)((m << (sh % 32)) >> 32);
    r.neg = (u >> 31) != 0;
    trim(r);
    return r;
}
int low_exp(float f, bool &nz) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    nz = (u & 0x7fffffffu) != 0;
    uint32_t ex = (u >> 23) & 0xff;
    return ex ? (int)ex - 150 : -149;
}

// ---------------------------------------------------------------- polynomials
template <class R>
struct P {
    R x, y, z, w;
};
template <class R>
struct V {
    R x, y, z;
};
template <class R>
V<R> dif(const P<R> &a, const P<R> &b) {
    return V<R>{a.x - b.x, a.y - b.y, a.z - b.z};
}
template <class R>
R dot(const V<R> &a, const V<R> &b) {
    return (a.x * b.x + a.y * b.y) + a.z * b.z;
}
template <class R>
V<R> cross(const V<R> &a, const V<R> &b) {
    return V<R>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R>
V<R> mul(const R &k, const V<R> &a) {
    return V<R>{k * a.x, k * a.y, k * a.z};
}
template <class R>
V<R> add(const V<R> &a, const V<R> &b) {
    return V<R>{a.x + b.x, a.y + b.y, a.z + b.z};
}
template <class R>
R times4(const R &a) {
    const R b = a + a;
    return b + b;
}

enum Kind { K_EDGE, K_NORMAL, K_TRI, K_DET, K_TET, K_EATT, K_TATT, K_ORIENT, K_INSPHERE };

template <class R>
R poly(int kind, const P<R> *p, const R &a) {
    switch (kind) {
    case K_EDGE: {
        const V<R> u = dif(p[1], p[0]);
        const R uu = dot(u, u), B2 = (uu + p[0].w) - p[1].w;
        return times4(uu) * (p[0].w + a) - B2 * B2;
    }
    case K_NORMAL: {
        const V<R> n = cross(dif(p[1], p[0]), dif(p[2], p[0]));
        return dot(n, n);
    }
    case K_TRI: {
        const V<R> u = dif(p[1], p[0]), v = dif(p[2], p[0]), n = cross(u, v);
        const R uu = dot(u, u), vv = dot(v, v), uv = dot(u, v);
        const R B2 = (uu + p[0].w) - p[1].w, B3 = (vv + p[0].w) - p[2].w;
        const R t = B2 * B3;
        return times4(p[0].w + a) * dot(n, n) - (((B2 * B2) * vv - (t + t) * uv) + (B3 * B3) * uu);
    }
    case K_DET:
        return dot(dif(p[1], p[0]), cross(dif(p[2], p[0]), dif(p[3], p[0])));
    case K_TET: {
        const V<R> u = dif(p[1], p[0]), v = dif(p[2], p[0]), s = dif(p[3], p[0]);
        const V<R> vs = cross(v, s), su = cross(s, u), uv = cross(u, v);
        const R d = dot(u, vs);
        const R B2 = (dot(u, u) + p[0].w) - p[1].w, B3 = (dot(v, v) + p[0].w) - p[2].w,
                B4 = (dot(s, s) + p[0].w) - p[3].w;
        const V<R> c = add(add(mul(B2, vs), mul(B3, su)), mul(B4, uv));
        return (times4(p[0].w + a) * d) * d - dot(c, c);
    }
    case K_EATT: {
        const V<R> u = dif(p[1], p[0]), q = dif(p[2], p[0]);
        const R uu = dot(u, u), B2 = (uu + p[0].w) - p[1].w;
        return ((dot(q, q) - p[2].w) + p[0].w) * uu - B2 * dot(u, q);
    }
    case K_TATT: {
        const V<R> u = dif(p[1], p[0]), v = dif(p[2], p[0]), q = dif(p[3], p[0]);
        const V<R> n = cross(u, v);
        const R B2 = (dot(u, u) + p[0].w) - p[1].w, B3 = (dot(v, v) + p[0].w) - p[2].w;
        const V<R> c = add(mul(B2, cross(v, n)), mul(B3, cross(n, u)));
        return ((dot(q, q) - p[3].w) + p[0].w) * dot(n, n) - dot(q, c);
    }
    case K_ORIENT: {
        const V<R> A = dif(p[0], p[3]), B = dif(p[1], p[3]), C = dif(p[2], p[3]);
        return dot(C, cross(A, B));
    }
    default: {  // K_INSPHERE
        V<R> d[4];
        R lw[4];
        for (int i = 0; i < 4; i++) {
            d[i] = dif(p[i], p[4]);
            lw[i] = dot(d[i], d[i]) - (p[i].w - p[4].w);
        }
        auto m2 = [&](int i, int j) { return d[i].x * d[j].y - d[j].x * d[i].y; };
        const R ab = m2(0, 1), bc = m2(1, 2), cd = m2(2, 3), da = m2(3, 0), ac = m2(0, 2),
                bd = m2(1, 3);
        const R abc = (d[0].z * bc - d[1].z * ac) + d[2].z * ab;
        const R bcd = (d[1].z * cd - d[2].z * bd) + d[3].z * bc;
        const R cda = (d[2].z * da + d[3].z * ac) + d[0].z * cd;
        const R dab = (d[3].z * ab + d[0].z * bd) + d[1].z * da;
        return (lw[3] * abc - lw[2] * dab) + (lw[1] * cda - lw[0] * bcd);
    }
    }
}

const int kPts[] = {2, 3, 3, 4, 4, 3, 4, 4, 5};

// balls: kPts[kind] x (x, y, z, r)
int sign_of(int kind, const float *b, float alpha, uint64_t *fallbacks) {
    const int np = kPts[kind];
    P<LM> pl[5];
    for (int i = 0; i < np; i++) {
        const long double x = b[4 * i], y = b[4 * i + 1], z = b[4 * i + 2], r = b[4 * i + 3];
        pl[i] = P<LM>{LM{x, fabsl(x)}, LM{y, fabsl(y)}, LM{z, fabsl(z)}, LM{r * r, r * r}};
    }
    const long double al = alpha;
    int s = lm_sign(poly(kind, pl, LM{al, fabsl(al)}));
    if (s) return s;
    if (fallbacks) __atomic_add_fetch(fallbacks, 1, __ATOMIC_RELAXED);
    int E = 0;
    bool nz;
    for (int i = 0; i < 4 * np; i++) {
        int e = low_exp(b[i], nz);
        if (nz && e < E) E = e;
    }
    int ea = low_exp(alpha, nz);
    if (nz && (ea >> 1) < E) E = ea >> 1;  // alpha sits at scale 2E
    P<Z> pz[5];
    for (int i = 0; i < np; i++) {
        const Z r = z_from(b[4 * i + 3], E);
        pz[i] = P<Z>{z_from(b[4 * i], E), z_from(b[4 * i + 1], E), z_from(b[4 * i + 2], E), r * r};
    }
    return z_sign(poly(kind, pz, z_from(alpha, 2 * E)));
}

}  // namespace

extern "C" {

uint64_t oex_fallbacks;  // integer evaluations since the counter was reset

// Decisions, as the oracle's pipeline asks them.  b holds the balls in
// order, 4 floats each.
int oex_edge(const float *b, float alpha) {
    if (b[0] == b[4] && b[1] == b[5] && b[2] == b[6]) return 0;  // 0/0 in the reference
    return sign_of(K_EDGE, b, alpha, &oex_fallbacks) >= 0;
}
int oex_tri(const float *b, float alpha) {
    if (sign_of(K_NORMAL, b, 0.0f, &oex_fallbacks) == 0) return 0;  // collinear
    return sign_of(K_TRI, b, alpha, &oex_fallbacks) >= 0;
}
// 1 alpha, 0 not, 2 flat (kept)
int oex_tet(const float *b, float alpha) {
    if (sign_of(K_DET, b, 0.0f, &oex_fallbacks) == 0) return 2;
    return sign_of(K_TET, b, alpha, &oex_fallbacks) >= 0;
}
int oex_orient(const float *b) { return sign_of(K_ORIENT, b, 0.0f, &oex_fallbacks); }
int oex_insphere(const float *b) { return sign_of(K_INSPHERE, b, 0.0f, &oex_fallbacks); }
int oex_edge_attached(const float *b) { return sign_of(K_EATT, b, 0.0f, &oex_fallbacks) <= 0; }
int oex_tri_attached(const float *b) { return sign_of(K_TATT, b, 0.0f, &oex_fallbacks) <= 0; }

// The polynomial's sign by integers alone (no filter), for the tests.
int oex_sign_integers(int kind, const float *b, float alpha) {
    const int np = kPts[kind];
    int E = 0;
    bool nz;
    for (int i = 0; i < 4 * np; i++) {
        int e = low_exp(b[i], nz);
        if (nz && e < E) E = e;
    }
    int ea = low_exp(alpha, nz);
    if (nz && (ea >> 1) < E) E = ea >> 1;
    P<Z> pz[5];
    for (int i = 0; i < np; i++) {
        const Z r = z_from(b[4 * i + 3], E);
        pz[i] = P<Z>{z_from(b[4 * i], E), z_from(b[4 * i + 1], E), z_from(b[4 * i + 2], E), r * r};
    }
    return z_sign(poly(kind, pz, z_from(alpha, 2 * E)));
}

}  // extern "C"
