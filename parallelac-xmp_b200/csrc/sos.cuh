// sos.cuh -- exact simulation of simplicity for the weighted insphere test.
//
// The reference breaks an insphere_w result of exactly 0.0f with
// orientation4SoS_w (predicates.h:4669-5462): the five points are put in
// ascending order of their 1-based input indices (counting the swaps), and
// a fixed sequence of 48 minors -- 3x3/2x2/1x1 orientation determinants on
// coordinate subsets, some with the lifted coordinate |p|^2 - w -- is
// evaluated until one is nonzero; that minor's sign, negated for the depths
// in kSosFlip and once more for an odd swap count, is the answer.  The
// reference evaluates the minors with single-precision expansion arithmetic,
// which is exact, so any exact evaluation gives the same signs.
//
// Here every input float is written as an integer multiple of a common
// power of two and the minors are evaluated with two's-complement integers
// of kLimbs 32-bit limbs.  This runs only in the fallback kernel that
// resolves the rare exact zeros, so it favours simplicity over speed.
#pragma once
#include <cstdint>

namespace pac {

constexpr int kLimbs = 20;  // 640-bit integers

struct BigInt {
    uint32_t w[kLimbs];
};

static __device__ inline void bi_zero(BigInt &r) {
#pragma unroll
    for (int i = 0; i < kLimbs; i++) r.w[i] = 0;
}
static __device__ inline void bi_add(BigInt &r, const BigInt &a, const BigInt &b) {
    uint64_t c = 0;
    for (int i = 0; i < kLimbs; i++) {
        uint64_t t = (uint64_t)a.w[i] + b.w[i] + c;
        r.w[i] = (uint32_t)t;
        c = t >> 32;
    }
}
static __device__ inline void bi_negate(BigInt &r) {
    uint64_t c = 1;
    for (int i = 0; i < kLimbs; i++) {
        uint64_t t = (uint64_t)(~r.w[i]) + c;
        r.w[i] = (uint32_t)t;
        c = t >> 32;
    }
}
static __device__ inline void bi_sub(BigInt &r, const BigInt &a, const BigInt &b) {
    BigInt nb = b;
    bi_negate(nb);
    bi_add(r, a, nb);
}
static __device__ inline int bi_sign(const BigInt &a) {
    if (a.w[kLimbs - 1] & 0x80000000u) return -1;
    for (int i = 0; i < kLimbs; i++)
        if (a.w[i]) return 1;
    return 0;
}
static __device__ inline void bi_mul(BigInt &r, const BigInt &a, const BigInt &b) {
    BigInt x = a, y = b;
    bool neg = false;
    if (bi_sign(x) < 0) { bi_negate(x); neg = !neg; }
    if (bi_sign(y) < 0) { bi_negate(y); neg = !neg; }
    uint32_t acc[kLimbs];
    for (int i = 0; i < kLimbs; i++) acc[i] = 0;
    for (int i = 0; i < kLimbs; i++) {
        uint32_t xi = x.w[i];
        if (!xi) continue;
        uint32_t carry = 0;
        for (int j = 0; i + j < kLimbs; j++) {
            // acc[i+j] + xi*y[j] + carry, with 64-bit intermediate
            uint64_t t = (uint64_t)xi * y.w[j] + acc[i + j] + carry;
            acc[i + j] = (uint32_t)t;
            carry = (uint32_t)(t >> 32);
        }
    }
    for (int i = 0; i < kLimbs; i++) r.w[i] = acc[i];
    if (neg) bi_negate(r);
}

// float -> integer at scale 2^scale (the float must be a multiple of it)
static __device__ inline void bi_from_float(BigInt &r, float f, int scale) {
    bi_zero(r);
    uint32_t u = __float_as_uint(f);
    uint32_t ex = (u >> 23) & 0xffu, fr = u & 0x7fffffu;
    uint32_t m = ex ? (fr | 0x800000u) : fr;
    int e = ex ? (int)ex - 150 : -149;
    if (!m) return;
    int sh = e - scale;
    int limb = sh >> 5, bit = sh & 31;
    if (limb < kLimbs) {
        uint64_t v = (uint64_t)m << bit;
        r.w[limb] = (uint32_t)v;
        if (limb + 1 < kLimbs) r.w[limb + 1] = (uint32_t)(v >> 32);
    }
    if (u >> 31) bi_negate(r);
}

// One step of the SoS minor sequence: dimension of the minor, whether the
// last column is the lifted coordinate, the rows (positions in index order)
// and the coordinate permutation applied to each row.
struct SosStep {
    int8_t kind, lifted, rows[4], perm[3];
};

// The minor sequence of predicates.h:4719-5417 (depth d at index d).
static __constant__ SosStep kSosSteps[49] = {
    {0, 0, {0, 0, 0, 0}, {0, 0, 0}},
    {3, 0, {1, 2, 3, 4}, {0, 1, 2}}, {3, 1, {1, 2, 3, 4}, {0, 1, 2}},
    {3, 1, {1, 2, 3, 4}, {0, 2, 1}}, {3, 1, {1, 2, 3, 4}, {1, 2, 0}},
    {3, 0, {0, 2, 3, 4}, {0, 1, 2}}, {2, 0, {2, 3, 4, 0}, {0, 1, 0}},
    {2, 0, {2, 3, 4, 0}, {0, 2, 0}}, {2, 0, {2, 3, 4, 0}, {1, 2, 0}},
    {3, 1, {0, 2, 3, 4}, {0, 1, 2}}, {2, 1, {2, 3, 4, 0}, {0, 1, 2}},
    {2, 1, {2, 3, 4, 0}, {1, 0, 2}}, {3, 1, {0, 2, 3, 4}, {0, 2, 1}},
    {2, 1, {2, 3, 4, 0}, {2, 0, 1}}, {3, 1, {0, 2, 3, 4}, {1, 2, 0}},
    {3, 0, {0, 1, 3, 4}, {0, 1, 2}}, {2, 0, {1, 3, 4, 0}, {0, 1, 0}},
    {2, 0, {1, 3, 4, 0}, {0, 2, 0}}, {2, 0, {1, 3, 4, 0}, {1, 2, 0}},
    {2, 0, {0, 3, 4, 0}, {0, 1, 0}}, {1, 0, {3, 4, 0, 0}, {0, 0, 0}},
    {1, 0, {3, 4, 0, 0}, {1, 0, 0}}, {2, 0, {0, 3, 4, 0}, {0, 2, 0}},
    {1, 0, {3, 4, 0, 0}, {2, 0, 0}}, {2, 0, {0, 3, 4, 0}, {1, 2, 0}},
    {3, 1, {0, 1, 3, 4}, {0, 1, 2}}, {2, 1, {1, 3, 4, 0}, {0, 1, 2}},
    {2, 1, {1, 3, 4, 0}, {1, 0, 2}}, {2, 1, {0, 3, 4, 0}, {0, 1, 2}},
    {1, 1, {3, 4, 0, 0}, {0, 1, 2}}, {2, 1, {0, 3, 4, 0}, {1, 0, 2}},
    {3, 1, {0, 1, 3, 4}, {0, 2, 1}}, {2, 1, {1, 3, 4, 0}, {2, 0, 1}},
    {2, 1, {0, 3, 4, 0}, {2, 0, 1}}, {3, 1, {0, 1, 3, 4}, {1, 2, 0}},
    {3, 0, {0, 1, 2, 4}, {0, 1, 2}}, {2, 0, {1, 2, 4, 0}, {0, 1, 0}},
    {2, 0, {1, 2, 4, 0}, {0, 2, 0}}, {2, 0, {1, 2, 4, 0}, {1, 2, 0}},
    {2, 0, {0, 2, 4, 0}, {0, 1, 0}}, {1, 0, {2, 4, 0, 0}, {0, 0, 0}},
    {1, 0, {2, 4, 0, 0}, {1, 0, 0}}, {2, 0, {0, 2, 4, 0}, {0, 2, 0}},
    {1, 0, {2, 4, 0, 0}, {2, 0, 0}}, {2, 0, {0, 2, 4, 0}, {1, 2, 0}},
    {2, 0, {0, 1, 4, 0}, {0, 1, 0}}, {1, 0, {1, 4, 0, 0}, {0, 0, 0}},
    {1, 0, {1, 4, 0, 0}, {1, 0, 0}}, {1, 0, {0, 4, 0, 0}, {0, 0, 0}},
};

// Depths whose minor sign is negated (predicates.h:5419-5450), as a bitmask.
constexpr uint64_t kSosFlip = (1ull << 1) | (1ull << 3) | (1ull << 7) | (1ull << 9) |
                              (1ull << 11) | (1ull << 14) | (1ull << 15) | (1ull << 16) |
                              (1ull << 18) | (1ull << 20) | (1ull << 22) | (1ull << 23) |
                              (1ull << 26) | (1ull << 30) | (1ull << 31) | (1ull << 32) |
                              (1ull << 37) | (1ull << 39) | (1ull << 41) | (1ull << 44) |
                              (1ull << 46);

struct SosPoints {
    BigInt c[5][3];  // coordinates at scale 2^E
    BigInt lift[5];  // |p|^2 - w at scale 2^(2E)
    BigInt w[5];     // w at scale 2^(2E)
};

// 4x4 orientation with rows (X, Y, L, 1), expanded as in
// orient3dexact_l_w (predicates.h:4466-4506).
static __device__ __noinline__ int sos_det3(const BigInt *X, const BigInt *Y, const BigInt *L) {
    BigInt m[6], t1, t2;
    const int P[6] = {0, 1, 2, 3, 0, 1}, Q[6] = {1, 2, 3, 0, 2, 3};  // ab bc cd da ac bd
    for (int k = 0; k < 6; k++) {
        bi_mul(t1, L[Q[k]], Y[P[k]]);
        bi_mul(t2, L[P[k]], Y[Q[k]]);
        bi_sub(m[k], t1, t2);
    }
    BigInt cda, dab, abc, bcd, acc;
    bi_add(cda, m[2], m[3]);
    bi_add(cda, cda, m[4]);
    bi_add(dab, m[3], m[0]);
    bi_add(dab, dab, m[5]);
    bi_add(abc, m[0], m[1]);
    bi_sub(abc, abc, m[4]);
    bi_add(bcd, m[1], m[2]);
    bi_sub(bcd, bcd, m[5]);
    bi_mul(acc, X[0], bcd);
    bi_mul(t1, X[1], cda);
    bi_sub(acc, acc, t1);
    bi_mul(t1, X[2], dab);
    bi_add(acc, acc, t1);
    bi_mul(t1, X[3], abc);
    bi_sub(acc, acc, t1);
    return bi_sign(acc);
}

// 3x3 orientation with rows (X, L, 1) (orient2dexact_l_w, predicates.h:4575-4596).
static __device__ __noinline__ int sos_det2(const BigInt *X, const BigInt *L) {
    BigInt d, t, acc;
    bi_sub(d, L[1], L[2]);
    bi_mul(acc, X[0], d);
    bi_sub(d, L[2], L[0]);
    bi_mul(t, X[1], d);
    bi_add(acc, acc, t);
    bi_sub(d, L[0], L[1]);
    bi_mul(t, X[2], d);
    bi_add(acc, acc, t);
    return bi_sign(acc);
}

static __device__ __noinline__ int sos_minor(const SosPoints &s, int depth) {
    const SosStep st = kSosSteps[depth];
    BigInt X[4], Y[4], L[4];
    if (st.kind == 3) {
        for (int r = 0; r < 4; r++) {
            int p = st.rows[r];
            X[r] = s.c[p][st.perm[0]];
            Y[r] = s.c[p][st.perm[1]];
            L[r] = st.lifted ? s.lift[p] : s.c[p][st.perm[2]];
        }
        return sos_det3(X, Y, L);
    }
    if (st.kind == 2) {
        for (int r = 0; r < 3; r++) {
            int p = st.rows[r];
            X[r] = s.c[p][st.perm[0]];
            L[r] = st.lifted ? s.lift[p] : s.c[p][st.perm[1]];
        }
        return sos_det2(X, L);
    }
    int a = st.rows[0], b = st.rows[1];
    BigInt t;
    if (!st.lifted) {
        bi_sub(t, s.c[a][st.perm[0]], s.c[b][st.perm[0]]);
        return bi_sign(t);
    }
    // orient1dexact_l_w with the lifted coordinate (predicates.h:4605-4647):
    // (|a|^2 - |b|^2) + (w_a - w_b) = (lift_a + 2 w_a) - (lift_b + 2 w_b)
    BigInt la, lb;
    bi_add(la, s.lift[a], s.w[a]);
    bi_add(la, la, s.w[a]);
    bi_add(lb, s.lift[b], s.w[b]);
    bi_add(lb, lb, s.w[b]);
    bi_sub(t, la, lb);
    return bi_sign(t);
}

// Sign of orientation4SoS_w(p[0..4], w[0..4], idx[0..4]).  Returns +1/-1;
// *status is 0, or 1 when the input range exceeds the integer width, or 2
// when every minor vanishes (the reference does not terminate there; this
// returns +1, the value its last depth is meant to give).  With radii set,
// w[] holds radii and the weights are their exact squares (the
// decision-exact mode); otherwise w[] holds the binary32 weights.
static __device__ __noinline__ int sos_orientation(const float (*p)[3], const float *w,
                                            const int *index, int *status, bool radii = false) {
    int idx[5], ord[5];
    for (int i = 0; i < 5; i++) { idx[i] = index[i]; ord[i] = i; }
    int swaps = 0;
    for (int i = 0; i < 4; i++)
        for (int j = 4; j > i; j--)
            if (idx[j] < idx[j - 1]) {
                int t = idx[j]; idx[j] = idx[j - 1]; idx[j - 1] = t;
                t = ord[j]; ord[j] = ord[j - 1]; ord[j - 1] = t;
                swaps++;
            }
    int emin = 0, emax = -1000;
    for (int i = 0; i < 5; i++)
        for (int k = 0; k < 4; k++) {
            float f = k < 3 ? p[ord[i]][k] : w[ord[i]];
            uint32_t u = __float_as_uint(f);
            uint32_t ex = (u >> 23) & 0xffu;
            if (!(u & 0x7fffffffu)) continue;
            int e = ex ? (int)ex - 150 : -149;
            emin = min(emin, e);
            emax = max(emax, e + 24);
        }
    *status = ((emax - emin) * 4 + 12 > kLimbs * 32 - 2) ? 1 : 0;
    SosPoints s;
    for (int i = 0; i < 5; i++) {
        BigInt sq, acc;
        bi_zero(acc);
        for (int k = 0; k < 3; k++) {
            bi_from_float(s.c[i][k], p[ord[i]][k], emin);
            bi_mul(sq, s.c[i][k], s.c[i][k]);
            bi_add(acc, acc, sq);
        }
        if (radii) {
            BigInt r;
            bi_from_float(r, w[ord[i]], emin);
            bi_mul(s.w[i], r, r);
        } else {
            bi_from_float(s.w[i], w[ord[i]], 2 * emin);
        }
        bi_sub(s.lift[i], acc, s.w[i]);
    }
    int sign = 0, depth = 0;
    for (depth = 1; depth <= 48; depth++) {
        sign = sos_minor(s, depth);
        if (sign) break;
    }
    if (!sign) {
        sign = 1;
        depth = 49;
        if (!*status) *status = 2;
    }
    if ((kSosFlip >> depth) & 1ull) sign = -sign;
    if (swaps & 1) sign = -sign;
    return sign;
}

}  // namespace pac
