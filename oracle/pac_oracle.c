/*
 * pac_oracle.c -- CPU restatement of the ParallelAC weighted alpha complex
 * pipeline (forest113/ParallelAC-xmp).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA engine
 * is compared against; it is linked by tests/, by __graft_entry__.smoke()
 * and by the bench's cpu_baseline leg, never by the product library.
 *
 * Arithmetic contract: every float operation below is one IEEE binary32
 * operation in the same order as the reference kernels, with no FMA
 * contraction (compile with -ffp-contract=off on x86-64/SSE).  This equals
 * the reference built with nvcc -fmad=false.  Where the reference mixes in
 * double (the `alpha + ATHRES` comparisons of the plain-xmp variant) the
 * same double operations are used.  Citations are to the reference tree:
 *   LD    = AlphaComplexLargeData.cu
 *   PLAIN = AlphaComplexParallel.cu
 *   PRED  = predicates.h
 */
#include "pac_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    float x, y, z, r; /* r = raw radius + solvent radius (LD:1085) */
    uint32_t idx;     /* 1-based original index (LD:1086) */
} oatom;

/* ------------------------------------------------------------------ */
/* CUDA float->int conversion semantics (cvt.rzi.s32.f32): truncation, */
/* saturation to the int range, NaN -> 0.  The reference converts with */
/* (int) in device code (LD:72-74, 621-623, 812-814, 951-953).          */
static inline int32_t f2i(float v) {
    if (v != v) return 0;
    if (v >= 2147483648.0f) return INT32_MAX;
    if (v <= -2147483648.0f) return INT32_MIN;
    return (int32_t)v;
}

/* 32-bit wrapping int arithmetic, as the reference's int expressions
   behave on the GPU. */
static inline int32_t wadd(int32_t a, int32_t b) {
    return (int32_t)((uint32_t)a + (uint32_t)b);
}
static inline int32_t lin3(int32_t X, int32_t Y, int32_t Z, int32_t gx,
                           int32_t gy) {
    /* gridZ * gx * gy + gridY * gx + gridX  (LD:625-626) */
    uint32_t r = (uint32_t)Z * (uint32_t)gx * (uint32_t)gy +
                 (uint32_t)Y * (uint32_t)gx + (uint32_t)X;
    return (int32_t)r;
}

/* ------------------------------------------------------------------ */
/* Single-precision predicates restated from PRED:2015-2054 and         */
/* PRED:4250-4367.  Only the determinant is live in the reference: both */
/* functions return it whatever the error bound says.                   */
float orc_orient3d(const float *pa, const float *pb, const float *pc,
                   const float *pd) {
    float adx = pa[0] - pd[0], bdx = pb[0] - pd[0], cdx = pc[0] - pd[0];
    float ady = pa[1] - pd[1], bdy = pb[1] - pd[1], cdy = pc[1] - pd[1];
    float adz = pa[2] - pd[2], bdz = pb[2] - pd[2], cdz = pc[2] - pd[2];
    float bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
    float cdxady = cdx * ady, adxcdy = adx * cdy;
    float adxbdy = adx * bdy, bdxady = bdx * ady;
    float det = adz * (bdxcdy - cdxbdy) + bdz * (cdxady - adxcdy);
    det = det + cdz * (adxbdy - bdxady);
    return det;
}

float orc_insphere_w(const float *pa, const float *pb, const float *pc,
                     const float *pd, const float *pe, float wa, float wb,
                     float wc, float wd, float we) {
    float aex = pa[0] - pe[0], bex = pb[0] - pe[0];
    float cex = pc[0] - pe[0], dex = pd[0] - pe[0];
    float aey = pa[1] - pe[1], bey = pb[1] - pe[1];
    float cey = pc[1] - pe[1], dey = pd[1] - pe[1];
    float aez = pa[2] - pe[2], bez = pb[2] - pe[2];
    float cez = pc[2] - pe[2], dez = pd[2] - pe[2];
    float aew = wa - we, bew = wb - we, cew = wc - we, dew = wd - we;
    float ab = aex * bey - bex * aey;
    float bc = bex * cey - cex * bey;
    float cd = cex * dey - dex * cey;
    float da = dex * aey - aex * dey;
    float ac = aex * cey - cex * aey;
    float bd = bex * dey - dex * bey;
    float abc = aez * bc - bez * ac;
    abc = abc + cez * ab;
    float bcd = bez * cd - cez * bd;
    bcd = bcd + dez * bc;
    float cda = cez * da + dez * ac;
    cda = cda + aez * cd;
    float dab = dez * ab + aez * bd;
    dab = dab + bez * da;
    float alift = aex * aex + aey * aey;
    alift = alift + aez * aez;
    float blift = bex * bex + bey * bey;
    blift = blift + bez * bez;
    float clift = cex * cex + cey * cey;
    clift = clift + cez * cez;
    float dlift = dex * dex + dey * dey;
    dlift = dlift + dez * dez;
    float alw = alift - aew, blw = blift - bew;
    float clw = clift - cew, dlw = dlift - dew;
    return (dlw * abc - clw * dab) + (blw * cda - alw * bcd);
}

/* ------------------------------------------------------------------ */
/* Exact integer arithmetic for the simulation-of-simplicity fallback.  */
/* A value is a two's-complement integer of BL 32-bit limbs.            */
#define BL 24
typedef struct {
    uint32_t w[BL];
} big;

static void big_zero(big *r) { memset(r, 0, sizeof(*r)); }
static void big_neg(big *r) {
    uint64_t c = 1;
    for (int i = 0; i < BL; i++) {
        uint64_t t = (uint64_t)(uint32_t)~r->w[i] + c;
        r->w[i] = (uint32_t)t;
        c = t >> 32;
    }
}
static int big_sign(const big *a) {
    if (a->w[BL - 1] & 0x80000000u) return -1;
    for (int i = 0; i < BL; i++)
        if (a->w[i]) return 1;
    return 0;
}
static void big_add(big *r, const big *a, const big *b) {
    uint64_t c = 0;
    for (int i = 0; i < BL; i++) {
        uint64_t t = (uint64_t)a->w[i] + b->w[i] + c;
        r->w[i] = (uint32_t)t;
        c = t >> 32;
    }
}
static void big_sub(big *r, const big *a, const big *b) {
    big nb = *b;
    big_neg(&nb);
    big_add(r, a, &nb);
}
static void big_mul(big *r, const big *a, const big *b) {
    big x = *a, y = *b;
    int s = 1;
    if (big_sign(&x) < 0) { big_neg(&x); s = -s; }
    if (big_sign(&y) < 0) { big_neg(&y); s = -s; }
    uint32_t acc[BL];
    memset(acc, 0, sizeof(acc));
    int nx = BL, ny = BL; /* limbs in use (magnitudes are non-negative now) */
    while (nx > 0 && !x.w[nx - 1]) nx--;
    while (ny > 0 && !y.w[ny - 1]) ny--;
    for (int i = 0; i < nx; i++) {
        if (!x.w[i]) continue;
        uint64_t c = 0;
        int j = 0;
        for (; j < ny && i + j < BL; j++) {
            uint64_t t = (uint64_t)x.w[i] * y.w[j] + acc[i + j] + c;
            acc[i + j] = (uint32_t)t;
            c = t >> 32;
        }
        for (; c && i + j < BL; j++) { /* carry out of the top limb */
            uint64_t t = (uint64_t)acc[i + j] + c;
            acc[i + j] = (uint32_t)t;
            c = t >> 32;
        }
    }
    memcpy(r->w, acc, sizeof(acc));
    if (s < 0) big_neg(r);
}
/* value = sign * mant * 2^shift, shift >= 0 */
static void big_set(big *r, uint32_t mant, int shift, int neg) {
    big_zero(r);
    int limb = shift / 32, bit = shift % 32;
    if (limb < BL) {
        uint64_t v = (uint64_t)mant << bit;
        r->w[limb] = (uint32_t)v;
        if (limb + 1 < BL) r->w[limb + 1] = (uint32_t)(v >> 32);
    }
    if (neg) big_neg(r);
}

/* binary32 -> sign, integer mantissa, exponent (value = m * 2^e) */
static void fdec(float f, uint32_t *m, int *e, int *neg) {
    uint32_t u;
    memcpy(&u, &f, 4);
    *neg = (u >> 31) & 1;
    uint32_t ex = (u >> 23) & 0xff, fr = u & 0x7fffff;
    if (ex == 0) {
        *m = fr;
        *e = -149;
    } else {
        *m = fr | 0x800000u;
        *e = (int)ex - 150;
    }
}

typedef struct {
    int E;          /* common scale exponent (<= 0) */
    big c[5][3];    /* coordinates at scale 2^E */
    big lift[5];    /* |p|^2 - w at scale 2^(2E) */
    big w2[5];      /* w at scale 2^(2E) */
    int overflow;
} sos_pts;

static void to_big(big *r, float f, int scale) {
    uint32_t m;
    int e, n;
    fdec(f, &m, &e, &n);
    if (m == 0) {
        big_zero(r);
        return;
    }
    big_set(r, m, e - scale, n);
}

/* Load the five points in SoS (sorted-index) order at one common scale. */
static void sos_load(sos_pts *s, float *const *ip, const float *iw, int radii) {
    int emin = 0, emax = -1000;
    for (int i = 0; i < 5; i++) {
        for (int k = 0; k < 4; k++) {
            float f = k < 3 ? ip[i][k] : iw[i];
            uint32_t m;
            int e, n;
            fdec(f, &m, &e, &n);
            if (!m) continue;
            if (e < emin) emin = e;
            if (e + 24 > emax) emax = e + 24;
        }
    }
    s->E = emin;
    /* magnitude bound: 4 factors of (emax - E) bits plus summation bits
       must stay inside BL*32 - 2 bits */
    s->overflow = (emax - emin) * 4 + 12 > BL * 32 - 2;
    for (int i = 0; i < 5; i++) {
        big sq, t;
        big_zero(&s->lift[i]);
        for (int k = 0; k < 3; k++) {
            to_big(&s->c[i][k], ip[i][k], emin);
            big_mul(&sq, &s->c[i][k], &s->c[i][k]);
            big_add(&t, &s->lift[i], &sq);
            s->lift[i] = t;
        }
        if (radii) { /* iw holds radii: the weight is their exact square */
            big r;
            to_big(&r, iw[i], emin);
            big_mul(&s->w2[i], &r, &r);
        } else {
            to_big(&s->w2[i], iw[i], 2 * emin);
        }
        big_sub(&t, &s->lift[i], &s->w2[i]);
        s->lift[i] = t;
    }
}

/* orient3dexact_l_w (PRED:4369-4507): rows (X, Y, L); the determinant is
   X_a*bcd - X_b*cda + X_c*dab - X_d*abc with the 2x2 minors below. */
static int det3(const big *X, const big *Y, const big *L) {
    big t1, t2, ab, bc, cd, da, ac, bd, cda, dab, abc, bcd, s, acc;
#define M2(out, p, q) /* L_q*Y_p - L_p*Y_q */ \
    big_mul(&t1, &L[q], &Y[p]);               \
    big_mul(&t2, &L[p], &Y[q]);               \
    big_sub(&out, &t1, &t2)
    M2(ab, 0, 1);
    M2(bc, 1, 2);
    M2(cd, 2, 3);
    M2(da, 3, 0);
    M2(ac, 0, 2);
    M2(bd, 1, 3);
#undef M2
    big_add(&s, &cd, &da);
    big_add(&cda, &s, &ac);
    big_add(&s, &da, &ab);
    big_add(&dab, &s, &bd);
    big_add(&s, &ab, &bc);
    big_sub(&abc, &s, &ac);
    big_add(&s, &bc, &cd);
    big_sub(&bcd, &s, &bd);
    big_mul(&t1, &X[0], &bcd);
    big_mul(&t2, &X[1], &cda);
    big_sub(&acc, &t1, &t2);
    big_mul(&t1, &X[2], &dab);
    big_add(&s, &acc, &t1);
    big_mul(&t2, &X[3], &abc);
    big_sub(&acc, &s, &t2);
    return big_sign(&acc);
}

/* orient2dexact_l_w (PRED:4515-4597): X_a(L_b-L_c) + X_b(L_c-L_a) + X_c(L_a-L_b) */
static int det2(const big *X, const big *L) {
    big d, t, acc, s;
    big_sub(&d, &L[1], &L[2]);
    big_mul(&acc, &X[0], &d);
    big_sub(&d, &L[2], &L[0]);
    big_mul(&t, &X[1], &d);
    big_add(&s, &acc, &t);
    big_sub(&d, &L[0], &L[1]);
    big_mul(&t, &X[2], &d);
    big_add(&acc, &s, &t);
    return big_sign(&acc);
}

/* SoS depth table restated from PRED:4719-5417: kind (3/2/1-D minor),
   lifted flag, rows (positions in sorted-index order) and the coordinate
   permutation applied to every row. */
typedef struct {
    signed char kind, lifted, rows[4], perm[3];
} sos_step;
static const sos_step SOS_TABLE[49] = {
    {0, 0, {0}, {0}},
    {3, 0, {1, 2, 3, 4}, {0, 1, 2}}, {3, 1, {1, 2, 3, 4}, {0, 1, 2}},
    {3, 1, {1, 2, 3, 4}, {0, 2, 1}}, {3, 1, {1, 2, 3, 4}, {1, 2, 0}},
    {3, 0, {0, 2, 3, 4}, {0, 1, 2}}, {2, 0, {2, 3, 4}, {0, 1}},
    {2, 0, {2, 3, 4}, {0, 2}},       {2, 0, {2, 3, 4}, {1, 2}},
    {3, 1, {0, 2, 3, 4}, {0, 1, 2}}, {2, 1, {2, 3, 4}, {0, 1, 2}},
    {2, 1, {2, 3, 4}, {1, 0, 2}},    {3, 1, {0, 2, 3, 4}, {0, 2, 1}},
    {2, 1, {2, 3, 4}, {2, 0, 1}},    {3, 1, {0, 2, 3, 4}, {1, 2, 0}},
    {3, 0, {0, 1, 3, 4}, {0, 1, 2}}, {2, 0, {1, 3, 4}, {0, 1}},
    {2, 0, {1, 3, 4}, {0, 2}},       {2, 0, {1, 3, 4}, {1, 2}},
    {2, 0, {0, 3, 4}, {0, 1}},       {1, 0, {3, 4}, {0}},
    {1, 0, {3, 4}, {1}},             {2, 0, {0, 3, 4}, {0, 2}},
    {1, 0, {3, 4}, {2}},             {2, 0, {0, 3, 4}, {1, 2}},
    {3, 1, {0, 1, 3, 4}, {0, 1, 2}}, {2, 1, {1, 3, 4}, {0, 1, 2}},
    {2, 1, {1, 3, 4}, {1, 0, 2}},    {2, 1, {0, 3, 4}, {0, 1, 2}},
    {1, 1, {3, 4}, {0, 1, 2}},       {2, 1, {0, 3, 4}, {1, 0, 2}},
    {3, 1, {0, 1, 3, 4}, {0, 2, 1}}, {2, 1, {1, 3, 4}, {2, 0, 1}},
    {2, 1, {0, 3, 4}, {2, 0, 1}},    {3, 1, {0, 1, 3, 4}, {1, 2, 0}},
    {3, 0, {0, 1, 2, 4}, {0, 1, 2}}, {2, 0, {1, 2, 4}, {0, 1}},
    {2, 0, {1, 2, 4}, {0, 2}},       {2, 0, {1, 2, 4}, {1, 2}},
    {2, 0, {0, 2, 4}, {0, 1}},       {1, 0, {2, 4}, {0}},
    {1, 0, {2, 4}, {1}},             {2, 0, {0, 2, 4}, {0, 2}},
    {1, 0, {2, 4}, {2}},             {2, 0, {0, 2, 4}, {1, 2}},
    {2, 0, {0, 1, 4}, {0, 1}},       {1, 0, {1, 4}, {0}},
    {1, 0, {1, 4}, {1}},             {1, 0, {0, 4}, {0}},
};
/* depths whose minor sign is negated (PRED:5419-5450) */
static int sos_flip(int d) {
    switch (d) {
    case 1: case 3: case 7: case 9: case 11: case 14: case 15: case 16:
    case 18: case 20: case 22: case 23: case 26: case 30: case 31: case 32:
    case 37: case 39: case 41: case 44: case 46:
        return 1;
    default:
        return 0;
    }
}

static int sos_minor(const sos_pts *s, int d) {
    const sos_step *st = &SOS_TABLE[d];
    big X[4], Y[4], L[4], t;
    if (st->kind == 3) {
        for (int r = 0; r < 4; r++) {
            int p = st->rows[r];
            X[r] = s->c[p][st->perm[0]];
            Y[r] = s->c[p][st->perm[1]];
            L[r] = st->lifted ? s->lift[p] : s->c[p][st->perm[2]];
        }
        return det3(X, Y, L);
    }
    if (st->kind == 2) {
        for (int r = 0; r < 3; r++) {
            int p = st->rows[r];
            X[r] = s->c[p][st->perm[0]];
            L[r] = st->lifted ? s->lift[p] : s->c[p][st->perm[1]];
        }
        return det2(X, L);
    }
    /* 1-D */
    int a = st->rows[0], b = st->rows[1];
    if (!st->lifted) {
        big_sub(&t, &s->c[a][st->perm[0]], &s->c[b][st->perm[0]]);
        return big_sign(&t);
    }
    /* orient1dexact_l_w lifted (PRED:4605-4647): |a|^2 - |b|^2 + (wa - wb) */
    big la, lb;
    big_add(&la, &s->lift[a], &s->w2[a]);
    big_add(&la, &la, &s->w2[a]);
    big_add(&lb, &s->lift[b], &s->w2[b]);
    big_add(&lb, &lb, &s->w2[b]);
    big_sub(&t, &la, &lb);
    return big_sign(&t);
}

static int sos4_impl(const float *p0, const float *p1, const float *p2,
                     const float *p3, const float *p4, float w0, float w1,
                     float w2, float w3, float w4, int i0, int i1, int i2,
                     int i3, int i4, int radii, int *depth_out);
int orc_sos4(const float *p0, const float *p1, const float *p2,
             const float *p3, const float *p4, float w0, float w1, float w2,
             float w3, float w4, int i0, int i1, int i2, int i3, int i4,
             int *depth_out) {
    return sos4_impl(p0, p1, p2, p3, p4, w0, w1, w2, w3, w4, i0, i1, i2, i3,
                     i4, 0, depth_out);
}
static int sos4_impl(const float *p0, const float *p1, const float *p2,
                     const float *p3, const float *p4, float w0, float w1,
                     float w2, float w3, float w4, int i0, int i1, int i2,
                     int i3, int i4, int radii, int *depth_out) {
    /* bubble sort of the indices recording the swap parity (PRED:4676-4707) */
    int idx[5] = {i0, i1, i2, i3, i4}, ord[5] = {0, 1, 2, 3, 4};
    int swaps = 0;
    for (int i = 0; i < 4; i++)
        for (int j = 4; j > i; j--)
            if (idx[j] < idx[j - 1]) {
                int t = idx[j]; idx[j] = idx[j - 1]; idx[j - 1] = t;
                t = ord[j]; ord[j] = ord[j - 1]; ord[j - 1] = t;
                swaps++;
            }
    const float *pts[5] = {p0, p1, p2, p3, p4};
    const float ws[5] = {w0, w1, w2, w3, w4};
    float *ip[5];
    float iw[5];
    for (int i = 0; i < 5; i++) {
        ip[i] = (float *)pts[ord[i]];
        iw[i] = ws[ord[i]];
    }
    sos_pts s;
    sos_load(&s, ip, iw, radii);
    int sign = 0, d;
    for (d = 1; d <= 48 && !sign; d++) sign = sos_minor(&s, d);
    d--;
    if (!sign) {
        /* the reference loops forever here (PRED:5409-5411 keeps orient at
           zero); the restatement stops and reports positive */
        sign = 1;
        d = 49;
    }
    if (sos_flip(d)) sign = -sign;
    if (swaps & 1) sign = -sign;
    if (depth_out) *depth_out = s.overflow ? -1 : d;
    return sign;
}

/* ------------------------------------------------------------------ */
/* Decision-exact predicates (ORC_EXACT): exact_oracle.cpp evaluates     */
/* them (extended-precision filter, then arbitrary-precision integers);  */
/* here the balls are handed over as (x, y, z, r) rows.                  */
int oex_edge(const float *b, float alpha);
int oex_tri(const float *b, float alpha);
int oex_tet(const float *b, float alpha);
int oex_orient(const float *b);
int oex_insphere(const float *b);
int oex_edge_attached(const float *b);
int oex_tri_attached(const float *b);
#define ORC_XV 2 /* internal formula code of the exact mode */

static void x_rows(float *b, const oatom *const *a, int k) {
    for (int i = 0; i < k; i++) {
        b[4 * i] = a[i]->x; b[4 * i + 1] = a[i]->y;
        b[4 * i + 2] = a[i]->z; b[4 * i + 3] = a[i]->r;
    }
}
static int x_edge(const oatom *a1, const oatom *a2, float alpha) {
    const oatom *a[2] = {a1, a2};
    float b[8];
    x_rows(b, a, 2);
    return oex_edge(b, alpha);
}
static int x_tri(const oatom *a1, const oatom *a2, const oatom *a3, float alpha) {
    const oatom *a[3] = {a1, a2, a3};
    float b[12];
    x_rows(b, a, 3);
    return oex_tri(b, alpha);
}
static int x_tet(const oatom *a1, const oatom *a2, const oatom *a3, const oatom *a4,
                 float alpha, int *flat) {
    const oatom *a[4] = {a1, a2, a3, a4};
    float b[16];
    x_rows(b, a, 4);
    int r = oex_tet(b, alpha);
    *flat = r == 2;
    return r != 0;
}
/* s[0..nv-1]: the simplex (nv = 2 or 3); q: the other ball */
static int x_attached(const oatom *const *s, int nv, const oatom *q) {
    const oatom *a[4] = {s[0], s[1], nv == 3 ? s[2] : q, q};
    float b[16];
    x_rows(b, a, nv + 1);
    return nv == 2 ? oex_edge_attached(b) : oex_tri_attached(b);
}
static int x_orient(const oatom *pa, const oatom *pb, const oatom *pc, const oatom *pd) {
    const oatom *a[4] = {pa, pb, pc, pd};
    float b[16];
    x_rows(b, a, 4);
    return oex_orient(b);
}
static int x_insphere(const oatom *const *a5) {
    float b[20];
    x_rows(b, a5, 5);
    return oex_insphere(b);
}

/* FP64 window centres of the exact mode (the decisions do not use them);
   the engine computes the same double operations in the same order. */
static void x_edge_centre(const oatom *a1, const oatom *a2, float *c) {
    const double ux = (double)a2->x - a1->x, uy = (double)a2->y - a1->y,
                 uz = (double)a2->z - a1->z;
    const double uu = ux * ux + uy * uy + uz * uz;
    const double w1 = (double)a1->r * a1->r, w2 = (double)a2->r * a2->r;
    const double t = (uu + w1 - w2) / (2.0 * uu);
    c[0] = (float)(a1->x + t * ux);
    c[1] = (float)(a1->y + t * uy);
    c[2] = (float)(a1->z + t * uz);
}
static void x_tri_centre(const oatom *a1, const oatom *a2, const oatom *a3, float *c) {
    const double ux = (double)a2->x - a1->x, uy = (double)a2->y - a1->y,
                 uz = (double)a2->z - a1->z;
    const double vx = (double)a3->x - a1->x, vy = (double)a3->y - a1->y,
                 vz = (double)a3->z - a1->z;
    const double nx = uy * vz - uz * vy, ny = uz * vx - ux * vz, nz = ux * vy - uy * vx;
    const double w1 = (double)a1->r * a1->r;
    const double B2 = ux * ux + uy * uy + uz * uz + w1 - (double)a2->r * a2->r;
    const double B3 = vx * vx + vy * vy + vz * vz + w1 - (double)a3->r * a3->r;
    const double cx = B2 * (vy * nz - vz * ny) + B3 * (ny * uz - nz * uy);
    const double cy = B2 * (vz * nx - vx * nz) + B3 * (nz * ux - nx * uz);
    const double cz = B2 * (vx * ny - vy * nx) + B3 * (nx * uy - ny * ux);
    const double k = 1.0 / (2.0 * (nx * nx + ny * ny + nz * nz));
    c[0] = (float)(a1->x + cx * k);
    c[1] = (float)(a1->y + cy * k);
    c[2] = (float)(a1->z + cz * k);
}
static void x_tet_centre(const oatom *a1, const oatom *a2, const oatom *a3,
                         const oatom *a4, float *c) {
    const double ux = (double)a2->x - a1->x, uy = (double)a2->y - a1->y,
                 uz = (double)a2->z - a1->z;
    const double vx = (double)a3->x - a1->x, vy = (double)a3->y - a1->y,
                 vz = (double)a3->z - a1->z;
    const double sx = (double)a4->x - a1->x, sy = (double)a4->y - a1->y,
                 sz = (double)a4->z - a1->z;
    const double w1 = (double)a1->r * a1->r;
    const double B2 = ux * ux + uy * uy + uz * uz + w1 - (double)a2->r * a2->r;
    const double B3 = vx * vx + vy * vy + vz * vz + w1 - (double)a3->r * a3->r;
    const double B4 = sx * sx + sy * sy + sz * sz + w1 - (double)a4->r * a4->r;
    const double vsx = vy * sz - vz * sy, vsy = vz * sx - vx * sz, vsz = vx * sy - vy * sx;
    const double sux = sy * uz - sz * uy, suy = sz * ux - sx * uz, suz = sx * uy - sy * ux;
    const double uvx = uy * vz - uz * vy, uvy = uz * vx - ux * vz, uvz = ux * vy - uy * vx;
    const double d = ux * vsx + uy * vsy + uz * vsz;
    const double k = 1.0 / (2.0 * d);
    c[0] = (float)(a1->x + (B2 * vsx + B3 * sux + B4 * uvx) * k);
    c[1] = (float)(a1->y + (B2 * vsy + B3 * suy + B4 * uvy) * k);
    c[2] = (float)(a1->z + (B2 * vsz + B3 * suz + B4 * uvz) * k);
}

/* ------------------------------------------------------------------ */
/* Reference-formula filters                                            */

/* markRealEdges: LD:167-190 (upstream), PLAIN:203-230 (plain-xmp) */
static int edge_alpha(const oatom *a1, const oatom *a2, float alpha,
                      int variant) {
    if (variant == ORC_XV) return x_edge(a1, a2, alpha);
    float a = a1->x - a2->x;
    float b = a1->y - a2->y;
    float c = a1->z - a2->z;
    float d = (a1->x * a1->x - a2->x * a2->x) + (a1->y * a1->y - a2->y * a2->y);
    d = d + (a1->z * a1->z - a2->z * a2->z);
    d = d - (a1->r * a1->r);
    d = d + (a2->r * a2->r);
    d = d / 2.0f;
    float t = d - a * a1->x;
    t = t - b * a1->y;
    t = t - c * a1->z;
    float nn = a * a + b * b;
    nn = nn + c * c;
    if (variant == ORC_UPSTREAM) {
        float cur = (t * t) / nn - (a1->r * a1->r);
        return (double)cur <= (double)alpha + 0.0;
    }
    float term = (t * t) - (a1->r * a1->r) * nn;
    return (double)term <= ((double)alpha + 0.0) * (double)nn;
}

/* markRealTriangles: LD:298-348 (upstream), PLAIN:310-372 (plain-xmp).
   Writes the orthosphere (X, Y, Z, power). */
static int tri_alpha(const oatom *a1, const oatom *a2, const oatom *a3,
                     float alpha, int variant, float *ortho) {
    if (variant == ORC_XV) {
        int m = x_tri(a1, a2, a3, alpha);
        ortho[0] = ortho[1] = ortho[2] = ortho[3] = 0.0f;
        if (m) x_tri_centre(a1, a2, a3, ortho);
        return m;
    }
    float a11 = a1->x - a2->x, a12 = a1->y - a2->y, a13 = a1->z - a2->z;
    float b1 = (a1->x * a1->x - a2->x * a2->x) + (a1->y * a1->y - a2->y * a2->y);
    b1 = b1 + (a1->z * a1->z - a2->z * a2->z);
    b1 = b1 - (a1->r * a1->r);
    b1 = b1 + (a2->r * a2->r);
    if (variant == ORC_UPSTREAM) b1 = b1 / 2.0f;
    float a21 = a2->x - a3->x, a22 = a2->y - a3->y, a23 = a2->z - a3->z;
    float b2 = (a2->x * a2->x - a3->x * a3->x) + (a2->y * a2->y - a3->y * a3->y);
    b2 = b2 + (a2->z * a2->z - a3->z * a3->z);
    b2 = b2 - (a2->r * a2->r);
    b2 = b2 + (a3->r * a3->r);
    if (variant == ORC_UPSTREAM) b2 = b2 / 2.0f;
    float a31 = (a2->y - a1->y) * (a3->z - a1->z) - (a3->y - a1->y) * (a2->z - a1->z);
    float a32 = (a2->z - a1->z) * (a3->x - a1->x) - (a3->z - a1->z) * (a2->x - a1->x);
    float a33 = (a2->x - a1->x) * (a3->y - a1->y) - (a3->x - a1->x) * (a2->y - a1->y);
    float b3 = a31 * a1->x + a32 * a1->y;
    if (variant == ORC_UPSTREAM)
        b3 = b3 + a33 * a1->z;
    else
        b3 = b3 + (a33 * a1->z) * 2.0f; /* PLAIN:344 precedence as written */
#define T3(p, q, r) (((p) * (q)) * (r))
    float D = T3(a11, a22, a33) + T3(a12, a23, a31);
    D = D + T3(a13, a21, a32);
    D = D - T3(a13, a22, a31);
    D = D - T3(a12, a21, a33);
    D = D - T3(a11, a23, a32);
    float Dx = T3(b1, a22, a33) + T3(a12, a23, b3);
    Dx = Dx + T3(a13, b2, a32);
    Dx = Dx - T3(a13, a22, b3);
    Dx = Dx - T3(a12, b2, a33);
    Dx = Dx - T3(b1, a23, a32);
    float Dy = T3(a11, b2, a33) + T3(b1, a23, a31);
    Dy = Dy + T3(a13, a21, b3);
    Dy = Dy - T3(a13, b2, a31);
    Dy = Dy - T3(b1, a21, a33);
    Dy = Dy - T3(a11, a23, b3);
    float Dz = T3(a11, a22, b3) + T3(a12, b2, a31);
    Dz = Dz + T3(b1, a21, a32);
    Dz = Dz - T3(b1, a22, a31);
    Dz = Dz - T3(a12, a21, b3);
    Dz = Dz - T3(a11, b2, a32);
#undef T3
    if (variant == ORC_UPSTREAM) {
        float X = Dx / D, Y = Dy / D, Z = Dz / D;
        float dist = (a1->x - X) * (a1->x - X) + (a1->y - Y) * (a1->y - Y);
        dist = dist + (a1->z - Z) * (a1->z - Z);
        dist = dist - a1->r * a1->r;
        ortho[0] = X; ortho[1] = Y; ortho[2] = Z; ortho[3] = dist;
        return (double)dist <= (double)alpha + 0.0;
    }
    D = D * 2.0f;
    float X = Dx, Y = Dy, Z = Dz;
    float ex = a1->x * D - X, ey = a1->y * D - Y, ez = a1->z * D - Z;
    float dist = ex * ex + ey * ey;
    dist = dist + ez * ez;
    dist = dist - ((a1->r * a1->r) * D) * D;
    int mark = (double)dist <= (((double)alpha + 0.0) * (double)D) * (double)D;
    X = X / D; Y = Y / D; Z = Z / D;
    dist = dist / (D * D);
    ortho[0] = X; ortho[1] = Y; ortho[2] = Z; ortho[3] = dist;
    return mark;
}

/* markRealTets: LD:531-591 (identical in both variants) */
static int tet_alpha(const oatom *a1, const oatom *a2, const oatom *a3,
                     const oatom *a4, float alpha, int variant, float *ortho) {
    if (variant == ORC_XV) {
        int flat, m = x_tet(a1, a2, a3, a4, alpha, &flat);
        ortho[0] = ortho[1] = ortho[2] = ortho[3] = 0.0f;
        if (m && !flat) x_tet_centre(a1, a2, a3, a4, ortho);
        return m;
    }
    float a11 = a1->x - a2->x, a12 = a1->y - a2->y, a13 = a1->z - a2->z;
    float b1 = (a1->x * a1->x - a2->x * a2->x) + (a1->y * a1->y - a2->y * a2->y);
    b1 = b1 + (a1->z * a1->z - a2->z * a2->z);
    b1 = b1 - (a1->r * a1->r);
    b1 = b1 + (a2->r * a2->r);
    b1 = b1 / 2.0f;
    float a21 = a2->x - a3->x, a22 = a2->y - a3->y, a23 = a2->z - a3->z;
    float b2 = (a2->x * a2->x - a3->x * a3->x) + (a2->y * a2->y - a3->y * a3->y);
    b2 = b2 + (a2->z * a2->z - a3->z * a3->z);
    b2 = b2 - (a2->r * a2->r);
    b2 = b2 + (a3->r * a3->r);
    b2 = b2 / 2.0f;
    float a31 = a3->x - a4->x, a32 = a3->y - a4->y, a33 = a3->z - a4->z;
    float b3 = (a3->x * a3->x - a4->x * a4->x) + (a3->y * a3->y - a4->y * a4->y);
    b3 = b3 + (a3->z * a3->z - a4->z * a4->z);
    b3 = b3 - (a3->r * a3->r);
    b3 = b3 + (a4->r * a4->r);
    b3 = b3 / 2.0f;
#define T3(p, q, r) (((p) * (q)) * (r))
    float D = T3(a11, a22, a33) + T3(a12, a23, a31);
    D = D + T3(a13, a21, a32);
    D = D - T3(a13, a22, a31);
    D = D - T3(a12, a21, a33);
    D = D - T3(a11, a23, a32);
    float Dx = T3(b1, a22, a33) + T3(a12, a23, b3);
    Dx = Dx + T3(a13, b2, a32);
    Dx = Dx - T3(a13, a22, b3);
    Dx = Dx - T3(a12, b2, a33);
    Dx = Dx - T3(b1, a23, a32);
    float Dy = T3(a11, b2, a33) + T3(b1, a23, a31);
    Dy = Dy + T3(a13, a21, b3);
    Dy = Dy - T3(a13, b2, a31);
    Dy = Dy - T3(b1, a21, a33);
    Dy = Dy - T3(a11, a23, b3);
    float Dz = T3(a11, a22, b3) + T3(a12, b2, a31);
    Dz = Dz + T3(b1, a21, a32);
    Dz = Dz - T3(b1, a22, a31);
    Dz = Dz - T3(a12, a21, b3);
    Dz = Dz - T3(a11, b2, a32);
#undef T3
    if (D == 0.0f) {
        ortho[0] = ortho[1] = ortho[2] = ortho[3] = 0.0f;
        return 1;
    }
    float X = Dx / D, Y = Dy / D, Z = Dz / D;
    float dist = (a2->x - X) * (a2->x - X) + (a2->y - Y) * (a2->y - Y);
    dist = dist + (a2->z - Z) * (a2->z - Z);
    dist = dist - a2->r * a2->r;
    ortho[0] = X; ortho[1] = Y; ortho[2] = Z; ortho[3] = dist;
    return (double)dist <= (double)alpha + 0.0;
}

/* ------------------------------------------------------------------ */
/* Grid                                                                 */
typedef struct {
    float minx, miny, minz, step;
    int32_t gx, gy, gz;
    int64_t ncell;
    const uint32_t *begin, *end;
} grid_t;

/* The 27-cell window around a point (LD:621-733, 812-871, 951-1009):
   the centre cell is read through its linear index without a range check
   (a wrapped cell when one coordinate leaves the grid); the 26 neighbours
   are range-checked per axis.  A centre index outside [0, ncell) is
   undefined behaviour in the reference; here it reads as an empty cell
   and is counted.  Visits atoms through cb(ctx, atom) until it returns
   nonzero; returns that value. */
typedef int (*visit_fn)(void *ctx, uint32_t atom);
static int window_visit(const grid_t *g, float px, float py, float pz,
                        visit_fn cb, void *ctx, uint64_t *oob) {
    int32_t X = f2i((px - g->minx) / g->step);
    int32_t Y = f2i((py - g->miny) / g->step);
    int32_t Z = f2i((pz - g->minz) / g->step);
    int32_t c = lin3(X, Y, Z, g->gx, g->gy);
    if (c >= 0 && (int64_t)c < g->ncell) {
        for (uint32_t a = g->begin[c]; a < g->end[c]; a++) {
            int r = cb(ctx, a);
            if (r) return r;
        }
    } else if (oob) {
#pragma omp atomic
        (*oob)++;
    }
    for (int i = -1; i < 2; i++)
        for (int j = -1; j < 2; j++)
            for (int k = -1; k < 2; k++) {
                if (i == 0 && j == 0 && k == 0) continue;
                int32_t zz = wadd(Z, i), yy = wadd(Y, j), xx = wadd(X, k);
                if (zz >= g->gz || yy >= g->gy || xx >= g->gx) continue;
                if (zz < 0 || yy < 0 || xx < 0) continue;
                int32_t oc = lin3(xx, yy, zz, g->gx, g->gy);
                for (uint32_t a = g->begin[oc]; a < g->end[oc]; a++) {
                    int r = cb(ctx, a);
                    if (r) return r;
                }
            }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Window callbacks                                                     */
typedef struct {
    const oatom *at;
    uint32_t v[4];
    float pa[3], pb[3], pc[3], pd[3];
    float wa, wb, wc, wd;
    float orientation;
    int exact;
    uint64_t evals, sos, sos_exh;
} tet_ctx;

/* checkTetsOrthosphere per-atom test (LD:630-670): 1 = violation */
static int tet_visit(void *vctx, uint32_t a) {
    tet_ctx *t = (tet_ctx *)vctx;
    if (a == t->v[0] || a == t->v[1] || a == t->v[2] || a == t->v[3])
        return 0;
    const oatom *e = &t->at[a];
    float pe[3] = {e->x, e->y, e->z};
    float we = e->r * e->r;
    t->evals++;
    float res;
    if (t->exact) {
        const oatom *a5[5] = {&t->at[t->v[0]], &t->at[t->v[1]], &t->at[t->v[2]],
                              &t->at[t->v[3]], e};
        res = (float)x_insphere(a5);
    } else {
        res = orc_insphere_w(t->pa, t->pb, t->pc, t->pd, pe, t->wa, t->wb,
                             t->wc, t->wd, we);
    }
    if (res == 0.0f) {
        int depth;
        t->sos++;
        /* exact mode: the weights are the radii squared exactly */
        res = (float)sos4_impl(
            t->pa, t->pb, t->pc, t->pd, pe,
            t->exact ? t->at[t->v[0]].r : t->wa, t->exact ? t->at[t->v[1]].r : t->wb,
            t->exact ? t->at[t->v[2]].r : t->wc, t->exact ? t->at[t->v[3]].r : t->wd,
            t->exact ? e->r : we, (int)t->at[t->v[0]].idx, (int)t->at[t->v[1]].idx,
            (int)t->at[t->v[2]].idx, (int)t->at[t->v[3]].idx, (int)e->idx,
            t->exact, &depth);
        if (depth == 49) t->sos_exh++;
    }
    if (t->orientation < 0) return res < 0;
    return res > 0;
}

typedef struct {
    const oatom *at;
    uint32_t v[3];
    int nv;
    int exact;
    float px, py, pz, cur;
} att_ctx;

/* attachment tests of checkDanglingTris / checkDanglingEdges
   (LD:819-871, 958-1009): 1 = some other ball is at least as close */
static int att_visit(void *vctx, uint32_t a) {
    att_ctx *t = (att_ctx *)vctx;
    for (int i = 0; i < t->nv; i++)
        if (a == t->v[i]) return 0;
    const oatom *e = &t->at[a];
    if (t->exact) {
        const oatom *sv[3] = {&t->at[t->v[0]], &t->at[t->v[1]],
                              t->nv == 3 ? &t->at[t->v[2]] : NULL};
        return x_attached(sv, t->nv, e);
    }
    float dx = e->x - t->px, dy = e->y - t->py, dz = e->z - t->pz;
    float pw = dx * dx + dy * dy;
    pw = pw + dz * dz;
    pw = pw - (e->r * e->r);
    return (double)pw + 0.0 <= (double)t->cur;
}

/* ------------------------------------------------------------------ */
static int cmp_tri(const void *a, const void *b) {
    const uint32_t *x = (const uint32_t *)a, *y = (const uint32_t *)b;
    for (int i = 0; i < 3; i++)
        if (x[i] != y[i]) return x[i] < y[i] ? -1 : 1;
    return 0;
}
static int cmp_edge(const void *a, const void *b) {
    const uint32_t *x = (const uint32_t *)a, *y = (const uint32_t *)b;
    for (int i = 0; i < 2; i++)
        if (x[i] != y[i]) return x[i] < y[i] ? -1 : 1;
    return 0;
}
static int64_t find2(const uint32_t *B, const uint32_t *C, uint64_t lo,
                     uint64_t hi, uint32_t b, uint32_t c) {
    uint64_t l = lo, h = hi;
    while (l < h) {
        uint64_t m = (l + h) / 2;
        if (B[m] < b || (B[m] == b && C[m] < c))
            l = m + 1;
        else
            h = m;
    }
    if (l < hi && B[l] == b && C[l] == c) return (int64_t)l;
    return -1;
}
static int64_t find1(const uint32_t *B, uint64_t lo, uint64_t hi, uint32_t b) {
    uint64_t l = lo, h = hi;
    while (l < h) {
        uint64_t m = (l + h) / 2;
        if (B[m] < b)
            l = m + 1;
        else
            h = m;
    }
    if (l < hi && B[l] == b) return (int64_t)l;
    return -1;
}

#define XMALLOC(T, n) ((T *)malloc(sizeof(T) * ((size_t)(n) > 0 ? (size_t)(n) : 1)))

int orc_alpha_complex(const float *xyzr, uint32_t n, float sol, float alpha,
                      int variant, int flags, int threads, orc_result *res) {
    memset(res, 0, sizeof(*res));
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    if (n == 0) return 0;
    const int exact = (flags & ORC_EXACT) != 0;
    if (exact) variant = ORC_XV;
    /* ---- input, bounding box (LD:1078-1111) ---- */
    oatom *in = XMALLOC(oatom, n);
    float minx = 0, miny = 0, minz = 0, maxx = 0, maxy = 0, maxz = 0;
    float minr = 0, maxr = 0;
    for (uint32_t i = 0; i < n; i++) {
        float x = xyzr[4 * i], y = xyzr[4 * i + 1], z = xyzr[4 * i + 2];
        float r = xyzr[4 * i + 3];
        in[i].x = x; in[i].y = y; in[i].z = z;
        in[i].r = r + sol;
        in[i].idx = i + 1;
        if (i == 0) {
            minx = maxx = x; miny = maxy = y; minz = maxz = z;
            minr = maxr = r;
        } else {
            if (x < minx) minx = x; else if (x > maxx) maxx = x;
            if (y < miny) miny = y; else if (y > maxy) maxy = y;
            if (z < minz) minz = z; else if (z > maxz) maxz = z;
            if (r < minr) minr = r; else if (r > maxr) maxr = r;
        }
    }
    /* ---- grid parameters (LD:1119-1123) ---- */
    float pmr = sqrtf(maxr * maxr + alpha);
    float step = 2.0f * pmr;
    int32_t gx = (int32_t)((maxx - minx) / step) + 1;
    int32_t gy = (int32_t)((maxy - miny) / step) + 1;
    int32_t gz = (int32_t)((maxz - minz) / step) + 1;
    int64_t ncell = (int64_t)gx * gy * gz;
    res->grid[0] = gx; res->grid[1] = gy; res->grid[2] = gz;
    res->step = step;
    /* ---- cell keys and stable sort (LD:65-78, 1164-1177) ---- */
    uint32_t *key = XMALLOC(uint32_t, n);
    for (uint32_t i = 0; i < n; i++) {
        int32_t cx = f2i((in[i].x - minx) / step);
        int32_t cy = f2i((in[i].y - miny) / step);
        int32_t cz = f2i((in[i].z - minz) / step);
        key[i] = (uint32_t)(cx + gx * cy + gx * gy * cz);
    }
    uint32_t *cbeg = XMALLOC(uint32_t, ncell), *cend = XMALLOC(uint32_t, ncell);
    memset(cbeg, 0, sizeof(uint32_t) * ncell);
    for (uint32_t i = 0; i < n; i++) cbeg[key[i]]++;
    {
        uint32_t run = 0;
        for (int64_t c = 0; c < ncell; c++) {
            uint32_t k = cbeg[c];
            cbeg[c] = run;
            run += k;
            cend[c] = run;
        }
    }
    oatom *at = XMALLOC(oatom, n);
    uint32_t *cellof = XMALLOC(uint32_t, n);
    {
        uint32_t *fill = XMALLOC(uint32_t, ncell);
        memcpy(fill, cbeg, sizeof(uint32_t) * ncell);
        for (uint32_t i = 0; i < n; i++) {
            uint32_t p = fill[key[i]]++;
            at[p] = in[i];
            cellof[p] = key[i];
        }
        free(fill);
    }
    grid_t g = {minx, miny, minz, step, gx, gy, gz, ncell, cbeg, cend};

    /* ---- candidate edges + alpha filter (LD:80-190, 1237-1296) ---- */
    uint64_t *ecnt = XMALLOC(uint64_t, n + 1);
    uint64_t *eoff = XMALLOC(uint64_t, n + 1);
    uint64_t cand_e = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : cand_e)
    for (uint32_t i = 0; i < n; i++) {
        int32_t cell = (int32_t)cellof[i];
        int32_t X = cell % gx, t = cell / gx, Y = t % gy, Z = t / gy;
        uint64_t c = 0, ca = 0;
        for (int di = -1; di < 2; di++)
            for (int dj = -1; dj < 2; dj++)
                for (int dk = -1; dk < 2; dk++) {
                    if (Z + di >= gz || Y + dj >= gy || X + dk >= gx) continue;
                    if (Z + di < 0 || Y + dj < 0 || X + dk < 0) continue;
                    int32_t adj = (Z + di) * gx * gy + (Y + dj) * gx + (X + dk);
                    if (adj < cell) continue;
                    for (uint32_t l = cbeg[adj]; l < cend[adj]; l++)
                        if (l > i) {
                            c++;
                            ca += edge_alpha(&at[i], &at[l], alpha, variant);
                        }
                }
        cand_e += c;
        ecnt[i] = ca;
    }
    res->cand_edges = cand_e;
    eoff[0] = 0;
    for (uint32_t i = 0; i < n; i++) eoff[i + 1] = eoff[i] + ecnt[i];
    uint64_t nE = eoff[n];
    uint32_t *EL = XMALLOC(uint32_t, nE), *ER = XMALLOC(uint32_t, nE);
#pragma omp parallel for schedule(dynamic, 256)
    for (uint32_t i = 0; i < n; i++) {
        int32_t cell = (int32_t)cellof[i];
        int32_t X = cell % gx, t = cell / gx, Y = t % gy, Z = t / gy;
        uint64_t o = eoff[i];
        for (int di = -1; di < 2; di++)
            for (int dj = -1; dj < 2; dj++)
                for (int dk = -1; dk < 2; dk++) {
                    if (Z + di >= gz || Y + dj >= gy || X + dk >= gx) continue;
                    if (Z + di < 0 || Y + dj < 0 || X + dk < 0) continue;
                    int32_t adj = (Z + di) * gx * gy + (Y + dj) * gx + (X + dk);
                    if (adj < cell) continue;
                    for (uint32_t l = cbeg[adj]; l < cend[adj]; l++)
                        if (l > i && edge_alpha(&at[i], &at[l], alpha, variant)) {
                            EL[o] = i;
                            ER[o] = l;
                            o++;
                        }
                }
    }
    res->alpha_edges = nE;
    /* the per-atom lists come out sorted by right vertex, so the stable
       sort by left vertex (LD:1295) leaves them as they are */

    /* ---- candidate triangles + alpha filter (LD:192-348) ---- */
    uint64_t *tcnt = XMALLOC(uint64_t, n + 1), *toff = XMALLOC(uint64_t, n + 1);
    uint64_t cand_t = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : cand_t)
    for (uint32_t i = 0; i < n; i++) {
        uint64_t b = eoff[i], e = eoff[i + 1], c = 0, ca = 0;
        float o4[4];
        for (uint64_t p = b; p < e; p++) {
            uint32_t v1 = ER[p];
            for (uint64_t q = p + 1; q < e; q++) {
                uint32_t v2 = ER[q];
                if (find1(ER, eoff[v1], eoff[v1 + 1], v2) >= 0) {
                    c++;
                    ca += tri_alpha(&at[i], &at[v1], &at[v2], alpha, variant, o4);
                }
            }
        }
        cand_t += c;
        tcnt[i] = ca;
    }
    res->cand_tris = cand_t;
    toff[0] = 0;
    for (uint32_t i = 0; i < n; i++) toff[i + 1] = toff[i] + tcnt[i];
    uint64_t nT = toff[n];
    uint32_t *T1 = XMALLOC(uint32_t, nT), *T2 = XMALLOC(uint32_t, nT),
             *T3 = XMALLOC(uint32_t, nT);
    float *TO = XMALLOC(float, 4 * nT);
#pragma omp parallel for schedule(dynamic, 64)
    for (uint32_t i = 0; i < n; i++) {
        uint64_t b = eoff[i], e = eoff[i + 1], o = toff[i];
        for (uint64_t p = b; p < e; p++) {
            uint32_t v1 = ER[p];
            for (uint64_t q = p + 1; q < e; q++) {
                uint32_t v2 = ER[q];
                float o4[4];
                if (find1(ER, eoff[v1], eoff[v1 + 1], v2) >= 0 &&
                    tri_alpha(&at[i], &at[v1], &at[v2], alpha, variant, o4)) {
                    T1[o] = i; T2[o] = v1; T3[o] = v2;
                    memcpy(&TO[4 * o], o4, 16);
                    o++;
                }
            }
        }
    }
    res->alpha_tris = nT;

    /* ---- candidate tetrahedra + alpha filter (LD:350-591) and the
            empty-orthosphere test (LD:597-735) ---- */
    uint64_t *qcnt = XMALLOC(uint64_t, n + 1), *qoff = XMALLOC(uint64_t, n + 1);
    uint32_t *Q = NULL, *FQ = NULL;
    float *QO = NULL;
    unsigned char *qkeep = NULL;
    uint64_t cand_q = 0, nQ = 0, nF = 0;
    uint64_t evals = 0, sos = 0, sosx = 0, oob = 0;
    if (flags & ORC_TET_ORTHO) {
        /* Each alpha tetrahedron is tested as soon as it is found and only
           survivors are kept: at 2.5 M balls there are 6.7 G alpha
           tetrahedra, too many to hold.  A ball is handled by one thread, in
           enumeration order, so collecting (ball, tetrahedron) per thread and
           placing them by per-ball survivor counts gives the reference's
           order (ball ascending, enumeration order within a ball). */
        int nth = 1;
#ifdef _OPENMP
        nth = omp_get_max_threads();
#endif
        uint32_t **tb = (uint32_t **)calloc((size_t)nth, sizeof(uint32_t *));
        uint64_t *tn = (uint64_t *)calloc((size_t)nth, sizeof(uint64_t));
        uint64_t *tcap = (uint64_t *)calloc((size_t)nth, sizeof(uint64_t));
        uint64_t alpha_q = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : cand_q, alpha_q, evals, sos, sosx)
        for (uint32_t i = 0; i < n; i++) {
            int me = 0;
#ifdef _OPENMP
            me = omp_get_thread_num();
#endif
            uint64_t b = toff[i], e = toff[i + 1], c = 0, ca = 0, kept = 0;
            float o4[4];
            uint64_t g0 = b;
            while (g0 < e) {
                uint32_t v2 = T2[g0];
                uint64_t g1 = g0 + 1;
                while (g1 < e && T2[g1] == v2) g1++;
                for (uint64_t j = g0; j < g1; j++) {
                    uint32_t v3 = T3[j];
                    for (uint64_t k = j + 1; k < g1; k++) {
                        uint32_t v4 = T3[k];
                        if (find2(T2, T3, b, e, v3, v4) < 0) continue;
                        if (find2(T2, T3, toff[v2], toff[v2 + 1], v3, v4) < 0) continue;
                        c++;
                        if (!tet_alpha(&at[i], &at[v2], &at[v3], &at[v4], alpha, variant, o4))
                            continue;
                        ca++;
                        tet_ctx t;
                        t.at = at;
                        t.v[0] = i; t.v[1] = v2; t.v[2] = v3; t.v[3] = v4;
                        const oatom *a1 = &at[i], *a2 = &at[v2], *a3 = &at[v3], *a4 = &at[v4];
                        t.pa[0] = a1->x; t.pa[1] = a1->y; t.pa[2] = a1->z; t.wa = a1->r * a1->r;
                        t.pb[0] = a2->x; t.pb[1] = a2->y; t.pb[2] = a2->z; t.wb = a2->r * a2->r;
                        t.pc[0] = a3->x; t.pc[1] = a3->y; t.pc[2] = a3->z; t.wc = a3->r * a3->r;
                        t.pd[0] = a4->x; t.pd[1] = a4->y; t.pd[2] = a4->z; t.wd = a4->r * a4->r;
                        t.exact = exact;
                        t.orientation = exact ? (float)x_orient(a1, a2, a3, a4)
                                              : orc_orient3d(t.pa, t.pb, t.pc, t.pd);
                        t.evals = t.sos = t.sos_exh = 0;
                        uint64_t oob1 = 0;
                        int viol = window_visit(&g, o4[0], o4[1], o4[2], tet_visit, &t, &oob1);
                        evals += t.evals;
                        sos += t.sos;
                        sosx += t.sos_exh;
                        if (oob1) {
#pragma omp atomic
                            oob += oob1;
                        }
                        if (viol) continue;
                        if (tn[me] == tcap[me]) {
                            tcap[me] = tcap[me] ? 2 * tcap[me] : 4096;
                            tb[me] = (uint32_t *)realloc(tb[me], 16 * tcap[me]);
                        }
                        uint32_t *o = &tb[me][4 * tn[me]++];
                        o[0] = i; o[1] = v2; o[2] = v3; o[3] = v4;
                        kept++;
                    }
                }
                g0 = g1;
            }
            cand_q += c;
            alpha_q += ca;
            qcnt[i] = kept;
        }
        res->cand_tets = cand_q;
        nQ = alpha_q;
        qoff[0] = 0;
        for (uint32_t i = 0; i < n; i++) qoff[i + 1] = qoff[i] + qcnt[i];
        nF = qoff[n];
        FQ = XMALLOC(uint32_t, 4 * nF);
        for (uint32_t i = 0; i < n; i++) qcnt[i] = 0;
        for (int t = 0; t < nth; t++) {
            for (uint64_t k = 0; k < tn[t]; k++) {
                const uint32_t *v = &tb[t][4 * k];
                memcpy(&FQ[4 * (qoff[v[0]] + qcnt[v[0]]++)], v, 16);
            }
            free(tb[t]);
        }
        free(tb); free(tn); free(tcap);
    } else {
        /* as run: every alpha tetrahedron is kept, in the reference's order */
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : cand_q)
        for (uint32_t i = 0; i < n; i++) {
            uint64_t b = toff[i], e = toff[i + 1], c = 0, ca = 0;
            float o4[4];
            uint64_t g0 = b;
            while (g0 < e) {
                uint32_t v2 = T2[g0];
                uint64_t g1 = g0 + 1;
                while (g1 < e && T2[g1] == v2) g1++;
                for (uint64_t j = g0; j < g1; j++) {
                    uint32_t v3 = T3[j];
                    for (uint64_t k = j + 1; k < g1; k++) {
                        uint32_t v4 = T3[k];
                        /* (i,v3,v4) lies after k in i's sorted list, so a
                           search over the whole list is equivalent to the
                           reference's scan of (k, end) (LD:409-415) */
                        if (find2(T2, T3, b, e, v3, v4) < 0) continue;
                        if (find2(T2, T3, toff[v2], toff[v2 + 1], v3, v4) < 0)
                            continue;
                        c++;
                        ca += tet_alpha(&at[i], &at[v2], &at[v3], &at[v4], alpha, variant, o4);
                    }
                }
                g0 = g1;
            }
            cand_q += c;
            qcnt[i] = ca;
        }
        qoff[0] = 0;
        for (uint32_t i = 0; i < n; i++) qoff[i + 1] = qoff[i] + qcnt[i];
        res->cand_tets = cand_q;
        nQ = qoff[n];
        Q = XMALLOC(uint32_t, 4 * nQ);
        QO = XMALLOC(float, 4 * nQ);
#pragma omp parallel for schedule(dynamic, 64)
        for (uint32_t i = 0; i < n; i++) {
            uint64_t b = toff[i], e = toff[i + 1], o = qoff[i];
            uint64_t g0 = b;
            while (g0 < e) {
                uint32_t v2 = T2[g0];
                uint64_t g1 = g0 + 1;
                while (g1 < e && T2[g1] == v2) g1++;
                for (uint64_t j = g0; j < g1; j++) {
                    uint32_t v3 = T3[j];
                    for (uint64_t k = j + 1; k < g1; k++) {
                        uint32_t v4 = T3[k];
                        if (find2(T2, T3, b, e, v3, v4) < 0) continue;
                        if (find2(T2, T3, toff[v2], toff[v2 + 1], v3, v4) < 0) continue;
                        float o4[4];
                        if (tet_alpha(&at[i], &at[v2], &at[v3], &at[v4], alpha, variant, o4)) {
                            Q[4 * o] = i; Q[4 * o + 1] = v2;
                            Q[4 * o + 2] = v3; Q[4 * o + 3] = v4;
                            memcpy(&QO[4 * o], o4, 16);
                            o++;
                        }
                    }
                }
                g0 = g1;
            }
        }
        nF = nQ;
        FQ = XMALLOC(uint32_t, 4 * nF);
        memcpy(FQ, Q, 16 * nF);
        qkeep = XMALLOC(unsigned char, 1);
    }
    res->alpha_tets = nQ;
    res->insphere_evals = evals;
    res->sos_calls = sos;
    res->sos_exhausted = sosx;

    /* ---- faces of the final tetrahedra (LD:737-760, 1546-1583) ---- */
    uint32_t *TI = XMALLOC(uint32_t, 12 * nF);
    for (uint64_t q = 0; q < nF; q++) {
        uint32_t *v = &FQ[4 * q], *o = &TI[12 * q];
        o[0] = v[0]; o[1] = v[1]; o[2] = v[2];
        o[3] = v[0]; o[4] = v[1]; o[5] = v[3];
        o[6] = v[0]; o[7] = v[2]; o[8] = v[3];
        o[9] = v[1]; o[10] = v[2]; o[11] = v[3];
    }
    qsort(TI, 4 * nF, 12, cmp_tri);
    uint64_t nTI = 0;
    for (uint64_t k = 0; k < 4 * nF; k++)
        if (nTI == 0 || cmp_tri(&TI[3 * k], &TI[3 * (nTI - 1)]) != 0) {
            memmove(&TI[3 * nTI], &TI[3 * k], 12);
            nTI++;
        }
    res->tris_in_tets = nTI;

    /* ---- alpha triangles that are not tet faces, attachment test,
            merge (LD:762-872, 1585-1690) ---- */
    unsigned char *tkeep = XMALLOC(unsigned char, nT);
#pragma omp parallel for schedule(dynamic, 256)
    for (uint64_t k = 0; k < nT; k++) {
        uint32_t key3[3] = {T1[k], T2[k], T3[k]};
        int found = bsearch(key3, TI, nTI, 12, cmp_tri) != NULL;
        if (found) {
            tkeep[k] = 0;
            continue;
        }
        att_ctx t;
        t.at = at;
        t.v[0] = T1[k]; t.v[1] = T2[k]; t.v[2] = T3[k];
        t.nv = 3;
        t.exact = exact;
        t.px = TO[4 * k]; t.py = TO[4 * k + 1]; t.pz = TO[4 * k + 2];
        t.cur = TO[4 * k + 3];
        tkeep[k] = !window_visit(&g, t.px, t.py, t.pz, att_visit, &t, &oob);
    }
    uint64_t nTk = 0;
    for (uint64_t k = 0; k < nT; k++) nTk += tkeep[k];
    uint64_t nFT = nTk + nTI;
    uint32_t *FT = XMALLOC(uint32_t, 3 * nFT);
    {
        uint64_t o = 0;
        for (uint64_t k = 0; k < nT; k++)
            if (tkeep[k]) {
                FT[3 * o] = T1[k]; FT[3 * o + 1] = T2[k]; FT[3 * o + 2] = T3[k];
                o++;
            }
        memcpy(&FT[3 * o], TI, 12 * nTI);
        qsort(FT, nFT, 12, cmp_tri);
    }

    /* ---- edges of the final triangles, alpha edges not in them,
            attachment test, merge (LD:874-1011, 1707-1856) ---- */
    uint32_t *EI = XMALLOC(uint32_t, 6 * nFT);
    for (uint64_t k = 0; k < nFT; k++) {
        uint32_t *v = &FT[3 * k], *o = &EI[6 * k];
        o[0] = v[0]; o[1] = v[1];
        o[2] = v[0]; o[3] = v[2];
        o[4] = v[1]; o[5] = v[2];
    }
    qsort(EI, 3 * nFT, 8, cmp_edge);
    uint64_t nEI = 0;
    for (uint64_t k = 0; k < 3 * nFT; k++)
        if (nEI == 0 || cmp_edge(&EI[2 * k], &EI[2 * (nEI - 1)]) != 0) {
            memmove(&EI[2 * nEI], &EI[2 * k], 8);
            nEI++;
        }
    res->edges_in_tris = nEI;
    unsigned char *ekeep = XMALLOC(unsigned char, nE);
#pragma omp parallel for schedule(dynamic, 256)
    for (uint64_t k = 0; k < nE; k++) {
        uint32_t key2[2] = {EL[k], ER[k]};
        if (bsearch(key2, EI, nEI, 8, cmp_edge) != NULL) {
            ekeep[k] = 0;
            continue;
        }
        const oatom *a1 = &at[EL[k]], *a2 = &at[ER[k]];
        float a = a1->x - a2->x, b = a1->y - a2->y, c = a1->z - a2->z;
        float d = (a1->x * a1->x - a2->x * a2->x) + (a1->y * a1->y - a2->y * a2->y);
        d = d + (a1->z * a1->z - a2->z * a2->z);
        d = d - (a1->r * a1->r);
        d = d + (a2->r * a2->r);
        d = d / 2.0f;
        float tt = d - a * a1->x;
        tt = tt - b * a1->y;
        tt = tt - c * a1->z;
        float nn = a * a + b * b;
        nn = nn + c * c;
        tt = tt / nn;
        att_ctx t;
        t.at = at;
        t.v[0] = EL[k]; t.v[1] = ER[k];
        t.nv = 2;
        t.px = a1->x + a * tt;
        t.py = a1->y + b * tt;
        t.pz = a1->z + c * tt;
        float ex = a1->x - t.px, ey = a1->y - t.py, ez = a1->z - t.pz;
        float cur = ex * ex + ey * ey;
        cur = cur + ez * ez;
        cur = cur - (a1->r * a1->r);
        t.cur = cur;
        t.exact = exact;
        if (exact) {
            float c[3];
            x_edge_centre(a1, a2, c);
            t.px = c[0]; t.py = c[1]; t.pz = c[2];
        }
        ekeep[k] = !window_visit(&g, t.px, t.py, t.pz, att_visit, &t, &oob);
    }
    uint64_t nEk = 0;
    for (uint64_t k = 0; k < nE; k++) nEk += ekeep[k];
    uint64_t nFE = nEk + nEI;
    uint32_t *FE = XMALLOC(uint32_t, 2 * nFE);
    {
        uint64_t o = 0;
        for (uint64_t k = 0; k < nE; k++)
            if (ekeep[k]) {
                FE[2 * o] = EL[k]; FE[2 * o + 1] = ER[k];
                o++;
            }
        memcpy(&FE[2 * o], EI, 8 * nEI);
        qsort(FE, nFE, 8, cmp_edge);
    }
    res->ortho_out_of_grid = oob;

    /* ---- map to original 0-based indices (LD:2036-2050) ---- */
    res->n_edges = nFE;
    res->n_tris = nFT;
    res->n_tets = nF;
    res->edges = XMALLOC(uint32_t, 2 * nFE);
    res->tris = XMALLOC(uint32_t, 3 * nFT);
    res->tets = XMALLOC(uint32_t, 4 * nF);
    for (uint64_t k = 0; k < 2 * nFE; k++) res->edges[k] = at[FE[k]].idx - 1;
    for (uint64_t k = 0; k < 3 * nFT; k++) res->tris[k] = at[FT[k]].idx - 1;
    for (uint64_t k = 0; k < 4 * nF; k++) res->tets[k] = at[FQ[k]].idx - 1;

    free(in); free(key); free(cbeg); free(cend); free(at); free(cellof);
    free(ecnt); free(eoff); free(EL); free(ER);
    free(tcnt); free(toff); free(T1); free(T2); free(T3); free(TO);
    free(qcnt); free(qoff); free(Q); free(QO); free(qkeep); free(FQ);
    free(TI); free(tkeep); free(FT); free(EI); free(ekeep); free(FE);
    return 0;
}

void orc_free(orc_result *res) {
    free(res->edges);
    free(res->tris);
    free(res->tets);
    res->edges = res->tris = res->tets = NULL;
}

int orc_exact_pred(int kind, const float *b, float alpha) {
    switch (kind) {
    case 0: return oex_edge(b, alpha);
    case 1: return oex_tri(b, alpha);
    case 2: return oex_tet(b, alpha);
    case 3: return oex_orient(b);
    case 4: return oex_insphere(b);
    case 5: return oex_edge_attached(b);
    case 6: return oex_tri_attached(b);
    }
    return -9;
}
