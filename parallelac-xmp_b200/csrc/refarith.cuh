// refarith.cuh -- the reference's single-precision filter arithmetic.
//
// Each function performs the float operations of one reference kernel in
// the reference's statement and operand order, written as the same C
// expressions so that the compiler sees the same expression trees.  The
// translation unit that includes this header is compiled twice:
//   -fmad=false : every operation is one IEEE binary32 op (the strict,
//                 oracle-identical flavour), and
//   -fmad=true  : nvcc may contract multiply-adds exactly as it does when
//                 it compiles the reference with default flags.
// The formulas themselves have to be the reference's for the decisions to
// match bit for bit; the statement layout is kept for the same reason.
//
// Citations: LD = AlphaComplexLargeData.cu, PLAIN = AlphaComplexParallel.cu,
//            PRED = predicates.h.
#pragma once
#include <cstdint>

namespace pac {

struct Ball {
    float x, y, z, r;  // r = raw radius + solvent radius (LD:1085)
};

__device__ __forceinline__ Ball ld_ball(const float4 *p) {
    float4 v = __ldg(p);
    return Ball{v.x, v.y, v.z, v.w};
}

// formula sets; kExact selects the decision-exact predicates (exactpred.cuh)
enum : int { kUpstream = 0, kPlainXmp = 1, kExact = 2 };

// The reference compares binary32 results in double precision: THRES and
// ATHRES are the double literal 0.0 (LD:48-49), so `x <= (alpha + ATHRES)`
// (LD:185, 347, 588) and `powDist + THRES <= currentDist` (LD:829, 968)
// convert their binary32 operands to double.  That conversion is exact and
// adding +0.0 changes no value a comparison sees, so each such test has the
// outcome of the binary32 comparison x <= y, NaNs included; that is what is
// evaluated here.  (Tests whose right-hand side is a double product, in the
// plain-xmp formulas, stay in double.)
__device__ __forceinline__ bool le_as_double(float x, float y) { return x <= y; }

// markRealEdges: LD:173-189 (upstream) / PLAIN:209-229 (plain-xmp).
template <int V>
__device__ __forceinline__ bool edge_alpha(const Ball a1, const Ball a2, float alpha) {
    float a = a1.x - a2.x;
    float b = a1.y - a2.y;
    float c = a1.z - a2.z;
    float d = (a1.x * a1.x - a2.x * a2.x) + (a1.y * a1.y - a2.y * a2.y) +
              (a1.z * a1.z - a2.z * a2.z) - (a1.r * a1.r) + (a2.r * a2.r);
    d /= 2;
    float t = (d - a * a1.x - b * a1.y - c * a1.z);
    if (V == kUpstream) {
        float currentDist = ((t * t) / (a * a + b * b + c * c)) - (a1.r * a1.r);
        return le_as_double(currentDist, alpha);
    } else {
        float currentDistTerm = ((t * t)) - (a1.r * a1.r) * (a * a + b * b + c * c);
        return currentDistTerm <= ((double)alpha + 0.0) * (a * a + b * b + c * c);
    }
}

// markRealTriangles: LD:308-347 (upstream) / PLAIN:320-370 (plain-xmp).
// Returns the alpha mark and writes the orthosphere (X, Y, Z, power).
template <int V>
__device__ __forceinline__ bool tri_alpha(const Ball a1, const Ball a2, const Ball a3,
                                          float alpha, float4 &ortho) {
    float a11 = a1.x - a2.x;
    float a12 = a1.y - a2.y;
    float a13 = a1.z - a2.z;
    float b1 = (a1.x * a1.x - a2.x * a2.x) + (a1.y * a1.y - a2.y * a2.y) +
               (a1.z * a1.z - a2.z * a2.z) - (a1.r * a1.r) + (a2.r * a2.r);
    if (V == kUpstream) b1 /= 2;
    float a21 = a2.x - a3.x;
    float a22 = a2.y - a3.y;
    float a23 = a2.z - a3.z;
    float b2 = (a2.x * a2.x - a3.x * a3.x) + (a2.y * a2.y - a3.y * a3.y) +
               (a2.z * a2.z - a3.z * a3.z) - (a2.r * a2.r) + (a3.r * a3.r);
    if (V == kUpstream) b2 /= 2;
    float a31 = (a2.y - a1.y) * (a3.z - a1.z) - (a3.y - a1.y) * (a2.z - a1.z);
    float a32 = (a2.z - a1.z) * (a3.x - a1.x) - (a3.z - a1.z) * (a2.x - a1.x);
    float a33 = (a2.x - a1.x) * (a3.y - a1.y) - (a3.x - a1.x) * (a2.y - a1.y);
    float b3;
    if (V == kUpstream)
        b3 = a31 * a1.x + a32 * a1.y + a33 * a1.z;
    else
        b3 = a31 * a1.x + a32 * a1.y + a33 * a1.z * 2;
    float D = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31 -
              a12 * a21 * a33 - a11 * a23 * a32;
    float Dx = b1 * a22 * a33 + a12 * a23 * b3 + a13 * b2 * a32 - a13 * a22 * b3 -
               a12 * b2 * a33 - b1 * a23 * a32;
    float Dy = a11 * b2 * a33 + b1 * a23 * a31 + a13 * a21 * b3 - a13 * b2 * a31 -
               b1 * a21 * a33 - a11 * a23 * b3;
    float Dz = a11 * a22 * b3 + a12 * b2 * a31 + b1 * a21 * a32 - b1 * a22 * a31 -
               a12 * a21 * b3 - a11 * b2 * a32;
    if (V == kUpstream) {
        float X = Dx / D;
        float Y = Dy / D;
        float Z = Dz / D;
        float dist = (a1.x - X) * (a1.x - X) + (a1.y - Y) * (a1.y - Y) +
                     (a1.z - Z) * (a1.z - Z) - a1.r * a1.r;
        ortho = make_float4(X, Y, Z, dist);
        return le_as_double(dist, alpha);
    } else {
        D = D * 2;
        float X = Dx;
        float Y = Dy;
        float Z = Dz;
        float dist = (a1.x * D - X) * (a1.x * D - X) + (a1.y * D - Y) * (a1.y * D - Y) +
                     (a1.z * D - Z) * (a1.z * D - Z) - a1.r * a1.r * D * D;
        bool mark = dist <= ((double)alpha + 0.0) * D * D;
        X = X / D;
        Y = Y / D;
        Z = Z / D;
        dist = dist / (D * D);
        ortho = make_float4(X, Y, Z, dist);
        return mark;
    }
}

// markRealTets: LD:542-590 (the same in both binaries).
__device__ __forceinline__ bool tet_alpha(const Ball a1, const Ball a2, const Ball a3,
                                          const Ball a4, float alpha, float4 &ortho) {
    float a11 = a1.x - a2.x;
    float a12 = a1.y - a2.y;
    float a13 = a1.z - a2.z;
    float b1 = (a1.x * a1.x - a2.x * a2.x) + (a1.y * a1.y - a2.y * a2.y) +
               (a1.z * a1.z - a2.z * a2.z) - (a1.r * a1.r) + (a2.r * a2.r);
    b1 /= 2;
    float a21 = a2.x - a3.x;
    float a22 = a2.y - a3.y;
    float a23 = a2.z - a3.z;
    float b2 = (a2.x * a2.x - a3.x * a3.x) + (a2.y * a2.y - a3.y * a3.y) +
               (a2.z * a2.z - a3.z * a3.z) - (a2.r * a2.r) + (a3.r * a3.r);
    b2 /= 2;
    float a31 = a3.x - a4.x;
    float a32 = a3.y - a4.y;
    float a33 = a3.z - a4.z;
    float b3 = (a3.x * a3.x - a4.x * a4.x) + (a3.y * a3.y - a4.y * a4.y) +
               (a3.z * a3.z - a4.z * a4.z) - (a3.r * a3.r) + (a4.r * a4.r);
    b3 /= 2;
    float D = a11 * a22 * a33 + a12 * a23 * a31 + a13 * a21 * a32 - a13 * a22 * a31 -
              a12 * a21 * a33 - a11 * a23 * a32;
    float Dx = b1 * a22 * a33 + a12 * a23 * b3 + a13 * b2 * a32 - a13 * a22 * b3 -
               a12 * b2 * a33 - b1 * a23 * a32;
    float Dy = a11 * b2 * a33 + b1 * a23 * a31 + a13 * a21 * b3 - a13 * b2 * a31 -
               b1 * a21 * a33 - a11 * a23 * b3;
    float Dz = a11 * a22 * b3 + a12 * b2 * a31 + b1 * a21 * a32 - b1 * a22 * a31 -
               a12 * a21 * b3 - a11 * b2 * a32;
    if (D == 0.0) {
        ortho = make_float4(0, 0, 0, 0);
        return true;
    }
    float X = Dx / D;
    float Y = Dy / D;
    float Z = Dz / D;
    float dist = (a2.x - X) * (a2.x - X) + (a2.y - Y) * (a2.y - Y) + (a2.z - Z) * (a2.z - Z) -
                 a2.r * a2.r;
    ortho = make_float4(X, Y, Z, dist);
    return le_as_double(dist, alpha);
}

// markRealTets in two parts, for the enumeration, where the tetrahedra of
// one triangle group (a1, a2, a3) differ only in a4.  Every product of the
// reference's determinants (LD:569-576) multiplies two factors that depend
// on a1, a2, a3 only, then one that involves a4: ((f * g) * h).  TetGroup
// holds the twelve (f * g) of a group, computed once by the same operations;
// tet_alpha_g completes a tetrahedron from them with the same operations in
// the same order, so its results are those of tet_alpha bit for bit.
struct TetGroup {
    float p11_22, p12_23, p13_21, p13_22, p12_21, p11_23;  // a1i * a2j
    float pb1_22, p13_b2, p12_b2, pb1_23, p11_b2, pb1_21;  // with b1, b2
};

__device__ __forceinline__ TetGroup tet_group(const Ball a1, const Ball a2, const Ball a3) {
    float a11 = a1.x - a2.x;
    float a12 = a1.y - a2.y;
    float a13 = a1.z - a2.z;
    float b1 = (a1.x * a1.x - a2.x * a2.x) + (a1.y * a1.y - a2.y * a2.y) +
               (a1.z * a1.z - a2.z * a2.z) - (a1.r * a1.r) + (a2.r * a2.r);
    b1 /= 2;
    float a21 = a2.x - a3.x;
    float a22 = a2.y - a3.y;
    float a23 = a2.z - a3.z;
    float b2 = (a2.x * a2.x - a3.x * a3.x) + (a2.y * a2.y - a3.y * a3.y) +
               (a2.z * a2.z - a3.z * a3.z) - (a2.r * a2.r) + (a3.r * a3.r);
    b2 /= 2;
    TetGroup g;
    g.p11_22 = a11 * a22;
    g.p12_23 = a12 * a23;
    g.p13_21 = a13 * a21;
    g.p13_22 = a13 * a22;
    g.p12_21 = a12 * a21;
    g.p11_23 = a11 * a23;
    g.pb1_22 = b1 * a22;
    g.p13_b2 = a13 * b2;
    g.p12_b2 = a12 * b2;
    g.pb1_23 = b1 * a23;
    g.p11_b2 = a11 * b2;
    g.pb1_21 = b1 * a21;
    return g;
}

__device__ __forceinline__ bool tet_alpha_g(const TetGroup &g, const Ball a2, const Ball a3,
                                            const Ball a4, float alpha, float4 &ortho) {
    float a31 = a3.x - a4.x;
    float a32 = a3.y - a4.y;
    float a33 = a3.z - a4.z;
    float b3 = (a3.x * a3.x - a4.x * a4.x) + (a3.y * a3.y - a4.y * a4.y) +
               (a3.z * a3.z - a4.z * a4.z) - (a3.r * a3.r) + (a4.r * a4.r);
    b3 /= 2;
    float D = g.p11_22 * a33 + g.p12_23 * a31 + g.p13_21 * a32 - g.p13_22 * a31 -
              g.p12_21 * a33 - g.p11_23 * a32;
    float Dx = g.pb1_22 * a33 + g.p12_23 * b3 + g.p13_b2 * a32 - g.p13_22 * b3 -
               g.p12_b2 * a33 - g.pb1_23 * a32;
    float Dy = g.p11_b2 * a33 + g.pb1_23 * a31 + g.p13_21 * b3 - g.p13_b2 * a31 -
               g.pb1_21 * a33 - g.p11_23 * b3;
    float Dz = g.p11_22 * b3 + g.p12_b2 * a31 + g.pb1_21 * a32 - g.pb1_22 * a31 -
               g.p12_21 * b3 - g.p11_b2 * a32;
    if (D == 0.0) {
        ortho = make_float4(0, 0, 0, 0);
        return true;
    }
    float X = Dx / D;
    float Y = Dy / D;
    float Z = Dz / D;
    float dist = (a2.x - X) * (a2.x - X) + (a2.y - Y) * (a2.y - Y) + (a2.z - Z) * (a2.z - Z) -
                 a2.r * a2.r;
    ortho = make_float4(X, Y, Z, dist);
    return le_as_double(dist, alpha);
}

// orient3d determinant (PRED:2015-2045); the error bound there is dead.
__device__ __forceinline__ float orient3d(const float *pa, const float *pb, const float *pc,
                                          const float *pd) {
    float adx = pa[0] - pd[0];
    float bdx = pb[0] - pd[0];
    float cdx = pc[0] - pd[0];
    float ady = pa[1] - pd[1];
    float bdy = pb[1] - pd[1];
    float cdy = pc[1] - pd[1];
    float adz = pa[2] - pd[2];
    float bdz = pb[2] - pd[2];
    float cdz = pc[2] - pd[2];
    float bdxcdy = bdx * cdy;
    float cdxbdy = cdx * bdy;
    float cdxady = cdx * ady;
    float adxcdy = adx * cdy;
    float adxbdy = adx * bdy;
    float bdxady = bdx * ady;
    return adz * (bdxcdy - cdxbdy) + bdz * (cdxady - adxcdy) + cdz * (adxbdy - bdxady);
}

// insphere_w determinant (PRED:4250-4322); the error bound there is dead.
__device__ __forceinline__ float insphere_w(const float *pa, const float *pb, const float *pc,
                                            const float *pd, const float *pe, float wa,
                                            float wb, float wc, float wd, float we) {
    float aex = pa[0] - pe[0];
    float bex = pb[0] - pe[0];
    float cex = pc[0] - pe[0];
    float dex = pd[0] - pe[0];
    float aey = pa[1] - pe[1];
    float bey = pb[1] - pe[1];
    float cey = pc[1] - pe[1];
    float dey = pd[1] - pe[1];
    float aez = pa[2] - pe[2];
    float bez = pb[2] - pe[2];
    float cez = pc[2] - pe[2];
    float dez = pd[2] - pe[2];
    float aew = wa - we;
    float bew = wb - we;
    float cew = wc - we;
    float dew = wd - we;
    float aexbey = aex * bey;
    float bexaey = bex * aey;
    float ab = aexbey - bexaey;
    float bexcey = bex * cey;
    float cexbey = cex * bey;
    float bc = bexcey - cexbey;
    float cexdey = cex * dey;
    float dexcey = dex * cey;
    float cd = cexdey - dexcey;
    float dexaey = dex * aey;
    float aexdey = aex * dey;
    float da = dexaey - aexdey;
    float aexcey = aex * cey;
    float cexaey = cex * aey;
    float ac = aexcey - cexaey;
    float bexdey = bex * dey;
    float dexbey = dex * bey;
    float bd = bexdey - dexbey;
    float abc = aez * bc - bez * ac + cez * ab;
    float bcd = bez * cd - cez * bd + dez * bc;
    float cda = cez * da + dez * ac + aez * cd;
    float dab = dez * ab + aez * bd + bez * da;
    float alift = aex * aex + aey * aey + aez * aez;
    float blift = bex * bex + bey * bey + bez * bez;
    float clift = cex * cex + cey * cey + cez * cez;
    float dlift = dex * dex + dey * dey + dez * dez;
    float alw = alift - aew;
    float blw = blift - bew;
    float clw = clift - cew;
    float dlw = dlift - dew;
    return (dlw * abc - clw * dab) + (blw * cda - alw * bcd);
}

// Attachment test of checkDanglingTris / checkDanglingEdges
// (LD:825-829, 964-968): true when ball e is at least as close (in power
// distance) to (px, py, pz) as the simplex's own balls.
__device__ __forceinline__ bool attached(const Ball e, float px, float py, float pz,
                                         float currentDist) {
    float powDist = (e.x - px) * (e.x - px) + (e.y - py) * (e.y - py) +
                    (e.z - pz) * (e.z - pz) - (e.r * e.r);
    return le_as_double(powDist, currentDist);
}

// Foot of the radical plane of an edge and its power (LD:936-949).
__device__ __forceinline__ void edge_foot(const Ball a1, const Ball a2, float &px, float &py,
                                          float &pz, float &currentDist) {
    float a = a1.x - a2.x;
    float b = a1.y - a2.y;
    float c = a1.z - a2.z;
    float d = (a1.x * a1.x - a2.x * a2.x) + (a1.y * a1.y - a2.y * a2.y) +
              (a1.z * a1.z - a2.z * a2.z) - (a1.r * a1.r) + (a2.r * a2.r);
    d /= 2;
    float t = (d - a * a1.x - b * a1.y - c * a1.z) / (a * a + b * b + c * c);
    px = a1.x + a * t;
    py = a1.y + b * t;
    pz = a1.z + c * t;
    currentDist = (a1.x - px) * (a1.x - px) + (a1.y - py) * (a1.y - py) +
                  (a1.z - pz) * (a1.z - pz) - (a1.r * a1.r);
}

// Cell coordinate of a point (LD:72-74, 621-623): float subtract, IEEE
// divide, truncating conversion (NaN -> 0, saturating).
__device__ __forceinline__ int cell_coord(float p, float lo, float step) {
    return (int)((p - lo) / step);
}

}  // namespace pac
