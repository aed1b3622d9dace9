// certify.cuh -- a certified sign filter for the reference's single-precision
// insphere test.
//
// The reference decides "ball e violates tetrahedron (a, b, c, d)" from the
// sign of insphere_w evaluated in binary32 (PRED:4250-4322; its exact
// fallback is dead, PRED:4357-4366), compared with the sign of orient3d in
// binary32 (PRED:2015-2045; LD:642-667):
//     viol = orient < 0 ? insphere < 0 : insphere > 0.
// Replaying those ~85 operations for every (tetrahedron, window ball) pair is
// the cost of the orthosphere scan.  This filter decides most pairs from the
// power distance of e to the tetrahedron's orthosphere (about 18 operations)
// and proves, per pair, that the replay would give the same answer;
// otherwise it says so and the caller replays.
//
// Identity.  For any point c and any constant rho, with
//     s_k = |p_k - c|^2 - w_k,  r_k = s_k - rho       (k = a, b, c, d)
//     pi(e) = |p_e - c|^2 - w_e - rho                 (power distance)
//     O = det(p_a - p_d, p_b - p_d, p_c - p_d)        (orient3d, exact)
// the lifted determinant that insphere_w evaluates satisfies exactly
//     insphere(e) = -pi(e) * O + det[p_k - p_e | r_k],
// because each lift |p_k - p_e|^2 - (w_k - w_e) equals
// 2 (p_k - p_e).(c - p_e) + r_k - pi(e), and the first term is a combination
// of the three coordinate columns.  When c is the orthocentre all r_k vanish.
// Expanding the last determinant along its r column, with every coordinate
// difference at most delta in magnitude, each 3x3 minor is at most
// (sqrt(3) delta)^3 < 5.2 delta^3 (Hadamard), so
//     |insphere(e) + pi(e) O| <= 21 r_max delta^3.
//
// Rounding of the reference's evaluation.  Counting roundings along each
// path of insphere_w's expression tree (a difference: 1; a product adds the
// two operands' counts plus 1; a sum takes the larger count plus 1) gives
// at most 17 for the final value, so (first order, u = 2^-24)
//     |fl(insphere) - insphere| <= 17 u P (1 + O(u)) <= 18 u P,
// P the same expression with every operand replaced by its magnitude.  With
// all coordinate differences <= delta and |w_k - w_e| <= W,
//     P <= 4 (3 delta^2 + W) 6 delta^3 = 24 delta^3 (3 delta^2 + W).
// FMA contraction only removes roundings, so the bound holds for both
// arithmetic flavours.  orient3d's tree gives 8 roundings: |fl(O) - O| <=
// 9 u P_O, P_O its magnitude expression.
//
// Decision.  If |fl(O)| > 9 u P_O then sign(O) = sign(fl(O)) and
// |O| >= O_lo = |fl(O)| - 9 u P_O.  If moreover
//     |pi(e)| O_lo > delta^3 (21 r_max + 432 u (3 delta^2 + W)) + eta
// (eta an absolute allowance for subnormal results), then fl(insphere) is
// nonzero with the sign of -pi(e) O, and the reference's decision is
//     viol  <=>  pi(e) < 0     (for either sign of O).
// Every quantity on the left is bounded from below and on the right from
// above, each computed in binary32 with a margin S = 1 + 2^-10 that covers
// the rounding of the bound computations themselves; sizes outside
// delta < 1000, W < 10^6 are never certified.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define PAC_CERT_FN __host__ __device__ __forceinline__
#else
#define PAC_CERT_FN inline
#endif

namespace pac {
namespace cert {

constexpr float kU = 5.9604645e-08f;          // 2^-24
constexpr float kS = 1.0f + 1.0f / 1024.0f;   // margin for the bound arithmetic
constexpr float kMaxDelta = 1000.0f;
constexpr float kMaxW = 1.0e6f;

struct Insphere {
    float cx, cy, cz;  // centre the power distances are measured from
    float rho;         // their constant (the power of the first vertex)
    float arho;        // |rho|
    float rinf;        // upper bound on max_k |p_k - c|_inf
    float k0, k2;      // threshold delta^3 (k0 + k2 delta^2) ...
    float kabs;        // ... + kabs, everything divided by O_lo
    bool ok;           // false: every ball must be replayed
};

PAC_CERT_FN float fmax3(float a, float b, float c) { return fmaxf(a, fmaxf(b, c)); }

// Setup for one tetrahedron: vertices (x, y, z) and binary32 weights as
// insphere_w takes them, the reference's binary32 orient3d value of the
// same vertex order, a centre c (any point; the orthocentre makes the
// filter sharp), and wmax >= every weight of the balls that will be tested.
PAC_CERT_FN Insphere setup(float ax, float ay, float az, float wa, float bx, float by, float bz,
                           float wb, float qx, float qy, float qz, float wc, float dx_, float dy_,
                           float dz_, float wd, float orient, float cx, float cy, float cz,
                           float wmax) {
    Insphere r;
    r.ok = false;
    r.cx = cx, r.cy = cy, r.cz = cz;
    r.rho = r.arho = r.rinf = r.k0 = r.k2 = r.kabs = 0.0f;
    // orientation: sign certain and |O| bounded from below
    const float adx = ax - dx_, bdx = bx - dx_, cdx = qx - dx_;
    const float ady = ay - dy_, bdy = by - dy_, cdy = qy - dy_;
    const float adz = az - dz_, bdz = bz - dz_, cdz = qz - dz_;
    const float po = fabsf(adz) * (fabsf(bdx * cdy) + fabsf(cdx * bdy)) +
                     fabsf(bdz) * (fabsf(cdx * ady) + fabsf(adx * cdy)) +
                     fabsf(cdz) * (fabsf(adx * bdy) + fabsf(bdx * ady));
    const float erro = 9.0f * kU * po * kS + 1e-24f;
    const float ao = fabsf(orient);
    if (!(ao > erro)) return r;
    const float olo = (ao - erro) / kS;
    // residuals of the four vertices' powers about c
    float m = 0.0f, s[4], e[4];
    const float px[4] = {ax, bx, qx, dx_}, py[4] = {ay, by, qy, dy_}, pz[4] = {az, bz, qz, dz_};
    const float pw[4] = {wa, wb, wc, wd};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float ex = px[k] - cx, ey = py[k] - cy, ez = pz[k] - cz;
        const float d2 = ex * ex + ey * ey + ez * ez;
        s[k] = d2 - pw[k];
        e[k] = 7.0f * kU * (d2 + pw[k]) * kS + 1e-30f;
        m = fmaxf(m, fmax3(fabsf(ex), fabsf(ey), fabsf(ez)));
    }
    float rmax = e[0];
#pragma unroll
    for (int k = 1; k < 4; k++) rmax = fmaxf(rmax, fabsf(s[k] - s[0]) + e[k]);
    rmax *= kS;
    r.rho = s[0];
    r.arho = fabsf(s[0]);
    r.rinf = m * kS;
    if (!(r.rinf < kMaxDelta) || !(wmax < kMaxW) || !(rmax < 1e30f)) return r;
    const float inv = kS / olo;  // >= 1 / O_lo
    r.k0 = (21.0f * rmax + 432.0f * kU * wmax) * inv * kS;
    r.k2 = 1296.0f * kU * inv * kS;
    r.kabs = 1e-24f * inv * kS + 1e-30f;
    r.ok = std::isfinite(r.k0) && std::isfinite(r.k2) && std::isfinite(r.kabs);
    return r;
}

// 1: certified violation, 0: certified no violation, -1: replay the
// reference's arithmetic for this ball.
PAC_CERT_FN int test(const Insphere &c, float ex, float ey, float ez, float we) {
    if (!c.ok) return -1;
    const float dx = ex - c.cx, dy = ey - c.cy, dz = ez - c.cz;
    const float d2 = dx * dx + dy * dy + dz * dz;
    const float pi = d2 - (we + c.rho);
    const float del = (c.rinf + fmax3(fabsf(dx), fabsf(dy), fabsf(dz))) * kS;
    if (!(del < kMaxDelta)) return -1;
    const float del2 = del * del;
    const float rhs = del * del2 * (c.k0 + c.k2 * del2) + c.kabs;
    const float epi = 8.0f * kU * kS * (d2 + we + c.arho) + 1e-30f;
    if (fabsf(pi) - epi > rhs) return pi < 0.0f ? 1 : 0;
    return -1;
}

}  // namespace cert
}  // namespace pac
