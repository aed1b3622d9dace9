// cert_harness.cpp -- checks the certified insphere filter (certify.cuh)
// against the reference's binary32 arithmetic as the oracle restates it
// (orc_orient3d, orc_insphere_w in oracle/pac_oracle.c): whenever the filter
// claims a decision it must be the replay's.  Built and run by
// tests/test_certify.py.
//   cert_harness SEED CASES
//     -> "cases N certified C mismatches M zeros Z generic G generic_certified GC"
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "../../parallelac-xmp_b200/csrc/certify.cuh"

extern "C" float orc_orient3d(const float *pa, const float *pb, const float *pc, const float *pd);
extern "C" float orc_insphere_w(const float *pa, const float *pb, const float *pc, const float *pd,
                                const float *pe, float wa, float wb, float wc, float wd, float we);

static uint64_t g_state;
static double urand() {  // splitmix64 -> [0, 1)
    uint64_t z = (g_state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}
static double sym(double s) { return (2.0 * urand() - 1.0) * s; }

// orthocentre of four weighted points in double (Cramer's rule)
static bool ortho(const double p[4][3], const double w[4], double c[3], double *rho) {
    double A[3][3], b[3];
    for (int k = 1; k < 4; k++) {
        for (int i = 0; i < 3; i++) A[k - 1][i] = 2.0 * (p[k][i] - p[0][i]);
        double s0 = 0, s1 = 0;
        for (int i = 0; i < 3; i++) {
            s0 += p[0][i] * p[0][i];
            s1 += p[k][i] * p[k][i];
        }
        b[k - 1] = s1 - s0 - w[k] + w[0];
    }
    auto det3 = [](double M[3][3]) {
        return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
               M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
               M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    };
    const double D = det3(A);
    if (D == 0) return false;
    for (int col = 0; col < 3; col++) {
        double M[3][3];
        for (int r = 0; r < 3; r++)
            for (int i = 0; i < 3; i++) M[r][i] = i == col ? b[r] : A[r][i];
        c[col] = det3(M) / D;
    }
    double d2 = 0;
    for (int i = 0; i < 3; i++) d2 += (p[0][i] - c[i]) * (p[0][i] - c[i]);
    *rho = d2 - w[0];
    return true;
}

int main(int argc, char **argv) {
    g_state = argc > 1 ? strtoull(argv[1], nullptr, 10) : 1;
    const long cases = argc > 2 ? atol(argv[2]) : 200000;
    long certified = 0, mismatches = 0, zeros = 0, generic = 0, generic_cert = 0;
    const float wmax = 3.3f * 3.3f * 1.001f;
    for (long t = 0; t < cases; t++) {
        const int kind = (int)(t % 5);
        float P[5][3], R[5];
        // 0: generic, 1: e near the orthosphere, 2: nearly flat tetrahedron,
        // 3: 0.25 A lattice with equal radii, 4: generic with a poor centre
        for (int k = 0; k < 5; k++) {
            for (int i = 0; i < 3; i++) {
                double v = sym(3.0) + 40.0;
                if (kind == 3) v = std::round(v * 4.0) / 4.0;
                P[k][i] = (float)v;
            }
            R[k] = kind == 3 ? 3.1f : (float)(1.5 + 1.4 + urand() * 0.3);
        }
        if (kind == 2) {  // d close to the plane of a, b, c
            const double s = urand(), u = urand() * (1 - s), eps = sym(1e-4);
            for (int i = 0; i < 3; i++)
                P[3][i] = (float)(P[0][i] + s * (P[1][i] - P[0][i]) + u * (P[2][i] - P[0][i]) +
                                  (i == 2 ? eps : 0.0));
        }
        float W[5];
        for (int k = 0; k < 5; k++) W[k] = R[k] * R[k];
        double p[4][3], w[4], c[3], rho;
        for (int k = 0; k < 4; k++) {
            for (int i = 0; i < 3; i++) p[k][i] = P[k][i];
            w[k] = W[k];
        }
        if (!ortho(p, w, c, &rho)) continue;
        if (kind == 1) {  // e at power ~0 from the orthosphere
            const double th = urand() * 6.283185307179586, ph = std::acos(sym(1.0));
            const double rad = 1.0 + urand() * 6.0;
            const double e[3] = {c[0] + rad * std::sin(ph) * std::cos(th),
                                 c[1] + rad * std::sin(ph) * std::sin(th), c[2] + rad * std::cos(ph)};
            for (int i = 0; i < 3; i++) P[4][i] = (float)e[i];
            double d2 = 0;
            for (int i = 0; i < 3; i++) d2 += (P[4][i] - c[i]) * (P[4][i] - c[i]);
            const double we = d2 - rho + sym(1e-3);
            if (we <= 0) continue;
            R[4] = (float)std::sqrt(we);
            W[4] = R[4] * R[4];
        }
        float cc[3] = {(float)c[0], (float)c[1], (float)c[2]};
        if (kind == 4)
            for (int i = 0; i < 3; i++) cc[i] += (float)sym(0.05);
        if (!(std::fabs(cc[0]) < 1e6f && std::fabs(cc[1]) < 1e6f && std::fabs(cc[2]) < 1e6f))
            continue;
        const float orient = orc_orient3d(P[0], P[1], P[2], P[3]);
        const pac::cert::Insphere ct = pac::cert::setup(
            P[0][0], P[0][1], P[0][2], W[0], P[1][0], P[1][1], P[1][2], W[1], P[2][0], P[2][1],
            P[2][2], W[2], P[3][0], P[3][1], P[3][2], W[3], orient, cc[0], cc[1], cc[2], wmax);
        const int dec = pac::cert::test(ct, P[4][0], P[4][1], P[4][2], W[4]);
        const float res = orc_insphere_w(P[0], P[1], P[2], P[3], P[4], W[0], W[1], W[2], W[3], W[4]);
        if (res == 0.0f) zeros++;
        const int rdec = (orient < 0 ? (res < 0) : (res > 0)) ? 1 : 0;
        if (kind == 0) generic++;
        if (dec >= 0) {
            certified++;
            if (kind == 0) generic_cert++;
            if (dec != rdec || res == 0.0f) mismatches++;
        }
    }
    std::printf("cases %ld certified %ld mismatches %ld zeros %ld generic %ld generic_certified %ld\n",
                cases, certified, mismatches, zeros, generic, generic_cert);
    return 0;
}
