// union_oracle.cpp -- FP64 CPU oracle of the union-of-balls volume and area
// over a fixed complex (inclusion-exclusion), with gradients by forward-mode
// automatic differentiation.
//
// TEST INFRASTRUCTURE ONLY (the checker of the engine's union measure).
//
// The value of each simplex term is computed from the patch decomposition of
// the intersection of its balls (spherical patches bounded by circle arcs:
// Gauss-Bonnet for the area, the divergence theorem for the volume).  The
// gradient is NOT taken from the closed-form first-variation identities the
// engine uses: every quantity is a dual number carrying the derivatives with
// respect to the 16 inputs (x, y, z, R of up to four balls), propagated
// through every operation, so the two gradients are computed independently.
#include <cmath>
#include <cstdint>
#include <cstring>

namespace {

constexpr int NG = 16;

struct D {
    double v;
    double g[NG];
    D() : v(0) { std::memset(g, 0, sizeof(g)); }
    D(double x) : v(x) { std::memset(g, 0, sizeof(g)); }
};
inline D operator+(const D &a, const D &b) {
    D r(a.v + b.v);
    for (int i = 0; i < NG; i++) r.g[i] = a.g[i] + b.g[i];
    return r;
}
inline D operator-(const D &a, const D &b) {
    D r(a.v - b.v);
    for (int i = 0; i < NG; i++) r.g[i] = a.g[i] - b.g[i];
    return r;
}
inline D operator-(const D &a) {
    D r(-a.v);
    for (int i = 0; i < NG; i++) r.g[i] = -a.g[i];
    return r;
}
inline D operator*(const D &a, const D &b) {
    D r(a.v * b.v);
    for (int i = 0; i < NG; i++) r.g[i] = a.g[i] * b.v + a.v * b.g[i];
    return r;
}
inline D operator/(const D &a, const D &b) {
    D r(a.v / b.v);
    for (int i = 0; i < NG; i++) r.g[i] = (a.g[i] * b.v - a.v * b.g[i]) / (b.v * b.v);
    return r;
}
inline D chain(const D &a, double f, double df) {
    D r(f);
    for (int i = 0; i < NG; i++) r.g[i] = df * a.g[i];
    return r;
}
inline D dsqrt(const D &a) {
    double s = std::sqrt(a.v > 0 ? a.v : 0.0);
    return chain(a, s, s > 0 ? 0.5 / s : 0.0);
}
inline D dcos(const D &a) { return chain(a, std::cos(a.v), -std::sin(a.v)); }
inline D dsin(const D &a) { return chain(a, std::sin(a.v), std::cos(a.v)); }
inline D dacos(const D &a) {
    double x = a.v > 1 ? 1 : (a.v < -1 ? -1 : a.v);
    double den = std::sqrt(1 - x * x);
    return chain(a, std::acos(x), den > 0 ? -1.0 / den : 0.0);
}
inline D datan2(const D &y, const D &x) {
    D r(std::atan2(y.v, x.v));
    double q = x.v * x.v + y.v * y.v;
    for (int i = 0; i < NG; i++) r.g[i] = (x.v * y.g[i] - y.v * x.g[i]) / q;
    return r;
}

struct V {
    D x, y, z;
};
inline V operator+(const V &a, const V &b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V operator-(const V &a, const V &b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V operator*(const D &s, const V &a) { return {s * a.x, s * a.y, s * a.z}; }
inline D dot(const V &a, const V &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V cross(const V &a, const V &b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V unit(const V &a) { return D(1.0) / dsqrt(dot(a, a)) * a; }

const double PI = 3.14159265358979323846;

// volume and boundary area of the intersection of k balls
void inter(int k, const V *c, const D *R, D &vol, D &area) {
    if (k == 1) {
        vol = D(4.0 / 3.0 * PI) * R[0] * R[0] * R[0];
        area = D(4 * PI) * R[0] * R[0];
        return;
    }
    if (k == 2) {
        V a = c[1] - c[0];
        D d = dsqrt(dot(a, a));
        D t0 = (d * d + R[0] * R[0] - R[1] * R[1]) / (D(2.0) * d);
        D t1 = d - t0;
        D h0 = R[0] - t0, h1 = R[1] - t1;
        vol = D(PI / 3) * (h0 * h0 * (D(3.0) * R[0] - h0) + h1 * h1 * (D(3.0) * R[1] - h1));
        area = D(2 * PI) * (R[0] * h0 + R[1] * h1);
        return;
    }
    V x0 = {D(0.0), D(0.0), D(0.0)};
    for (int i = 0; i < k; i++) x0 = x0 + c[i];
    x0 = D(1.0 / k) * x0;
    vol = D(0.0);
    area = D(0.0);
    for (int i = 0; i < k; i++) {
        D gb(0.0), ext(0.0);
        V M = {D(0.0), D(0.0), D(0.0)};
        for (int j = 0; j < k; j++) {
            if (j == i) continue;
            V a = c[j] - c[i];
            D d = dsqrt(dot(a, a));
            V u = D(1.0) / d * a;
            D t = (d * d + R[i] * R[i] - R[j] * R[j]) / (D(2.0) * d);
            D rho = dsqrt(R[i] * R[i] - t * t);
            V o = t * u;
            int m1 = -1, m2 = -1;
            for (int m = 0; m < k; m++)
                if (m != i && m != j) (m1 < 0 ? m1 : m2) = m;
            // triple point data for (i, j, m): x +- eta nh, relative to c_i
            auto triple = [&](int m, V &x, V &nh, D &eta) {
                V b = c[m] - c[i];
                V n = cross(a, b);
                D nn = dot(n, n);
                D a1 = D(0.5) * (dot(a, a) + R[i] * R[i] - R[j] * R[j]);
                D a2 = D(0.5) * (dot(b, b) + R[i] * R[i] - R[m] * R[m]);
                x = D(1.0) / nn * (a1 * cross(b, n) + a2 * cross(n, a));
                nh = D(1.0) / dsqrt(nn) * n;
                eta = dsqrt(R[i] * R[i] - dot(x, x));
            };
            V w1 = c[m1] - c[i] - o;
            w1 = unit(w1 - dot(w1, u) * u);
            V e2 = cross(u, w1);
            V X1, N1;
            D eta1;
            triple(m1, X1, N1, eta1);
            D b1 = datan2(eta1, dot(X1 - o, w1));
            D lo = -b1, hi = b1;
            if (m2 >= 0) {
                V w2 = c[m2] - c[i] - o;
                w2 = unit(w2 - dot(w2, u) * u);
                V X2, N2;
                D eta2;
                triple(m2, X2, N2, eta2);
                D b2 = datan2(eta2, dot(X2 - o, w2));
                D dl = datan2(dot(w2, e2), dot(w2, w1));
                double best = 0;
                D blo(0.0), bhi(0.0);
                for (int s = -1; s <= 1; s++) {
                    D l2 = (lo.v > (dl - b2).v + 2 * PI * s) ? lo : dl - b2 + D(2 * PI * s);
                    D h2 = (hi.v < (dl + b2).v + 2 * PI * s) ? hi : dl + b2 + D(2 * PI * s);
                    if ((h2 - l2).v > best) {
                        best = (h2 - l2).v;
                        blo = l2;
                        bhi = h2;
                    }
                }
                lo = blo;
                hi = bhi;
            }
            D phi = hi - lo;
            V qs = o + rho * (dcos(lo) * w1 + dsin(lo) * e2);
            V qe = o + rho * (dcos(hi) * w1 + dsin(hi) * e2);
            gb = gb + phi * t / R[i];
            M = M + D(0.5) * (rho * rho * phi * u + t * cross(u, qe - qs));
            for (int m = j + 1; m < k; m++) {
                if (m == i) continue;
                V Xm, Nm;
                D etam;
                // triple of (i, j, m) with this j as the pair's first member
                {
                    V b = c[m] - c[i];
                    V n = cross(a, b);
                    D nn = dot(n, n);
                    D a1 = D(0.5) * (dot(a, a) + R[i] * R[i] - R[j] * R[j]);
                    D a2 = D(0.5) * (dot(b, b) + R[i] * R[i] - R[m] * R[m]);
                    Xm = D(1.0) / nn * (a1 * cross(b, n) + a2 * cross(n, a));
                    Nm = D(1.0) / dsqrt(nn) * n;
                    etam = dsqrt(R[i] * R[i] - dot(Xm, Xm));
                }
                V bm = c[m] - c[i];
                V um = D(1.0) / dsqrt(dot(bm, bm)) * bm;
                auto corner = [&](const V &q) {
                    V qh = D(1.0) / R[i] * q;
                    V na = unit(u - dot(u, qh) * qh), nb = unit(um - dot(um, qh) * qh);
                    return dacos(dot(na, nb));
                };
                V qp = Xm + etam * Nm, qm = Xm - etam * Nm;
                if (k == 3) {
                    ext = ext + corner(qp) + corner(qm);
                } else {
                    int f = 6 - i - j - m;
                    V cf = c[f] - c[i];
                    double pp = dot(qp - cf, qp - cf).v, pm = dot(qm - cf, qm - cf).v;
                    ext = ext + corner(pp < pm ? qp : qm);
                }
            }
        }
        D A = R[i] * R[i] * (D(2 * PI) - gb - ext);
        area = area + A;
        vol = vol + R[i] * A + dot(c[i] - x0, M);
    }
    vol = vol / D(3.0);
}

}  // namespace

extern "C" int orc_union_measure(const double *xyzr, uint32_t n, const uint32_t *edges,
                                 uint64_t ne, const uint32_t *tris, uint64_t nt,
                                 const uint32_t *tets, uint64_t nq, double *vol, double *area,
                                 double *dvol, double *darea) {
    double tv = 0, ta = 0;
    if (dvol) std::memset(dvol, 0, sizeof(double) * 4 * n);
    if (darea) std::memset(darea, 0, sizeof(double) * 4 * n);
    const uint32_t *lists[4] = {nullptr, edges, tris, tets};
    uint64_t counts[4] = {n, ne, nt, nq};
    for (int k = 1; k <= 4; k++) {
        for (uint64_t s = 0; s < counts[k - 1]; s++) {
            uint32_t id[4];
            V c[4];
            D R[4];
            for (int q = 0; q < k; q++) {
                id[q] = k == 1 ? (uint32_t)s : lists[k - 1][(uint64_t)k * s + q];
                const double *b = xyzr + 4 * (uint64_t)id[q];
                // relative to the first ball's centre; the shift is a constant
                c[q].x = D(b[0] - xyzr[4 * (uint64_t)id[0]]);
                c[q].y = D(b[1] - xyzr[4 * (uint64_t)id[0] + 1]);
                c[q].z = D(b[2] - xyzr[4 * (uint64_t)id[0] + 2]);
                R[q] = D(b[3]);
            }
            // seed: derivative of every input; the first centre enters through
            // the differences
            for (int q = 0; q < k; q++) {
                c[q].x.g[4 * q + 0] += 1;
                c[q].y.g[4 * q + 1] += 1;
                c[q].z.g[4 * q + 2] += 1;
                c[q].x.g[0] -= 1;
                c[q].y.g[1] -= 1;
                c[q].z.g[2] -= 1;
                R[q].g[4 * q + 3] = 1;
            }
            D v, a;
            inter(k, c, R, v, a);
            double sg = (k & 1) ? 1.0 : -1.0;
            tv += sg * v.v;
            ta += sg * a.v;
            for (int q = 0; q < k; q++)
                for (int p = 0; p < 4; p++) {
                    if (dvol) dvol[4 * (uint64_t)id[q] + p] += sg * v.g[4 * q + p];
                    if (darea) darea[4 * (uint64_t)id[q] + p] += sg * a.g[4 * q + p];
                }
        }
    }
    if (vol) *vol = tv;
    if (area) *area = ta;
    return 0;
}
