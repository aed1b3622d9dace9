// union_measure.cu -- volume and surface area of a union of balls by
// inclusion-exclusion over a fixed complex, with the gradient with respect
// to every centre and radius.
//
//   vol(U)  = sum_s (-1)^dim(s) vol(B_s),       B_s = intersection of the balls of s
//   area(U) = sum_s (-1)^dim(s) area(dB_s)
// summed over the vertices, edges, triangles and tetrahedra of the complex
// (Edelsbrunner 1995: exact when the complex is the dual complex of the
// balls, i.e. the weighted alpha complex with radii sqrt(r^2 + alpha)).
//
// Per simplex, the boundary of B_s is a set of spherical patches F_i (the
// part of sphere i inside the other balls of s), bounded by circle arcs
// ("ridges") that meet at triple points.  For every patch the kernel
// computes its area A_i (Gauss-Bonnet: R^2 (2 pi - sum_arcs phi cos(theta)
// - sum_corners exterior angle)) and its vector area M_i (half the loop
// integral of p x dp); the volume follows from the divergence theorem,
// vol = 1/3 sum_i (R_i A_i + (c_i - x0) . M_i).
//
// Gradient (the adjoint), from the first variation of volume and area:
//   d vol  / d R_i = A_i                 d vol  / d c_i = M_i
//   d area / d R_i = 2 A_i / R_i + sum_j r_ij l_ij
//   d area / d c_i = 2 M_i / R_i + sum_j r_ij N_ij
// where l_ij is the length of the ridge on circle ij, N_ij the integral of
// sphere i's unit normal along it, and r_ij = (d_ij^2 - (R_i - R_j)^2) /
// (2 d_ij rho_ij) the rate at which a ridge of two spheres at distance d_ij
// (circle radius rho_ij) changes the area per unit normal motion.  Every
// term is accumulated with the simplex's sign, so the result is the exact
// gradient of the inclusion-exclusion sum for the complex held fixed.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "pac_internal.h"

namespace pac_union {

struct V3 {
    double x, y, z;
};
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ V3 normalize(V3 a) {
    double l = sqrt(dot(a, a));
    return l > 0 ? (1.0 / l) * a : a;
}

constexpr double kPi = 3.14159265358979323846;

// circle of sphere i with sphere j, seen from i
struct Circle {
    V3 u;        // unit axis from c_i towards c_j
    double d;    // centre distance
    double t;    // signed distance of the circle's plane from c_i along u
    double rho;  // circle radius
};
__device__ __forceinline__ Circle make_circle(V3 ci, double Ri, V3 cj, double Rj) {
    Circle C;
    V3 a = cj - ci;
    C.d = sqrt(dot(a, a));
    C.u = (1.0 / C.d) * a;
    C.t = (C.d * C.d + Ri * Ri - Rj * Rj) / (2 * C.d);
    C.rho = sqrt(fmax(Ri * Ri - C.t * C.t, 0.0));
    return C;
}

// the two points common to spheres i, j, m: x +- eta * nh (relative to c_i)
struct Triple {
    V3 x, nh;
    double eta;
};
__device__ __forceinline__ Triple make_triple(V3 a, V3 b, double Ri, double Rj, double Rm) {
    // a = c_j - c_i, b = c_m - c_i; x in the plane of the centres with equal power
    V3 n = cross(a, b);
    double nn = dot(n, n);
    double a1 = 0.5 * (dot(a, a) + Ri * Ri - Rj * Rj);
    double a2 = 0.5 * (dot(b, b) + Ri * Ri - Rm * Rm);
    Triple T;
    T.x = (1.0 / nn) * (a1 * cross(b, n) + a2 * cross(n, a));
    T.nh = (1.0 / sqrt(nn)) * n;
    T.eta = sqrt(fmax(Ri * Ri - dot(T.x, T.x), 0.0));
    return T;
}

// exterior angle at corner q (relative to c_i) between the cap boundaries
// with axes ua and ub
__device__ __forceinline__ double corner(V3 q, double Ri, V3 ua, V3 ub) {
    V3 qh = (1.0 / Ri) * q;
    V3 na = normalize(ua - dot(ua, qh) * qh), nb = normalize(ub - dot(ub, qh) * qh);
    return acos(fmin(1.0, fmax(-1.0, dot(na, nb))));
}

struct Terms {
    double V;
    double A[4];
    V3 M[4];
    double rl[4];  // sum_j r_ij l_ij
    V3 rN[4];      // sum_j r_ij N_ij
};

// Patch quantities of the k balls (k = 1..4), centres relative to c[0].
__device__ void simplex_terms(int k, const V3 *c, const double *R, Terms &T) {
    for (int i = 0; i < 4; i++) {
        T.A[i] = 0;
        T.M[i] = {0, 0, 0};
        T.rl[i] = 0;
        T.rN[i] = {0, 0, 0};
    }
    if (k == 1) {
        T.V = 4.0 / 3.0 * kPi * R[0] * R[0] * R[0];
        T.A[0] = 4 * kPi * R[0] * R[0];
        return;
    }
    if (k == 2) {
        Circle C = make_circle(c[0], R[0], c[1], R[1]);
        double t1 = C.d - C.t;
        double h0 = R[0] - C.t, h1 = R[1] - t1;
        T.V = kPi * h0 * h0 * (3 * R[0] - h0) / 3 + kPi * h1 * h1 * (3 * R[1] - h1) / 3;
        T.A[0] = 2 * kPi * R[0] * h0;
        T.A[1] = 2 * kPi * R[1] * h1;
        double disk = kPi * C.rho * C.rho;
        T.M[0] = disk * C.u;
        T.M[1] = -disk * C.u;
        // full circle: l = 2 pi rho, N_i = t_i l u_i / R_i
        double g = (C.d * C.d - (R[0] - R[1]) * (R[0] - R[1])) / (2 * C.d);  // r * rho
        T.rl[0] = T.rl[1] = g * 2 * kPi;
        T.rN[0] = (g * 2 * kPi * C.t / R[0]) * C.u;
        T.rN[1] = (g * 2 * kPi * t1 / R[1]) * (-1.0 * C.u);
        return;
    }
    V3 x0 = {0, 0, 0};
    for (int i = 0; i < k; i++) x0 = x0 + c[i];
    x0 = (1.0 / k) * x0;
    double vol = 0;
    for (int i = 0; i < k; i++) {
        double gb = 0, ext = 0;
        V3 M = {0, 0, 0}, rN = {0, 0, 0};
        double rl = 0;
        for (int j = 0; j < k; j++) {
            if (j == i) continue;
            Circle C = make_circle(c[i], R[i], c[j], R[j]);
            V3 o = C.t * C.u;  // circle centre relative to c_i
            // the other one or two balls of the simplex
            int m1 = -1, m2 = -1;
            for (int m = 0; m < k; m++)
                if (m != i && m != j) {
                    if (m1 < 0)
                        m1 = m;
                    else
                        m2 = m;
                }
            // arc of this circle inside ball m1: centred on w1, half-width b1
            V3 w1 = c[m1] - c[i] - o;
            w1 = normalize(w1 - dot(w1, C.u) * C.u);
            V3 e2 = cross(C.u, w1);
            Triple P1 = make_triple(c[j] - c[i], c[m1] - c[i], R[i], R[j], R[m1]);
            double b1 = atan2(P1.eta, dot(P1.x - o, w1));
            double lo = -b1, hi = b1;
            if (m2 >= 0) {
                V3 w2 = c[m2] - c[i] - o;
                w2 = normalize(w2 - dot(w2, C.u) * C.u);
                Triple P2 = make_triple(c[j] - c[i], c[m2] - c[i], R[i], R[j], R[m2]);
                double b2 = atan2(P2.eta, dot(P2.x - o, w2));
                double dl = atan2(dot(w2, e2), dot(w2, w1));
                // overlap of [-b1, b1] with [dl - b2, dl + b2] on the circle
                double best = 0, blo = 0, bhi = 0;
                for (int s = -1; s <= 1; s++) {
                    double l2 = fmax(lo, dl - b2 + 2 * kPi * s), h2 = fmin(hi, dl + b2 + 2 * kPi * s);
                    if (h2 - l2 > best) {
                        best = h2 - l2;
                        blo = l2;
                        bhi = h2;
                    }
                }
                lo = blo;
                hi = bhi;
            }
            double phi = hi - lo;
            V3 qs = o + C.rho * (cos(lo) * w1 + sin(lo) * e2);
            V3 qe = o + C.rho * (cos(hi) * w1 + sin(hi) * e2);
            double cth = C.t / R[i];
            gb += phi * cth;
            V3 chord = qe - qs;
            M = M + 0.5 * (C.rho * C.rho * phi * C.u + C.t * cross(C.u, chord));
            double g = (C.d * C.d - (R[i] - R[j]) * (R[i] - R[j])) / (2 * C.d);  // r * rho
            rl += g * phi;
            rN = rN + (g / R[i]) * (C.t * phi * C.u - cross(C.u, chord));
            // corners at triple points (i, j, m) with j < m
            for (int m = j + 1; m < k; m++) {
                if (m == i) continue;
                Triple P = make_triple(c[j] - c[i], c[m] - c[i], R[i], R[j], R[m]);
                Circle Cm = make_circle(c[i], R[i], c[m], R[m]);
                if (k == 3) {
                    ext += corner(P.x + P.eta * P.nh, R[i], C.u, Cm.u);
                    ext += corner(P.x - P.eta * P.nh, R[i], C.u, Cm.u);
                } else {
                    // the corner is the triple point inside the fourth ball
                    int f = 6 - i - j - m;
                    V3 qp = P.x + P.eta * P.nh, qm = P.x - P.eta * P.nh;
                    V3 cf = c[f] - c[i];
                    double pp = dot(qp - cf, qp - cf), pm = dot(qm - cf, qm - cf);
                    ext += corner(pp < pm ? qp : qm, R[i], C.u, Cm.u);
                }
            }
        }
        T.A[i] = R[i] * R[i] * (2 * kPi - gb - ext);
        T.M[i] = M;
        T.rl[i] = rl;
        T.rN[i] = rN;
        vol += R[i] * T.A[i] + dot(c[i] - x0, M);
    }
    T.V = vol / 3.0;
}

// double-double accumulation (TwoSum), so the totals do not depend on the
// order in which the blocks finish: each block reduces its simplices in a
// fixed shuffle/shared-memory order and writes one (hi, lo) pair; one block
// then sums the pairs in index order.
__device__ __forceinline__ void dd_add(double &hi, double &lo, double bh, double bl) {
    double s = hi + bh;
    double v = s - hi;
    double e = (hi - (s - v)) + (bh - v);
    e += lo + bl;
    hi = s + e;
    lo = e - (hi - s);
}

// one thread per simplex; simplices of dimension dim with k = dim + 1
// vertices, indices in idx[k * s + ...]
__global__ void __launch_bounds__(128) k_union(int k, uint64_t ns, const uint32_t *idx,
                                               const double4 *balls, double4 *partial,
                                               double *dV, double *dA, int want_grad) {
    __shared__ double4 wpart[4];
    uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double vh = 0, vl = 0, ah = 0, al = 0;
    if (s < ns) {
        uint32_t id[4];
        V3 c[4];
        double R[4];
        for (int q = 0; q < k; q++) {
            id[q] = k == 1 ? (uint32_t)s : idx[(uint64_t)k * s + q];
            double4 b = balls[id[q]];
            R[q] = b.w;
            c[q] = {b.x, b.y, b.z};
        }
        V3 c0 = c[0];
        for (int q = 0; q < k; q++) c[q] = c[q] - c0;
        Terms T;
        simplex_terms(k, c, R, T);
        double sg = (k & 1) ? 1.0 : -1.0;
        vh = sg * T.V;
        for (int q = 0; q < k; q++) dd_add(ah, al, sg * T.A[q], 0.0);
        if (want_grad)
            for (int q = 0; q < k; q++) {
                double *gv = dV + 4 * (uint64_t)id[q], *ga = dA + 4 * (uint64_t)id[q];
                atomicAdd(gv + 0, sg * T.M[q].x);
                atomicAdd(gv + 1, sg * T.M[q].y);
                atomicAdd(gv + 2, sg * T.M[q].z);
                atomicAdd(gv + 3, sg * T.A[q]);
                double inv = 2.0 / R[q];
                atomicAdd(ga + 0, sg * (inv * T.M[q].x + T.rN[q].x));
                atomicAdd(ga + 1, sg * (inv * T.M[q].y + T.rN[q].y));
                atomicAdd(ga + 2, sg * (inv * T.M[q].z + T.rN[q].z));
                atomicAdd(ga + 3, sg * (inv * T.A[q] + T.rl[q]));
            }
    }
    for (int o = 16; o; o >>= 1) {
        double h1 = __shfl_xor_sync(0xffffffffu, vh, o), l1 = __shfl_xor_sync(0xffffffffu, vl, o);
        double h2 = __shfl_xor_sync(0xffffffffu, ah, o), l2 = __shfl_xor_sync(0xffffffffu, al, o);
        dd_add(vh, vl, h1, l1);
        dd_add(ah, al, h2, l2);
    }
    if ((threadIdx.x & 31) == 0) wpart[threadIdx.x >> 5] = make_double4(vh, vl, ah, al);
    __syncthreads();
    if (threadIdx.x == 0) {
        double4 r = wpart[0];
        for (int w = 1; w < 4; w++) {
            dd_add(r.x, r.y, wpart[w].x, wpart[w].y);
            dd_add(r.z, r.w, wpart[w].z, wpart[w].w);
        }
        partial[blockIdx.x] = r;
    }
}

__global__ void k_union_total(const double4 *partial, uint64_t np, double *out) {
    __shared__ double4 sp[256];
    double vh = 0, vl = 0, ah = 0, al = 0;
    for (uint64_t i = threadIdx.x; i < np; i += 256) {
        double4 r = partial[i];
        dd_add(vh, vl, r.x, r.y);
        dd_add(ah, al, r.z, r.w);
    }
    sp[threadIdx.x] = make_double4(vh, vl, ah, al);
    __syncthreads();
    if (threadIdx.x == 0) {
        double4 r = sp[0];
        for (int t = 1; t < 256; t++) {
            dd_add(r.x, r.y, sp[t].x, sp[t].y);
            dd_add(r.z, r.w, sp[t].z, sp[t].w);
        }
        out[0] = r.x + r.y;
        out[1] = r.z + r.w;
    }
}

}  // namespace pac_union

namespace pac {

// Runs the measure on device-resident balls and lists.  Gradients go to the
// device buffers d_dV / d_dA (n x 4 each) when given; vol/area to the host.
int union_measure_device(Ctx &ctx, const double4 *d_balls, uint32_t n, const uint32_t *d_edges,
                         uint64_t ne, const uint32_t *d_tris, uint64_t nt, const uint32_t *d_tets,
                         uint64_t nq, double *vol, double *area, double *d_dV, double *d_dA,
                         float *ms) {
    cudaStream_t s = ctx.stream;
    double *acc = ctx.arena.alloc_n<double>(2);
    bool grad = d_dV || d_dA;
    double *dV = d_dV, *dA = d_dA;
    if (grad && !dV) dV = ctx.arena.alloc_n<double>(4 * (size_t)n);
    if (grad && !dA) dA = ctx.arena.alloc_n<double>(4 * (size_t)n);
    const uint32_t *lists[4] = {nullptr, d_edges, d_tris, d_tets};
    uint64_t counts[4] = {n, ne, nt, nq};
    uint64_t nblocks = 0;
    for (int k = 0; k < 4; k++) nblocks += (counts[k] + 127) / 128;
    double4 *partial = ctx.arena.alloc_n<double4>(nblocks);
    if (!acc || !partial || (grad && (!dV || !dA))) return PAC_ERR_OOM;
    // two timing events, destroyed on every return path
    struct Events {
        cudaEvent_t e[2] = {nullptr, nullptr};
        Events() {
            cudaEventCreate(&e[0]);
            cudaEventCreate(&e[1]);
        }
        ~Events() {
            for (cudaEvent_t x : e)
                if (x) cudaEventDestroy(x);
        }
    } ev;
    cudaEvent_t e0 = ev.e[0], e1 = ev.e[1];
    cudaEventRecord(e0, s);
    if (grad) {
        cudaMemsetAsync(dV, 0, 4 * sizeof(double) * n, s);
        cudaMemsetAsync(dA, 0, 4 * sizeof(double) * n, s);
    }
    uint64_t off = 0;
    for (int k = 1; k <= 4; k++) {
        if (!counts[k - 1]) continue;
        unsigned blocks = (unsigned)((counts[k - 1] + 127) / 128);
        pac_union::k_union<<<blocks, 128, 0, s>>>(k, counts[k - 1], lists[k - 1], d_balls,
                                                  partial + off, dV, dA, grad ? 1 : 0);
        ctx.launches++;
        off += blocks;
    }
    pac_union::k_union_total<<<1, 256, 0, s>>>(partial, off, acc);
    ctx.launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        cudaStreamSynchronize(s);  // the launches that did start finish first
        return set_error(PAC_ERR_CUDA, std::string("union measure launch: ") + cudaGetErrorString(e));
    }
    cudaEventRecord(e1, s);
    double h[2];
    cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return set_error(PAC_ERR_CUDA, std::string("union measure: ") + cudaGetErrorString(e));
    if (ms) cudaEventElapsedTime(ms, e0, e1);
    if (vol) *vol = h[0];
    if (area) *area = h[1];
    return PAC_OK;
}

}  // namespace pac

// ---------------------------------------------------------------------------
// pac_union_measure_noalloc: the same measure for callers that cannot
// allocate device memory.
//
// Some callers cannot call cudaMalloc: a process whose device memory is
// reserved up front by another allocator (a framework's caching pool that
// owns nearly all of the GPU), or a latency-bound loop that cannot afford
// cudaMalloc's implicit device synchronisation.  This entry point allocates
// nothing: the caller passes the balls, the complex and the gradient buffers
// in device memory, and the only scratch -- one partial (volume, area) sum
// per block of 128 simplices and the two totals -- lives in the file-scope
// array below, which every GPU that loads this library holds until the
// process exits (2 MiB).
//
// Limit: the four simplex lists together may need at most kNoAllocBlocks
// blocks of 128, i.e. sum over vertices, edges, triangles and tetrahedra of
// ceil(count / 128) <= 65,536 (about 8.4 million simplices); larger
// complexes are rejected with PAC_ERR_CAPACITY before anything runs.
// ---------------------------------------------------------------------------
namespace {

constexpr uint64_t kNoAllocBlocks = 65536;
constexpr int kMaxDevices = 64;

// partial sums (one double4 per block), then one slot for the two totals
static __device__ __align__(256) double4 g_noalloc_scratch[kNoAllocBlocks + 1];

std::mutex g_noalloc_mutex;
double4 *g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on `device` (which must be current).
// The first call on each device looks it up with cudaGetSymbolAddress; in
// host code the array's name only stands in for the symbol.
int noalloc_scratch(int device, double4 **out) {
    if (device < 0 || device >= kMaxDevices)
        return pac::set_error(PAC_ERR_INVALID_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess)
            return pac::set_error(PAC_ERR_CUDA, std::string("cudaGetSymbolAddress: ") +
                                                    cudaGetErrorString(e));
        g_noalloc_ptr[device] = static_cast<double4 *>(ptr);
    }
    *out = g_noalloc_ptr[device];
    return PAC_OK;
}

}  // namespace

extern "C" int pac_union_measure_noalloc(pac_ctx *ctx, const double *d_xyzr, uint32_t n,
                                         const pac_complex *cx, double *vol, double *area,
                                         double *d_dvol, double *d_darea) {
    if (!ctx || !cx || (n && !d_xyzr))
        return pac::set_error(PAC_ERR_INVALID_ARG, "null argument");
    if ((d_dvol == nullptr) != (d_darea == nullptr))
        return pac::set_error(PAC_ERR_INVALID_ARG,
                              "pass both gradient buffers or neither (nothing is allocated)");
    // The kernels read the lists in place: they must be device lists of this
    // many balls (host lists would be dereferenced as device addresses).
    if (cx->on_device != 1)
        return pac::set_error(PAC_ERR_INVALID_ARG,
                              "pac_union_measure_noalloc needs device lists (on_device = 1)");
    if (cx->n_vertices && cx->n_vertices != n)
        return pac::set_error(PAC_ERR_INVALID_ARG, "complex and balls differ in size");
    if ((cx->n_edges && !cx->edges) || (cx->n_tris && !cx->tris) || (cx->n_tets && !cx->tets))
        return pac::set_error(PAC_ERR_INVALID_ARG, "a non-empty list has a null pointer");
    const uint32_t *lists[4] = {nullptr, cx->edges, cx->tris, cx->tets};
    const uint64_t counts[4] = {n, cx->n_edges, cx->n_tris, cx->n_tets};
    uint64_t blocks = 0;
    for (int k = 0; k < 4; k++) blocks += (counts[k] + 127) / 128;
    if (blocks > kNoAllocBlocks)
        return pac::set_error(PAC_ERR_CAPACITY,
                              "complex too large for pac_union_measure_noalloc: needs " +
                                  std::to_string(blocks) + " blocks of 128 simplices, the fixed "
                                  "scratch holds " + std::to_string(kNoAllocBlocks));
    pac::Ctx &c = pac_ctx_internal(ctx);
    cudaError_t e = cudaSetDevice(c.device);
    if (e != cudaSuccess)
        return pac::set_error(PAC_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    double4 *scratch = nullptr;
    int rc = noalloc_scratch(c.device, &scratch);
    if (rc) return rc;
    cudaStream_t s = c.stream;
    const bool grad = d_dvol != nullptr;
    if (grad) {
        // the gradients accumulate: they must start at zero
        cudaMemsetAsync(d_dvol, 0, 4 * sizeof(double) * n, s);
        cudaMemsetAsync(d_darea, 0, 4 * sizeof(double) * n, s);
    }
    uint64_t off = 0;
    for (int k = 1; k <= 4; k++) {
        if (!counts[k - 1]) continue;
        unsigned nb = (unsigned)((counts[k - 1] + 127) / 128);
        pac_union::k_union<<<nb, 128, 0, s>>>(k, counts[k - 1], lists[k - 1],
                                              reinterpret_cast<const double4 *>(d_xyzr),
                                              scratch + off, d_dvol, d_darea, grad ? 1 : 0);
        off += nb;
    }
    // every partial slot used is written above; the totals slot is written here
    double *totals = reinterpret_cast<double *>(scratch + kNoAllocBlocks);
    pac_union::k_union_total<<<1, 256, 0, s>>>(scratch, off, totals);
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return pac::set_error(PAC_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    double h[2] = {0, 0};
    e = cudaMemcpyAsync(h, totals, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return pac::set_error(PAC_ERR_CUDA, std::string("union measure: ") + cudaGetErrorString(e));
    if (vol) *vol = h[0];
    if (area) *area = h[1];
    return PAC_OK;
}
