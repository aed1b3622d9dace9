// pipeline.cu -- the single device pass: balls in, weighted alpha complex out.
//
// Compiled twice: with -DPAC_NS=pac_strict -fmad=false (IEEE op-by-op, the
// oracle-identical flavour) and with -DPAC_NS=pac_fma -fmad=true (nvcc's
// default contraction, the flavour that follows the reference binary built
// with default flags).  Nothing else differs between the two.
//
// Layout in HBM (n balls, molecules back to back):
//   at[n]        float4 (x, y, z, r + sol) in (molecule, cell, input index)
//                order -- the reference's stable sort by cell key
//                (AlphaComplexLargeData.cu:1174-1177)
//   orig[n]      molecule-local 0-based input index of each sorted ball
//   cellbeg[]    CSR cell ranges over the sorted balls (all molecules)
//   eoff[n+1], ER[]   alpha edges (i, ER[k]) with i < ER[k], CSR by i,
//                each row ascending (= the reference's sorted edge list)
//   loff[n+1], link[] per ball i, a deg(i) x deg(i) bit matrix over the
//                row of i in ER: bit (a, b) set <=> (i, ER[a], ER[b]) is an
//                alpha triangle.  faces[] has the same shape and marks final
//                triangles.
// Candidate tetrahedra are never stored: one kernel enumerates them from
// the link matrices, applies the alpha filter and the empty-orthosphere
// test, and writes only the survivors.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "certify.cuh"
#include "exactpred.cuh"
#include "pac_internal.h"
#include "refarith.cuh"
#include "sos.cuh"

#ifndef PAC_NS
#error "PAC_NS must name the arithmetic flavour namespace"
#endif

namespace PAC_NS {

using pac::Ball;

constexpr int kMaxDeg = 256;  // upper neighbours per ball supported
constexpr int kMaxW = kMaxDeg / 64;
constexpr unsigned kFull = 0xffffffffu;

// device-side counters (one slot each)
enum Counter {
    C_CAND_E, C_ALPHA_E, C_CAND_T, C_ALPHA_T, C_CAND_Q, C_ALPHA_Q, C_INSPHERE, C_SOS,
    C_OOB, C_SURV, C_PEND, C_MAXDEG, C_SOS_RANGE, C_BADDEG, C_NEXT, C_FILTER, C_FALLBACK,
    C_KILLED, C_KTESTS, C_CERT, C_CERT_BAD,
    C_NCOUNTERS
};

struct MolGrid {
    float minx, miny, minz, step;
    int gx, gy, gz;
    float wmax;  // upper bound on every ball's binary32 weight (r + sol)^2
    uint64_t cell_base;  // first global cell of this molecule
    uint64_t ncell;
    uint64_t atom_base;  // first ball (sorted and input) of this molecule
};

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return pac::set_error(PAC_ERR_CUDA, std::string(#call) + ": " +               \
                                                    cudaGetErrorString(e_));              \
    } while (0)

#define LAUNCH_CHECK(ctx)                                                                 \
    do {                                                                                  \
        (ctx).launches++;                                                                 \
        cudaError_t e_ = cudaGetLastError();                                              \
        if (e_ != cudaSuccess)                                                            \
            return pac::set_error(PAC_ERR_CUDA, std::string("launch: ") +                 \
                                                    cudaGetErrorString(e_));              \
    } while (0)

// ------------------------------------------------------------------ utils
__device__ __forceinline__ int fkey(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float funkey(int k) {
    return __int_as_float(k >= 0 ? k : k ^ 0x7fffffff);
}
__device__ __forceinline__ uint32_t mol_of(const uint32_t *mol, uint64_t i) {
    return mol ? mol[i] : 0u;
}
// 32-bit wrapping linear cell index, as the reference's int arithmetic
// behaves on the GPU (AlphaComplexLargeData.cu:625-626).
__device__ __forceinline__ int lin3(int X, int Y, int Z, int gx, int gy) {
    return (int)((unsigned)Z * (unsigned)gx * (unsigned)gy + (unsigned)Y * (unsigned)gx +
                 (unsigned)X);
}
// lower_bound of v in sorted a[0..n)
__device__ __forceinline__ int lbound(const uint32_t *a, int n, uint32_t v) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int m = (lo + hi) >> 1;
        if (__ldg(&a[m]) < v)
            lo = m + 1;
        else
            hi = m;
    }
    return lo;
}
// position of the k-th set bit (0-based) of a W-word mask, or -1
__device__ __forceinline__ int select_bit(const uint64_t *m, int W, int k) {
    for (int w = 0; w < W; w++) {
        int c = __popcll(m[w]);
        if (k < c) {
            uint32_t lo = (uint32_t)m[w], hi = (uint32_t)(m[w] >> 32);
            int cl = __popc(lo);
            if (k < cl) return w * 64 + __fns(lo, 0, k + 1);
            return w * 64 + 32 + __fns(hi, 0, k - cl + 1);
        }
        k -= c;
    }
    return -1;
}
// position of the k-th set bit (0-based) of x, k < popcount(x): halve the
// word by popcounts
__device__ __forceinline__ int select64(uint64_t x, int k) {
    uint32_t v = (uint32_t)x;
    int pos = 0;
    const int pl = __popc(v);
    if (k >= pl) {
        k -= pl;
        v = (uint32_t)(x >> 32);
        pos = 32;
    }
    int q = __popc(v & 0xffffu);
    if (k >= q) k -= q, v >>= 16, pos += 16;
    q = __popc(v & 0xffu);
    if (k >= q) k -= q, v >>= 8, pos += 8;
    q = __popc(v & 0xfu);
    if (k >= q) k -= q, v >>= 4, pos += 4;
    q = __popc(v & 0x3u);
    if (k >= q) k -= q, v >>= 2, pos += 2;
    return pos + (k >= (int)(v & 1u) ? 1 : 0);
}
// the same over a KW-word mask, k < its popcount
template <int KW>
__device__ __forceinline__ int select_kw(const uint64_t *m, int k) {
    int w = 0;
    uint64_t x = m[0];
#pragma unroll
    for (int v = 0; v + 1 < KW; v++) {
        const int q = __popcll(x);
        if (k < q) break;
        k -= q;
        w = v + 1;
        x = m[v + 1];
    }
    return w * 64 + select64(x, k);
}
// bits of word w whose global position is greater than b
__device__ __forceinline__ uint64_t above_mask(int b, int w) {
    if (w * 64 + 63 <= b) return 0ull;
    if (w * 64 > b) return ~0ull;
    int j = b & 63;
    return j == 63 ? 0ull : (~0ull << (j + 1));
}
__device__ __forceinline__ void bump(unsigned long long *ctr, int which, unsigned long long v) {
    if (v) atomicAdd(&ctr[which], v);
}
__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// ------------------------------------------------------------------ decisions
// Each test of the pipeline in one of two arithmetics: the reference's
// single-precision formulas (V = kUpstream, kPlainXmp; refarith.cuh) or the
// decision-exact cascade (V = kExact; exactpred.cuh).  In the exact mode the
// "weight" slots of the insphere/orientation helpers carry radii, squared
// exactly inside the predicates.
using pac::ex::Tally;

template <int V>
__device__ __forceinline__ float wt(float r) {
    if constexpr (V == pac::kExact) return r;
    else return r * r;
}

template <int V>
__device__ __forceinline__ bool dec_edge(const Ball a, const Ball b, float alpha, Tally &t) {
    if constexpr (V == pac::kExact) return pac::ex::edge_alpha(a, b, alpha, t);
    else return pac::edge_alpha<V>(a, b, alpha);
}

// alpha mark of a triangle; the orthosphere (centre, power) goes to o
template <int V>
__device__ __forceinline__ bool dec_tri(const Ball a, const Ball b, const Ball c, float alpha,
                                        float4 &o, Tally &t) {
    if constexpr (V == pac::kExact) {
        o = make_float4(0.f, 0.f, 0.f, 0.f);
        return pac::ex::tri_alpha(a, b, c, alpha, t);
    } else {
        return pac::tri_alpha<V>(a, b, c, alpha, o);
    }
}

// window centre (and the reference's power) of an alpha triangle
template <int V>
__device__ __forceinline__ float4 tri_sphere(const Ball a, const Ball b, const Ball c, float alpha) {
    if constexpr (V == pac::kExact) {
        const float3 q = pac::ex::tri_centre(a, b, c);
        return make_float4(q.x, q.y, q.z, 0.f);
    } else {
        float4 o;
        pac::tri_alpha<V>(a, b, c, alpha, o);
        return o;
    }
}

// alpha mark of a tetrahedron; its orthosphere centre goes to o (zeros when
// the tetrahedron is flat, as in the reference)
template <int V>
__device__ __forceinline__ bool dec_tet(const Ball a, const Ball b, const Ball c, const Ball d,
                                        float alpha, float4 &o, Tally &t) {
    if constexpr (V == pac::kExact) {
        bool flat = false;
        const bool m = pac::ex::tet_alpha(a, b, c, d, alpha, flat, t);
        o = make_float4(0.f, 0.f, 0.f, 0.f);
        if (m && !flat) {
            const float3 q = pac::ex::tet_centre(a, b, c, d);
            o = make_float4(q.x, q.y, q.z, 0.f);
        }
        return m;
    } else {
        return pac::tet_alpha(a, b, c, d, alpha, o);
    }
}

template <int V>
__device__ __forceinline__ float dec_orient(const float *pa, const float *pb, const float *pc,
                                            const float *pd, float wa, float wb, float wc, float wd,
                                            Tally &t) {
    if constexpr (V == pac::kExact)
        return (float)pac::ex::orient_sign(Ball{pa[0], pa[1], pa[2], wa}, Ball{pb[0], pb[1], pb[2], wb},
                                           Ball{pc[0], pc[1], pc[2], wc}, Ball{pd[0], pd[1], pd[2], wd}, t);
    else
        return pac::orient3d(pa, pb, pc, pd);
}

template <int V>
__device__ __forceinline__ float dec_insphere(const float *pa, const float *pb, const float *pc,
                                              const float *pd, const float *pe, float wa, float wb,
                                              float wc, float wd, float we, Tally &t) {
    if constexpr (V == pac::kExact)
        return (float)pac::ex::insphere_sign(
            Ball{pa[0], pa[1], pa[2], wa}, Ball{pb[0], pb[1], pb[2], wb}, Ball{pc[0], pc[1], pc[2], wc},
            Ball{pd[0], pd[1], pd[2], wd}, Ball{pe[0], pe[1], pe[2], we}, t);
    else
        return pac::insphere_w(pa, pb, pc, pd, pe, wa, wb, wc, wd, we);
}

// Attachment of the triangle (a0, v1, v2) by ball q; (px, py, pz, cur) is
// the reference's orthosphere of the triangle (unused in the exact mode).
template <int V>
__device__ __forceinline__ bool dec_tri_attached(const Ball a0, const float4 *at, uint32_t v1,
                                                 uint32_t v2, const Ball q, float px, float py,
                                                 float pz, float cur, Tally &t) {
    if constexpr (V == pac::kExact)
        return pac::ex::tri_attached(a0, pac::ld_ball(&at[v1]), pac::ld_ball(&at[v2]), q, t);
    else
        return pac::attached(q, px, py, pz, cur);
}

// Window centre of an alpha edge and the reference's power there.
template <int V>
__device__ __forceinline__ void edge_sphere(const Ball a1, const Ball a2, float &px, float &py,
                                            float &pz, float &cur) {
    if constexpr (V == pac::kExact) {
        const float3 c = pac::ex::edge_centre(a1, a2);
        px = c.x, py = c.y, pz = c.z, cur = 0.f;
    } else {
        pac::edge_foot(a1, a2, px, py, pz, cur);
    }
}

template <int V>
__device__ __forceinline__ bool dec_edge_attached(const Ball a1, const Ball a2, const Ball q,
                                                  float px, float py, float pz, float cur,
                                                  Tally &t) {
    if constexpr (V == pac::kExact) return pac::ex::edge_attached(a1, a2, q, t);
    else return pac::attached(q, px, py, pz, cur);
}

// End of a warp-per-ball kernel (all lanes present): add the lanes'
// tallies to the counters.
template <int V>
__device__ __forceinline__ void flush_tally(const Tally &t, unsigned long long *ctr) {
    if constexpr (V == pac::kExact) {
        const unsigned long long e = warp_sum(t.evals), f = warp_sum(t.fallbacks);
        const bool r = __any_sync(kFull, t.range != 0);
        if ((threadIdx.x & 31) == 0) {
            bump(ctr, C_FILTER, e);
            bump(ctr, C_FALLBACK, f);
            if (r) bump(ctr, C_SOS_RANGE, 1);
        }
    }
}
// The same from a single thread.
template <int V>
__device__ __forceinline__ void flush_tally_thread(const Tally &t, unsigned long long *ctr) {
    if constexpr (V == pac::kExact) {
        if (t.evals) atomicAdd(&ctr[C_FILTER], (unsigned long long)t.evals);
        if (t.fallbacks) atomicAdd(&ctr[C_FALLBACK], (unsigned long long)t.fallbacks);
        if (t.range) atomicAdd(&ctr[C_SOS_RANGE], 1ull);
    }
}

// ------------------------------------------------------------------ scan
// Exclusive prefix sum of n values into out[0..n], out[n] = total.
template <class Tin>
__global__ void k_scan_reduce(const Tin *in, uint64_t n, uint64_t *bsum) {
    __shared__ uint64_t s[32];
    uint64_t base = (uint64_t)blockIdx.x * 4096;
    uint64_t acc = 0;
    for (int k = 0; k < 4; k++) {
        uint64_t i = base + (uint64_t)k * 1024 + threadIdx.x;
        if (i < n) acc += (uint64_t)in[i];
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint64_t v = s[threadIdx.x];
        v = warp_sum(v);
        if (threadIdx.x == 0) bsum[blockIdx.x] = v;
    }
}
__global__ void k_scan_blocks(uint64_t *bsum, uint64_t nb) {
    // single block: exclusive scan of nb block sums in place
    __shared__ uint64_t s[1024];
    uint64_t carry = 0;
    for (uint64_t base = 0; base < nb; base += 1024) {
        uint64_t i = base + threadIdx.x;
        uint64_t v = i < nb ? bsum[i] : 0;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            uint64_t t = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < nb) bsum[i] = carry + s[threadIdx.x] - v;
        uint64_t tot = s[1023];
        __syncthreads();
        carry += tot;
    }
    if (threadIdx.x == 0) bsum[nb] = carry;
}
template <class Tin, class Tout>
__global__ void k_scan_apply(const Tin *in, uint64_t n, const uint64_t *bsum, Tout *out) {
    __shared__ uint64_t s[1024];
    uint64_t base = (uint64_t)blockIdx.x * 4096;
    uint64_t carry = bsum[blockIdx.x];
    for (int k = 0; k < 4; k++) {
        uint64_t i = base + (uint64_t)k * 1024 + threadIdx.x;
        uint64_t v = i < n ? (uint64_t)in[i] : 0;
        s[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            uint64_t t = threadIdx.x >= (unsigned)o ? s[threadIdx.x - o] : 0;
            __syncthreads();
            s[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < n) out[i] = (Tout)(carry + s[threadIdx.x] - v);
        uint64_t tot = s[1023];
        __syncthreads();
        carry += tot;
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = (Tout)bsum[gridDim.x];
}

template <class Tin, class Tout>
static int exclusive_scan(pac::Ctx &ctx, const Tin *in, uint64_t n, Tout *out) {
    uint64_t nb = (n + 4095) / 4096;
    if (nb == 0) nb = 1;
    uint64_t *bsum = ctx.arena.alloc_n<uint64_t>(nb + 1);
    if (!bsum) return PAC_ERR_OOM;
    k_scan_reduce<Tin><<<(unsigned)nb, 1024, 0, ctx.stream>>>(in, n, bsum);
    LAUNCH_CHECK(ctx);
    k_scan_blocks<<<1, 1024, 0, ctx.stream>>>(bsum, nb);
    LAUNCH_CHECK(ctx);
    k_scan_apply<Tin, Tout><<<(unsigned)nb, 1024, 0, ctx.stream>>>(in, n, bsum, out);
    LAUNCH_CHECK(ctx);
    return PAC_OK;
}

// ------------------------------------------------------------------ grid
__global__ void k_mol_ids(const uint64_t *off, uint32_t n_mol, uint32_t *mol) {
    uint32_t m = blockIdx.x;
    if (m >= n_mol) return;
    for (uint64_t i = off[m] + threadIdx.x; i < off[m + 1]; i += blockDim.x) mol[i] = m;
}

// min/max of raw x, y, z, r per molecule (AlphaComplexLargeData.cu:1088-1110).
// Floats are compared through an order-preserving int key.
__global__ void k_bbox(const float4 *balls, uint64_t n, const uint32_t *mol, int *mm) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool act = i < n;
    uint32_t m = act ? mol_of(mol, i) : 0xffffffffu;
    float4 b = act ? balls[i] : make_float4(0, 0, 0, 0);
    int k[4] = {fkey(b.x), fkey(b.y), fkey(b.z), fkey(b.w)};
    uint32_t m0 = __shfl_sync(kFull, m, 0);
    bool uniform = __all_sync(kFull, act && m == m0);
    for (int q = 0; q < 4; q++) {
        if (uniform) {
            int lo = k[q], hi = k[q];
            for (int o = 16; o; o >>= 1) {
                lo = min(lo, __shfl_xor_sync(kFull, lo, o));
                hi = max(hi, __shfl_xor_sync(kFull, hi, o));
            }
            if ((threadIdx.x & 31) == 0) {
                atomicMin(&mm[m * 8 + q], lo);
                atomicMax(&mm[m * 8 + 4 + q], hi);
            }
        } else if (act) {
            atomicMin(&mm[m * 8 + q], k[q]);
            atomicMax(&mm[m * 8 + 4 + q], k[q]);
        }
    }
}

// grid parameters per molecule (AlphaComplexLargeData.cu:1119-1123)
__global__ void k_grid(const int *mm, uint32_t n_mol, float sol, float alpha, MolGrid *g,
                       uint64_t *ncell) {
    uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n_mol) return;
    float minX = funkey(mm[m * 8 + 0]), minY = funkey(mm[m * 8 + 1]),
          minZ = funkey(mm[m * 8 + 2]);
    float maxX = funkey(mm[m * 8 + 4]), maxY = funkey(mm[m * 8 + 5]),
          maxZ = funkey(mm[m * 8 + 6]), maxRadius = funkey(mm[m * 8 + 7]);
    float possibleMaxRadius = __fsqrt_rn(__fadd_rn(__fmul_rn(maxRadius, maxRadius), alpha));
    float stepSize = __fmul_rn(2.0f, possibleMaxRadius);
    int gx = (int)__fdiv_rn(__fsub_rn(maxX, minX), stepSize) + 1;
    int gy = (int)__fdiv_rn(__fsub_rn(maxY, minY), stepSize) + 1;
    int gz = (int)__fdiv_rn(__fsub_rn(maxZ, minZ), stepSize) + 1;
    MolGrid r;
    r.minx = minX;
    r.miny = minY;
    r.minz = minZ;
    r.step = stepSize;
    r.gx = gx;
    r.gy = gy;
    r.gz = gz;
    // r + sol is rounded monotonically, so the extreme radii bound every
    // ball's weight; the margin covers the rounding of the square
    const float rlo = fabsf(__fadd_rn(funkey(mm[m * 8 + 3]), sol)), rhi = fabsf(__fadd_rn(maxRadius, sol));
    const float rm = fmaxf(rlo, rhi);
    r.wmax = __fmul_rn(__fmul_rn(rm, rm), 1.0f + 1.0f / 1024.0f);
    r.cell_base = 0;
    r.ncell = (uint64_t)max(gx, 0) * (uint64_t)max(gy, 0) * (uint64_t)max(gz, 0);
    r.atom_base = 0;
    g[m] = r;
    ncell[m] = r.ncell;
}

// cell key (AlphaComplexLargeData.cu:65-78) and a slot within the cell
__global__ void k_cellkey(const float4 *balls, uint64_t n, const uint32_t *mol, const MolGrid *g,
                          uint32_t *gcell, uint32_t *slot, uint32_t *cellcnt) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const MolGrid G = g[mol_of(mol, i)];
    float4 b = balls[i];
    int cellX = (int)__fdiv_rn(__fsub_rn(b.x, G.minx), G.step);
    int cellY = (int)__fdiv_rn(__fsub_rn(b.y, G.miny), G.step);
    int cellZ = (int)__fdiv_rn(__fsub_rn(b.z, G.minz), G.step);
    int cell = cellX + G.gx * cellY + G.gx * G.gy * cellZ;
    uint32_t gc = (uint32_t)(G.cell_base + (uint64_t)cell);
    gcell[i] = gc;
    slot[i] = atomicAdd(&cellcnt[gc], 1u);
}

__global__ void k_scatter(uint64_t n, const uint32_t *gcell, const uint32_t *slot,
                          const uint32_t *cellbeg, uint32_t *perm) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    perm[cellbeg[gcell[i]] + slot[i]] = (uint32_t)i;
}

// order each cell by input index: the stable sort's tie order
__global__ void k_cellsort(uint64_t ncell, const uint32_t *cellbeg, uint32_t *perm) {
    uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    uint32_t b = cellbeg[c], e = cellbeg[c + 1];
    for (uint32_t i = b + 1; i < e; i++) {
        uint32_t v = perm[i];
        uint32_t j = i;
        while (j > b && perm[j - 1] > v) {
            perm[j] = perm[j - 1];
            j--;
        }
        perm[j] = v;
    }
}

__global__ void k_gather(uint64_t n, const uint32_t *perm, const float4 *balls, float sol,
                         const uint32_t *gcell, const uint32_t *mol, const MolGrid *g,
                         float4 *at, uint32_t *orig, uint32_t *cellof) {
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    uint32_t i = perm[p];
    float4 b = balls[i];
    at[p] = make_float4(b.x, b.y, b.z, __fadd_rn(b.w, sol));
    orig[p] = (uint32_t)(i - g[mol_of(mol, i)].atom_base);
    cellof[p] = gcell[i];
}

// ------------------------------------------------------------------ edges
// One warp per ball i: the candidates are the balls l > i of the 27 cells
// around i's cell whose linear index is >= i's (AlphaComplexLargeData.cu:
// 80-165); each passes the power filter (markRealEdges) or not.  Lane k < 27
// owns neighbour cell k in the reference's loop order, so a warp prefix sum
// over the cell sizes enumerates the candidates in ascending l.
template <int V, bool FILL>
__global__ void __launch_bounds__(256) k_edges(uint64_t n, const float4 *__restrict__ at,
                                               const uint32_t *__restrict__ cellof,
                                               const uint32_t *__restrict__ cellbeg,
                                               const uint32_t *__restrict__ mol,
                                               const MolGrid *__restrict__ grids, float alpha,
                                               uint32_t *ecount, const uint64_t *eoff,
                                               uint32_t *ER, unsigned long long *ctr) {
    const int lane = threadIdx.x & 31;
    uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long cand_acc = 0, alpha_acc = 0;
    Tally tally;
    for (uint64_t p = warp; p < n; p += nwarps) {
        const MolGrid G = grids[mol_of(mol, p)];
        int cell = (int)(cellof[p] - G.cell_base);
        int gX = cell % G.gx, t = cell / G.gx, gY = t % G.gy, gZ = t / G.gy;
        uint32_t beg = 0, cnt = 0;
        if (lane < 27) {
            int i = lane / 9 - 1, j = (lane / 3) % 3 - 1, k = lane % 3 - 1;
            bool ok = !((gZ + i >= G.gz) || (gY + j >= G.gy) || (gX + k >= G.gx)) &&
                      !((gZ + i < 0) || (gY + j < 0) || (gX + k < 0));
            if (ok) {
                int adj = (gZ + i) * G.gx * G.gy + (gY + j) * G.gx + (gX + k);
                if (adj >= cell) {
                    uint64_t gc = G.cell_base + (uint64_t)adj;
                    uint32_t b = cellbeg[gc], e = cellbeg[gc + 1];
                    if (adj == cell) b = (uint32_t)p + 1;
                    if (e > b) {
                        beg = b;
                        cnt = e - b;
                    }
                }
            }
        }
        uint32_t incl = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t v = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += v;
        }
        uint32_t total = __shfl_sync(kFull, incl, 31);
        const Ball A = pac::ld_ball(&at[p]);
        uint64_t out = FILL ? eoff[p] : 0;
        uint32_t kept = 0;
        for (uint32_t base = 0; base < total; base += 32) {
            uint32_t s = base + lane;
            bool act = s < total;
            // segment owning slot s: first lane whose inclusive sum exceeds s
            int lo = 0;
            for (int step = 16; step; step >>= 1) {
                uint32_t v = __shfl_sync(kFull, incl, lo + step - 1);
                if (v <= s) lo += step;
            }
            uint32_t sinc = __shfl_sync(kFull, incl, lo & 31);
            uint32_t sbeg = __shfl_sync(kFull, beg, lo & 31);
            uint32_t scnt = __shfl_sync(kFull, cnt, lo & 31);
            bool pass = false;
            uint32_t l = 0;
            if (act) {
                l = sbeg + (s - (sinc - scnt));
                pass = dec_edge<V>(A, pac::ld_ball(&at[l]), alpha, tally);
            }
            unsigned m = __ballot_sync(kFull, pass);
            if (FILL && pass) ER[out + kept + __popc(m & ((1u << lane) - 1))] = l;
            kept += __popc(m);
        }
        if (lane == 0) {
            if (!FILL) ecount[p] = kept;
            cand_acc += total;
            alpha_acc += kept;
        }
    }
    if (!FILL) flush_tally<V>(tally, ctr);
    if (!FILL && lane == 0) {
        bump(ctr, C_CAND_E, cand_acc);
        bump(ctr, C_ALPHA_E, alpha_acc);
    }
}

// words of link matrix per ball
__global__ void k_link_size(uint64_t n, const uint64_t *eoff, uint64_t *lsize,
                            unsigned long long *ctr) {
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    uint64_t deg = eoff[p + 1] - eoff[p];
    uint64_t W = (deg + 63) >> 6;
    lsize[p] = deg * W;
    atomicMax(&ctr[C_MAXDEG], (unsigned long long)deg);
}

// ------------------------------------------------------------------ triangles
// One warp per ball i: bit (a, b) of i's link matrix is set when
// (i, v1 = N[a], v2 = N[b]) is a candidate triangle -- edge v1v2 is an alpha
// edge (AlphaComplexLargeData.cu:192-296) -- and passes markRealTriangles.
template <int V>
__global__ void __launch_bounds__(256) k_link(uint64_t n, const float4 *__restrict__ at,
                                              const uint64_t *__restrict__ eoff,
                                              const uint32_t *__restrict__ ER,
                                              const uint64_t *__restrict__ loff, uint64_t *link,
                                              float alpha, unsigned long long *ctr) {
    __shared__ uint64_t srow[8][kMaxW];
    __shared__ uint64_t sL[8][64];  // link rows of a ball of <= 64 upper neighbours
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned long long cand_acc = 0, alpha_acc = 0;
    Tally tally;
    // balls handed out by a counter: a warp that finishes a small ball takes
    // the next one instead of waiting for its block's largest
    for (;;) {
        uint64_t p = 0;
        if (lane == 0) p = atomicAdd(&ctr[C_NEXT], 1ull);
        p = __shfl_sync(kFull, p, 0);
        if (p >= n) break;
        const uint64_t e0 = eoff[p];
        const int deg = (int)(eoff[p + 1] - e0);
        if (deg < 2) continue;
        const int W = (deg + 63) >> 6;
        const uint32_t *N = ER + e0;
        uint64_t *L = link + loff[p];
        const Ball A = pac::ld_ball(&at[p]);
        if (deg <= 64) {
            // all pairs (a, b), a < b, flattened over the lanes: row a holds
            // deg - 1 - a of them, P(a) = a (2 deg - 1 - a) / 2 before it
            const int total = deg * (deg - 1) / 2;
            for (int k = lane; k < deg; k += 32) sL[wib][k] = 0;
            __syncwarp();
            for (int base = 0; base < total; base += 32) {
                const int s2 = base + lane;
                bool cand = false, pass = false;
                int a = 0, b = 0;
                if (s2 < total) {
                    const float D = (float)(2 * deg - 1);
                    a = (int)((D - sqrtf(D * D - 8.0f * (float)s2)) * 0.5f);
                    a = max(0, min(a, deg - 2));
                    while (a > 0 && a * (2 * deg - 1 - a) / 2 > s2) a--;
                    while (a + 1 <= deg - 2 && (a + 1) * (2 * deg - 2 - a) / 2 <= s2) a++;
                    b = a + 1 + (s2 - a * (2 * deg - 1 - a) / 2);
                    const uint32_t v1 = __ldg(&N[a]), v2 = __ldg(&N[b]);
                    const uint64_t e1 = eoff[v1];
                    const int deg1 = (int)(eoff[v1 + 1] - e1);
                    const int pos = lbound(ER + e1, deg1, v2);
                    cand = pos < deg1 && __ldg(&ER[e1 + pos]) == v2;
                    if (cand) {
                        float4 o;
                        pass = dec_tri<V>(A, pac::ld_ball(&at[v1]), pac::ld_ball(&at[v2]), alpha, o,
                                          tally);
                    }
                    if (pass) atomicOr((unsigned long long *)&sL[wib][a], 1ull << b);
                }
                const unsigned cm = __ballot_sync(kFull, cand), pm = __ballot_sync(kFull, pass);
                if (lane == 0) {
                    cand_acc += __popc(cm);
                    alpha_acc += __popc(pm);
                }
            }
            __syncwarp();
            for (int k = lane; k < deg; k += 32) L[k] = sL[wib][k];
            __syncwarp();
            continue;
        }
        for (int a = 0; a < deg - 1; a++) {
            if (lane < kMaxW) srow[wib][lane] = 0;
            __syncwarp();
            const uint32_t v1 = __ldg(&N[a]);
            const Ball A1 = pac::ld_ball(&at[v1]);
            const uint32_t *N1 = ER + eoff[v1];
            const int deg1 = (int)(eoff[v1 + 1] - eoff[v1]);
            for (int base = a + 1; base < deg; base += 32) {
                int b = base + lane;
                bool cand = false, pass = false;
                if (b < deg) {
                    uint32_t v2 = __ldg(&N[b]);
                    int pos = lbound(N1, deg1, v2);
                    cand = pos < deg1 && __ldg(&N1[pos]) == v2;
                    if (cand) {
                        float4 o;
                        pass = dec_tri<V>(A, A1, pac::ld_ball(&at[v2]), alpha, o, tally);
                    }
                }
                unsigned cm = __ballot_sync(kFull, cand), pm = __ballot_sync(kFull, pass);
                if (lane == 0) {
                    cand_acc += __popc(cm);
                    alpha_acc += __popc(pm);
                    int w = base >> 6, sh = base & 63;
                    srow[wib][w] |= (uint64_t)pm << sh;
                    if (sh > 32 && w + 1 < kMaxW) srow[wib][w + 1] |= (uint64_t)pm >> (64 - sh);
                }
                __syncwarp();
            }
            if (lane < W) L[(uint64_t)a * W + lane] = srow[wib][lane];
            __syncwarp();
        }
        if (lane < W) L[(uint64_t)(deg - 1) * W + lane] = 0;
    }
    flush_tally<V>(tally, ctr);
    if (lane == 0) {
        bump(ctr, C_CAND_T, cand_acc);
        bump(ctr, C_ALPHA_T, alpha_acc);
    }
}

// ------------------------------------------------------------------ tetrahedra
struct TetArgs {
    uint64_t n;
    const float4 *at;
    const uint32_t *orig;
    const uint64_t *eoff;
    const uint32_t *ER;
    const uint64_t *loff;
    const uint64_t *link;
    uint64_t *faces;
    const uint32_t *cellbeg;
    const uint32_t *mol;
    const MolGrid *grids;
    float alpha;
    // survivors (as-written) / ordered output (as-run fill)
    uint2 *surv;          // (ball, packed a | b << 8 | c << 16)
    uint64_t surv_cap;
    uint32_t *tcount;     // per ball
    uint2 *pend;          // tetrahedra waiting for the exact SoS
    uint64_t pend_cap;
    const uint64_t *toff; // as-run fill: output offsets per ball
    uint32_t *tets_out;   // as-run fill: sorted-space vertex quadruples
    unsigned long long *ctr;   // the pass's counters, or a chunk's (enumeration)
    const uint32_t *cellof;    // global cell of each sorted ball
    int refute;                // enumeration: refute early against the group's best candidate
    int verify;                // scan: replay every certified decision and count disagreements
    int unit_rows;             // rows of a large ball per enumeration work unit
    int scan_claim;            // queue entries a scan warp claims at a time
};

__device__ __forceinline__ void mark_face(uint64_t *F, uint64_t row_base, int W, int a, int b) {
    atomicOr((unsigned long long *)&F[row_base + (uint64_t)a * W + (b >> 6)],
             1ull << (b & 63));
}

// One warp per ball v1.  For each upper neighbour v2 = N[a] the lanes take
// the alpha triangles (v1, v2, v3 = N[b]); the fourth vertices v4 = N[c]
// (c > b) are the common bits of rows a and b of v1's link matrix whose
// face (v2, v3, v4) is also an alpha triangle -- exactly the reference's
// candidate tetrahedra (AlphaComplexLargeData.cu:350-529).  Each candidate
// then passes markRealTets and, as written, the empty-orthosphere test.
// As run (the orthosphere test skipped): MODE 1 counts per ball, MODE 2
// writes in reference order (needs MODE 1's offsets).
template <int V, int MODE>
__global__ void __launch_bounds__(256) k_tets(TetArgs A) {
    __shared__ uint16_t smap[8][kMaxDeg];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long cand_acc = 0, alpha_acc = 0;
    Tally tally;
    for (uint64_t p = warp; p < A.n; p += nwarps) {
        const uint64_t e0 = A.eoff[p];
        const int deg = (int)(A.eoff[p + 1] - e0);
        uint32_t ball_count = 0;
        if (deg >= 3) {
            const int W = (deg + 63) >> 6;
            const uint32_t *N = A.ER + e0;
            const uint64_t lp = A.loff[p];
            const uint64_t *Lp = A.link + lp;
            const Ball B1 = pac::ld_ball(&A.at[p]);
            uint64_t out_base = (MODE == 2) ? A.toff[p] : 0;
            for (int a = 0; a < deg - 2; a++) {
                uint64_t ra[kMaxW];
                int nb = 0;
#pragma unroll
                for (int w = 0; w < kMaxW; w++) {
                    ra[w] = w < W ? Lp[(uint64_t)a * W + w] : 0;
                    nb += __popcll(ra[w]);
                }
                if (nb < 2) continue;
                const uint32_t v2 = __ldg(&N[a]);
                const uint64_t e2 = A.eoff[v2];
                const int deg2 = (int)(A.eoff[v2 + 1] - e2);
                const int W2 = (deg2 + 63) >> 6;
                const uint64_t l2 = A.loff[v2];
                const uint64_t *L2 = A.link + l2;
                for (int c = a + 1 + lane; c < deg; c += 32) {
                    uint32_t x = __ldg(&N[c]);
                    int pos = lbound(A.ER + e2, deg2, x);
                    smap[wib][c] = (pos < deg2 && __ldg(&A.ER[e2 + pos]) == x) ? (uint16_t)pos
                                                                               : (uint16_t)0xffff;
                }
                __syncwarp();
                const Ball B2 = pac::ld_ball(&A.at[v2]);
                for (int k0 = 0; k0 < nb; k0 += 32) {
                    int b = (k0 + lane < nb) ? select_bit(ra, W, k0 + lane) : -1;
                    uint32_t lane_cnt = 0;
                    // MODE 2 needs each lane's count first to place its rows
                    uint64_t lane_off = 0;
                    for (int sweep = (MODE == 2 ? 0 : 1); sweep < 2; sweep++) {
                        if (MODE == 2 && sweep == 1) {
                            uint32_t incl = lane_cnt;
                            for (int o = 1; o < 32; o <<= 1) {
                                uint32_t v = __shfl_up_sync(kFull, incl, o);
                                if (lane >= o) incl += v;
                            }
                            lane_off = out_base + ball_count + (incl - lane_cnt);
                            ball_count += __shfl_sync(kFull, incl, 31);
                            lane_cnt = 0;
                        }
                        if (b >= 0) {
                            const uint32_t v3 = __ldg(&N[b]);
                            const Ball B3 = pac::ld_ball(&A.at[v3]);
                            const int mb = smap[wib][b];
                            uint64_t m[kMaxW];
#pragma unroll
                            for (int w = 0; w < kMaxW; w++)
                                m[w] = w < W ? (ra[w] & Lp[(uint64_t)b * W + w] & above_mask(b, w))
                                             : 0;
                            const uint64_t *R2 = L2 + (uint64_t)mb * W2;
                            for (int w = 0; w < kMaxW; w++) {
                                uint64_t bits = m[w];
                                while (bits) {
                                    int c = w * 64 + __ffsll((long long)bits) - 1;
                                    bits &= bits - 1;
                                    int mc = smap[wib][c];
                                    if (mb == 0xffff || mc == 0xffff) continue;
                                    if (!((__ldg(&R2[mc >> 6]) >> (mc & 63)) & 1ull)) continue;
                                    if (sweep == 1) cand_acc++;
                                    const uint32_t v4 = __ldg(&N[c]);
                                    const Ball B4 = pac::ld_ball(&A.at[v4]);
                                    float4 o;
                                    if (!dec_tet<V>(B1, B2, B3, B4, A.alpha, o, tally)) continue;
                                    if (sweep == 1) alpha_acc++;
                                    if (MODE == 1) {
                                        lane_cnt++;
                                        continue;
                                    }
                                    if (MODE == 2) {
                                        if (sweep == 0) {
                                            lane_cnt++;
                                            continue;
                                        }
                                        uint64_t q = lane_off + lane_cnt++;
                                        uint4 t4 = make_uint4((uint32_t)p, v2, v3, v4);
                                        *(uint4 *)&A.tets_out[4 * q] = t4;
                                        mark_face(A.faces, lp, W, a, b);
                                        mark_face(A.faces, lp, W, a, c);
                                        mark_face(A.faces, lp, W, b, c);
                                        mark_face(A.faces, l2, W2, mb, mc);
                                        continue;
                                    }
                                }
                            }
                        }
                    }
                    if (MODE != 2) {
                        uint32_t s = lane_cnt;
                        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
                        ball_count += s;
                    }
                }
                __syncwarp();
            }
        }
        if (lane == 0 && MODE != 2) A.tcount[p] = ball_count;
    }
    cand_acc = warp_sum(cand_acc);
    alpha_acc = warp_sum(alpha_acc);
    if (MODE == 1) flush_tally<V>(tally, A.ctr);  // MODE 2 repeats MODE 1's tests
    if (lane == 0) {
        bump(A.ctr, C_CAND_Q, cand_acc);
        bump(A.ctr, C_ALPHA_Q, alpha_acc);
    }
}

// Positions of v2 < v3 < v4 in ball p's upper-neighbour list N (ascending,
// deg entries), packed a | b << 8 | c << 16 as the survivor lists hold them.
__device__ __forceinline__ uint32_t key_of(const uint32_t *N, int deg, uint32_t v2, uint32_t v3,
                                           uint32_t v4) {
    return (uint32_t)lbound(N, deg, v2) | ((uint32_t)lbound(N, deg, v3) << 8) |
           ((uint32_t)lbound(N, deg, v4) << 16);
}

// Records one tetrahedron that passed the orthosphere test (or, pending,
// one whose window held an exact zero): the survivor list, the per-ball
// count, and the marks of its four faces in the `faces` matrices.
__device__ __noinline__ void emit_survivor(const uint64_t *__restrict__ eoff,
                                           const uint32_t *__restrict__ ER,
                                           const uint64_t *__restrict__ loff, uint64_t *faces,
                                           uint2 *surv, uint64_t surv_cap, uint2 *pend,
                                           uint64_t pend_cap, unsigned long long *ctr,
                                           uint32_t *tcount, uint32_t p, uint32_t v2, uint32_t v3,
                                           uint32_t v4, bool pending) {
    const uint64_t e0 = eoff[p];
    const int deg = (int)(eoff[p + 1] - e0);
    const uint32_t *N = ER + e0;
    const uint32_t key = key_of(N, deg, v2, v3, v4);
    if (pending) {
        unsigned long long q = atomicAdd(&ctr[C_PEND], 1ull);
        if (q < pend_cap) pend[q] = make_uint2(p, key);
        return;
    }
    unsigned long long q = atomicAdd(&ctr[C_SURV], 1ull);
    if (q < surv_cap) surv[q] = make_uint2(p, key);
    atomicAdd(&tcount[p], 1u);
    const int W = (deg + 63) >> 6;
    const uint64_t lp = loff[p];
    const int a = key & 0xff, b = (key >> 8) & 0xff, c = (key >> 16) & 0xff;
    mark_face(faces, lp, W, a, b);
    mark_face(faces, lp, W, a, c);
    mark_face(faces, lp, W, b, c);
    const uint64_t e2 = eoff[v2];
    const int deg2 = (int)(eoff[v2 + 1] - e2);
    const int mb = lbound(ER + e2, deg2, v3), mc = lbound(ER + e2, deg2, v4);
    mark_face(faces, loff[v2], (deg2 + 63) >> 6, mb, mc);
}

// The 27-cell window of the orthosphere and attachment tests, visited as
// the centre cell first (window_centre) and then ten parts (window_part):
// the two side cells of the centre row, then the eight other x-rows -- for
// z and y offsets (i, j) the cells (gX-1 .. gX+1, gY+j, gZ+i), clipped to
// the grid, are consecutive in the cell order, so their balls form one range
// of the sorted balls.  Faces before corners, so the balls nearest the
// window centre come first and most tests end early.  Together these are the
// reference's window (AlphaComplexLargeData.cu:621-733): the centre cell
// through its wrapped linear index, the 26 neighbours range-checked per
// axis; the same cells in another order, and the tests' outcome does not
// depend on the order.
constexpr int kWindowParts = 10;
// rows 2..9 as (i + 1) | (j + 1) << 2, 4 bits each:
// (0,-1) (0,1) (-1,0) (1,0) (-1,-1) (-1,1) (1,-1) (1,1)
constexpr uint64_t kRowOrder = 0x1ull | 0x9ull << 4 | 0x4ull << 8 | 0x6ull << 12 | 0x0ull << 16 |
                               0x8ull << 20 | 0x2ull << 24 | 0xAull << 28;

// [beg, end) of window part r, or false when it lies outside the grid.
__device__ __forceinline__ bool window_part(const MolGrid &G, const uint32_t *cellbeg, int gX,
                                            int gY, int gZ, int r, uint32_t &beg, uint32_t &end) {
    long long zz = gZ, yy = gY, xlo, xhi;
    if (r < 2) {  // a side cell of the centre row
        xlo = xhi = (long long)gX + (r == 0 ? -1 : 1);
    } else {
        const int code = (int)((kRowOrder >> (4 * (r - 2))) & 0xf);
        zz += (code & 3) - 1;
        yy += (code >> 2) - 1;
        xlo = (long long)gX - 1;
        xhi = (long long)gX + 1;
    }
    if (zz < 0 || zz >= G.gz || yy < 0 || yy >= G.gy) return false;
    xlo = max(xlo, 0ll);
    xhi = min(xhi, (long long)G.gx - 1);
    if (xlo > xhi) return false;
    const uint64_t row = G.cell_base + (uint64_t)(zz * G.gy + yy) * (uint64_t)G.gx;
    beg = cellbeg[row + (uint64_t)xlo];
    end = cellbeg[row + (uint64_t)xhi + 1];
    return true;
}

// The window's centre cell as the reference reads it, through its wrapped
// linear index cl.w: [beg, end), or an empty range (counted) when cl.w names
// no cell (out-of-range read in the reference, AlphaComplexLargeData.cu:
// 625-627).  When the centre (cl.x, cl.y, cl.z) lies inside the grid this is
// the centre cell itself, which no part holds; when it lies outside, the
// parts hold the window's in-grid cells and this is the extra cell the
// wrapped index names.
__device__ __forceinline__ void window_centre(const MolGrid &G, const uint32_t *cellbeg, int4 cl,
                                              uint32_t &beg, uint32_t &end,
                                              unsigned long long &oob) {
    beg = end = 0;
    if (cl.w < 0 || (uint64_t)cl.w >= G.ncell) {
        oob++;
        return;
    }
    beg = cellbeg[G.cell_base + (uint64_t)cl.w];
    end = cellbeg[G.cell_base + (uint64_t)cl.w + 1];
}

// Cell coordinate (int)((p - lo) / step) of the reference (LD:621-623), with
// the IEEE division replaced by a multiplication by inv = fl(1 / step)
// whenever that provably truncates to the same integer: the product is
// within 3.1 ulp of the quotient, so when no integer lies within 16 ulp of
// it both truncate alike.  Otherwise (and for huge or non-finite values)
// the division itself.
__device__ __forceinline__ int cell_coord_fast(float p, float lo, float step, float inv) {
    const float d = __fsub_rn(p, lo);
    const float q = __fmul_rn(d, inv);
    const float t = truncf(q);
    const float f = fabsf(__fsub_rn(q, t));
    if (fabsf(q) < 4194304.0f && fminf(f, __fsub_rn(1.0f, f)) > 16.0f * pac::cert::kU * fabsf(q) + 1e-30f)
        return (int)t;
    return pac::cell_coord(p, lo, step);
}

// The window cell of an orthosphere centre: (gridX, gridY, gridZ, wrapped
// linear index), as the reference forms it (LD:621-626).
__device__ __forceinline__ int4 window_cell(const MolGrid &G, float x, float y, float z) {
    const float inv = __frcp_rn(G.step);
    const int gX = cell_coord_fast(x, G.minx, G.step, inv);
    const int gY = cell_coord_fast(y, G.miny, G.step, inv);
    const int gZ = cell_coord_fast(z, G.minz, G.step, inv);
    return make_int4(gX, gY, gZ, lin3(gX, gY, gZ, G.gx, G.gy));
}

// Whether the reference's window of an orthosphere centre (x, y, z) holds
// a ball at (bx, by, bz) in the grid: certainly so when the two are less
// than 0.99 cell steps apart on every axis.  The cells are truncations of
// the monotone binary32 map v -> (v - lo) / step (LD:72-74, 621-623), so the
// two quotients differ by less than one (the rounding is far below the 1 %
// margin for grids of at most 16384 cells per axis); the ball's quotient is
// non-negative, so the centre's truncated cell is never below -0 and the
// ball's cell lies within one of it per axis.  A centre cell inside the grid
// is read as itself; outside the grid the ball's cell differs from it and is
// one of the 26 in-grid neighbours.  Either way the reference visits it.
__device__ __forceinline__ bool surely_in_window(float x, float y, float z, float bx, float by,
                                                 float bz, float reach) {
    return fmaxf(fabsf(bx - x), fmaxf(fabsf(by - y), fabsf(bz - z))) <= reach;
}

// Queue slots are handed out to warps in blocks (one atomic per block, not
// per batch: a single counter served every warp).  Slots a warp reserved
// but did not fill are marked with this ball index, and the scan skips them.
constexpr uint32_t kNoTet = 0xffffffffu;
constexpr uint64_t kQBlock = 128;

// ---- the as-written tetrahedra: enumeration, then a scan over an HBM queue
// Enumeration (k_tets_enum): ball p's candidate tetrahedra are the
// (p, v2 = N[a], v3 = N[b], v4 = N[c]), a < b < c, with (p, v2, v3),
// (p, v2, v4), (p, v3, v4) alpha triangles (bits of p's link rows) and
// (v2, v3, v4) one too (a bit of v2's link matrix) -- exactly the
// reference's candidates (AlphaComplexLargeData.cu:350-529).  Per row a the
// candidate set of every triangle group (a, b) is built bitwise, the pairs
// (b, c) are written group by group to a per-warp list in shared memory, and
// the list is evaluated 32 at a time with every lane busy: markRealTets,
// then an early refutation, then the queue.
//
// Early refutation.  Within one group the fourth vertices lie in the pencil
// of spheres orthogonal to the balls p, v2, v3; on either side of the
// triangle's plane the candidate whose orthosphere comes first along the
// pencil lies inside the orthosphere of every other candidate on that side.
// Each lane's tetrahedron is therefore tested against the best candidate
// of its group and side found so far (a shared-memory minimum over the
// lanes' orthocentres projected on the triangle normal), with the
// reference's own arithmetic (orient3d, insphere_w), provided that ball lies
// in the reference's window of the tetrahedron (surely_in_window).  A violation there is a
// violation the reference finds: the tetrahedron is dropped.  The rest
// (a few per cent) go to the queue.
struct TetQueue {
    uint4 *vid;    // (v1, v2, v3, v4); v1 = kNoTet marks an unused slot
    float4 *sph;   // orthosphere centre (x, y, z) and power of v2, as markRealTets gives them
    uint64_t cap;
};

template <int KW>
struct EnumSmem;
// balls of at most 64 upper neighbours: one link word per row, all staged
template <>
struct EnumSmem<1> {
    static constexpr int kDeg = 64, kL2Cap = 64, kWarps = 8, kBufs = 2, kLBufs = 2;
    float4 sb[kWarps][kDeg];      // balls of p's upper neighbours
    uint64_t sL[kWarps][kDeg];    // p's link rows
    uint64_t sL2[kWarps][kLBufs][kL2Cap]; // v2's link rows (when they fit), this row and the next
    uint32_t sN2[kWarps][kBufs][kMaxDeg];// v2's upper neighbours, this row and the next
    uint64_t sE2[kWarps][kDeg];   // per neighbour v2: its first upper neighbour's index,
    uint64_t sLo[kWarps][kDeg];   // its link rows' offset,
    uint16_t sD2[kWarps][kDeg];   // its upper degree
    uint32_t sN[kWarps][kDeg];    // p's upper neighbours
    uint16_t smap[kWarps][kDeg];  // position of N[c] in v2's list, 0xffff: absent
    uint64_t pm[kWarps][32][1];   // the chunk's groups' fourth vertices (bits c)
    uint8_t gstart[kWarps][32];   // group starting at each slot of a batch
    uint8_t sBl[kWarps][kDeg];    // the b's of the row, ascending
    unsigned long long best[kWarps][64];  // per (j, side): orderable key << 32 | c
    pac::TetGroup grp[kWarps][32];        // markRealTets' products of the chunk's groups
};
// larger balls: rows read in place, v2's rows staged when they fit
template <>
struct EnumSmem<kMaxW> {
    static constexpr int kDeg = kMaxDeg, kL2Cap = 256, kWarps = 4, kBufs = 2, kLBufs = 1;
    float4 sb[kWarps][kDeg];
    uint64_t sL2[kWarps][kLBufs][kL2Cap];  // this row's only
    uint32_t sN2[kWarps][kBufs][kMaxDeg];  // this row and the next
    uint32_t sN[kWarps][kDeg];
    uint16_t smap[kWarps][kDeg];
    uint64_t pm[kWarps][32][kMaxW];
    uint8_t gstart[kWarps][32];
    uint8_t sBl[kWarps][kDeg];
    unsigned long long best[kWarps][64];
    pac::TetGroup grp[kWarps][32];
};

// Per-warp state of the queue reservation.
struct QRes {
    uint64_t pos, end;  // next free slot of the warp's block, its end
};

// Appends the lanes with `take` to the queue (warp-uniform call).
__device__ __forceinline__ void queue_append(const TetQueue &Q, unsigned long long *ctr, QRes &qr,
                                             bool take, uint4 vid, float4 sph) {
    const int lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(kFull, take);
    if (!m) return;
    const int k = __popc(m), rank = __popc(m & ((1u << lane) - 1));
    const uint64_t left = qr.end - qr.pos;
    uint64_t nb = 0;
    if ((uint64_t)k > left) {
        if (lane == 0) nb = atomicAdd(&ctr[C_SURV], (unsigned long long)kQBlock);
        nb = __shfl_sync(kFull, nb, 0);
    }
    if (take) {
        const uint64_t pos = (uint64_t)rank < left ? qr.pos + rank : nb + (rank - left);
        if (pos < Q.cap) {
            Q.vid[pos] = vid;
            Q.sph[pos] = sph;
        }
    }
    if ((uint64_t)k > left) {
        qr.pos = nb + (k - left);
        qr.end = nb + kQBlock;
    } else {
        qr.pos += k;
    }
}

// Marks the rest of the warp's block unused.
__device__ __forceinline__ void queue_close(const TetQueue &Q, QRes &qr) {
    const int lane = threadIdx.x & 31;
    for (uint64_t s = qr.pos + lane; s < qr.end; s += 32)
        if (s < Q.cap) Q.vid[s] = make_uint4(kNoTet, 0, 0, 0);
    qr.pos = qr.end;
}

// Asynchronous global -> shared copies (cp.async): the row after the
// current one is fetched while the current one is worked on.
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Starts copying row a's v2 (upper neighbours and, when they fit, link
// rows) into buffer buf of the warp's staging (KW = 1), as one cp.async
// group of this thread.
__device__ __forceinline__ void row_fetch(const TetArgs &A, EnumSmem<1> &S, int wib, int a,
                                          int buf) {
    const int lane = threadIdx.x & 31;
    const uint64_t e2 = S.sE2[wib][a];
    const int deg2 = S.sD2[wib][a];
    const int W2 = (deg2 + 63) >> 6;
    for (int k = lane; k < deg2; k += 32) cp_async4(&S.sN2[wib][buf][k], &A.ER[e2 + k]);
    if (deg2 * W2 <= EnumSmem<1>::kL2Cap) {
        const uint64_t *L2g = A.link + S.sLo[wib][a];
        for (int k = lane; k < deg2 * W2; k += 32) cp_async8(&S.sL2[wib][buf][k], &L2g[k]);
    }
    cp_async_commit();
}

// A heavy row's v2: where its upper neighbours and link rows start, and
// how many (KW = kMaxW; the light kernel stages these per ball).
struct RowSrc {
    uint64_t e2, loff;
    int deg2;
    bool valid;
};
__device__ __forceinline__ RowSrc row_src(const TetArgs &A, uint32_t v2) {
    const uint64_t e2 = A.eoff[v2];
    return RowSrc{e2, A.loff[v2], (int)(A.eoff[v2 + 1] - e2), true};
}
// Starts copying a heavy row's v2 neighbours into buffer buf (one cp.async
// group of this thread, empty when there is no such row).
__device__ __forceinline__ void heavy_fetch_n2(const TetArgs &A, EnumSmem<kMaxW> &S, int wib,
                                               const RowSrc &r, int buf) {
    const int lane = threadIdx.x & 31;
    if (r.valid)
        for (int k = lane; k < r.deg2; k += 32) cp_async4(&S.sN2[wib][buf][k], &A.ER[r.e2 + k]);
    cp_async_commit();
}

// One row a of ball p: v2 = N[a].  N, sb, sCell hold p's upper neighbours,
// their balls and cells (shared memory); L its link rows (W words each,
// shared or global); the rest is per-warp scratch.
template <int V, int KW>
__device__ __forceinline__ void tet_row(const TetArgs &A, const TetQueue &Q, EnumSmem<KW> &S,
                                        const int wib, QRes &qr, uint32_t p, int a, int buf,
                                        const RowSrc &cur, const RowSrc &nxt, int deg, int W,
                                        const uint64_t *L, const Ball B1, const MolGrid &G,
                                        bool refute, unsigned long long &cand_acc,
                                        unsigned long long &alpha_acc, unsigned long long &kill_acc,
                                        unsigned long long &ktest_acc, Tally &tally) {
    constexpr int kL2Cap = EnumSmem<KW>::kL2Cap;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1;
    const uint32_t *N = S.sN[wib];
    const float4 *sb = S.sb[wib];
    uint64_t ra[KW];
    int nb = 0;
#pragma unroll
    for (int w = 0; w < KW; w++) {
        ra[w] = w < W ? L[(uint64_t)a * W + w] : 0ull;
        nb += __popcll(ra[w]);
    }
    if constexpr (KW != 1) {
        // heavy rows in a pipeline of cp.async groups: this row's
        // neighbours (issued with the row before), its link rows (now), the
        // next row's neighbours (after the search below); every path
        // leaves exactly the next row's group pending
        const int W2c = (cur.deg2 + 63) >> 6;
        if (nb >= 2 && cur.deg2 * W2c <= EnumSmem<KW>::kL2Cap)
            for (int k = lane; k < cur.deg2 * W2c; k += 32)
                cp_async8(&S.sL2[wib][0][k], &A.link[cur.loff + k]);
        cp_async_commit();
        cp_async_wait<1>();  // this row's neighbours
        __syncwarp();
        if (nb < 2) {
            if constexpr (KW == kMaxW) heavy_fetch_n2(A, S, wib, nxt, buf ^ 1);
            cp_async_wait<1>();
            return;
        }
    } else {
        if (nb < 2) return;
    }
    const uint32_t v2 = N[a];
    uint32_t *sN2 = S.sN2[wib][buf];
    uint64_t *sL2 = S.sL2[wib][KW == 1 ? buf : 0];
    uint16_t *smap = S.smap[wib];
    uint8_t *sBl = S.sBl[wib];
    int deg2;
    const uint64_t *L2g;
    if constexpr (KW == 1) {
        // v2's lists were copied into buffer buf by row_fetch
        deg2 = S.sD2[wib][a];
        L2g = A.link + S.sLo[wib][a];
    } else {
        deg2 = cur.deg2;
        L2g = A.link + cur.loff;
    }
    const int W2 = (deg2 + 63) >> 6;
    const bool l2s = deg2 * W2 <= kL2Cap;
    // the b's of the row, ascending
#pragma unroll
    for (int w = 0; w < KW; w++) {
        if (w >= W) break;
        int before = 0;
#pragma unroll
        for (int v = 0; v < KW; v++)
            if (v < w) before += __popcll(ra[v]);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const bool bit = (ra[w] >> (32 * h + lane)) & 1ull;
            const unsigned bm = __ballot_sync(kFull, bit);
            const int lo = (int)__popcll(ra[w] & ((1ull << (32 * h)) - 1ull)) * (h ? 1 : 0);
            if (bit) sBl[before + lo + __popc(bm & lt_mask)] = (uint8_t)(w * 64 + 32 * h + lane);
        }
    }
    __syncwarp();
    // position of N[c] in v2's list, for c > a
    for (int c = a + 1 + lane; c < deg; c += 32) {
        const uint32_t x = N[c];
        int lo2 = 0, n2 = deg2;
        while (n2 > 0) {
            const int h = n2 >> 1;
            if (sN2[lo2 + h] < x) {
                lo2 += h + 1;
                n2 -= h + 1;
            } else {
                n2 = h;
            }
        }
        smap[c] = (lo2 < deg2 && sN2[lo2] == x) ? (uint16_t)lo2 : (uint16_t)0xffff;
    }
    if constexpr (KW == kMaxW) {
        heavy_fetch_n2(A, S, wib, nxt, buf ^ 1);
        cp_async_wait<1>();  // this row's link rows
    }
    __syncwarp();
    const float e12x = sb[a].x - B1.x, e12y = sb[a].y - B1.y, e12z = sb[a].z - B1.z;
    const float4 b2 = sb[a];
    const Ball B2{b2.x, b2.y, b2.z, b2.w};
    // groups (a, b) in chunks of 32 b's, lane j owning group j
    for (int k0 = 0; k0 < nb; k0 += 32) {
        const int nj = min(32, nb - k0);
        // lane j: the fourth vertices c > b with the three faces at p
        // (ra & L[b] & above b)
        uint64_t pm[KW];
        if (lane < nj) {
            const int b = sBl[k0 + lane];
            const int mb = smap[b];  // 0xffff: (v2, v3) has no alpha edge in v2's list
            if constexpr (V != pac::kExact) {
                const float4 b3 = sb[b];
                S.grp[wib][lane] = pac::tet_group(B1, B2, Ball{b3.x, b3.y, b3.z, b3.w});
            }
#pragma unroll
            for (int w = 0; w < KW; w++)
                pm[w] = (w < W && mb != 0xffff) ? (ra[w] & L[(uint64_t)b * W + w] & above_mask(b, w))
                                                : 0ull;
        } else {
#pragma unroll
            for (int w = 0; w < KW; w++) pm[w] = 0ull;
        }
        // the pre-candidates (faces at p only); the face (v2, v3, v4) is
        // checked in the batches below, where every lane is busy
        int cnt = 0;
#pragma unroll
        for (int w = 0; w < KW; w++) cnt += __popcll(pm[w]);
        int incl = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(kFull, incl, 31);
        // best-so-far slots of the chunk's groups (j, side)
        S.best[wib][lane] = ~0ull;
        S.best[wib][lane + 32] = ~0ull;
        const int myoff = incl - cnt;
#pragma unroll
        for (int w = 0; w < KW; w++) S.pm[wib][lane][w] = pm[w];
        // the chunk's candidates in group order, 32 per batch: slot t holds
        // the r-th fourth vertex of group j, t = start(j) + r.  A batch finds
        // its slots' groups from the mask of the group starts inside it; a
        // slot before the first start continues the previous batch's last
        // group.
        int jcarry = 0;
        for (int s0 = 0; s0 < total; s0 += 32) {
            __syncwarp();
            const int rel = myoff - s0;
            const bool starts = cnt > 0 && rel >= 0 && rel < 32;
            if (starts) S.gstart[wib][rel] = (uint8_t)lane;
            const unsigned M = __reduce_or_sync(kFull, starts ? 1u << rel : 0u);
            __syncwarp();
            const unsigned upto = M & (0xffffffffu >> (31 - lane));
            const int j = upto ? (int)S.gstart[wib][31 - __clz(upto)] : jcarry;
            jcarry = __shfl_sync(kFull, j, 31);
            const int r = s0 + lane - __shfl_sync(kFull, myoff, j);
            const bool act = s0 + lane < total;
            const int c = act ? select_kw<KW>(S.pm[wib][j], r) : 0;
            const int b = act ? (int)sBl[k0 + j] : 0;
            bool face = false;
            if (act) {  // (v2, v3, v4) an alpha triangle: bit of v2's link
                const int mb = smap[b], mc = smap[c];
                if (mc != 0xffff) {
                    const uint64_t at2 = (uint64_t)mb * W2 + (mc >> 6);
                    face = ((l2s ? sL2[at2] : __ldg(&L2g[at2])) >> (mc & 63)) & 1ull;
                }
            }
            const unsigned mF = __ballot_sync(kFull, face);
            if (lane == 0) cand_acc += __popc(mF);
            bool passA = false, side = false;
            float4 sphere = make_float4(0.f, 0.f, 0.f, 0.f);
            float key = 0.f;
            Ball B3{0.f, 0.f, 0.f, 0.f}, B4{0.f, 0.f, 0.f, 0.f};
            // markRealTets for every candidate, the alpha tetrahedra being
            // those with the face (v2, v3, v4): a candidate without it, or
            // outside alpha, can still refute the others (exact mode: the
            // alpha tetrahedra only)
            if (V == pac::kExact ? face : act) {
                const float4 b3 = sb[b], b4 = sb[c];
                B3 = Ball{b3.x, b3.y, b3.z, b3.w};
                B4 = Ball{b4.x, b4.y, b4.z, b4.w};
                if constexpr (V == pac::kExact)
                    passA = dec_tet<V>(B1, B2, B3, B4, A.alpha, sphere, tally);
                else
                    passA = pac::tet_alpha_g(S.grp[wib][j], B2, B3, B4, A.alpha, sphere) && face;
                {
                    // the triangle (p, v2, v3)'s normal; the side of v4
                    // and the pencil position of the orthocentre
                    const float e13x = B3.x - B1.x, e13y = B3.y - B1.y, e13z = B3.z - B1.z;
                    const float nx = e12y * e13z - e12z * e13y;
                    const float ny = e12z * e13x - e12x * e13z;
                    const float nz = e12x * e13y - e12y * e13x;
                    side = nx * (B4.x - B1.x) + ny * (B4.y - B1.y) + nz * (B4.z - B1.z) > 0.f;
                    key = nx * sphere.x + ny * sphere.y + nz * sphere.z;
                    if (!side) key = -key;
                }
            }
            const unsigned mA = __ballot_sync(kFull, passA);
            if (lane == 0) alpha_acc += __popc(mA);
            bool keep = passA;
            if constexpr (V != pac::kExact) {
                // the flat tetrahedra (orthocentre 0, LD:577-580) and
                // non-finite keys take no part
                const bool suspect = refute && act && isfinite(key) &&
                                     !(sphere.x == 0.f && sphere.y == 0.f && sphere.z == 0.f);
                const bool cand_best = suspect && passA;
                const int slot = j + (side ? 32 : 0);
                if (suspect) {
                    const uint32_t kb = __float_as_uint(key);
                    const uint32_t ok = (kb & 0x80000000u) ? ~kb : (kb | 0x80000000u);
                    atomicMin(&S.best[wib][slot], ((unsigned long long)ok << 32) | (uint32_t)c);
                }
                __syncwarp();
                if (cand_best) {
                    int y = (int)(S.best[wib][slot] & 0xffffffffull);
                    if (y == c) {
                        // the best so far of its side: the other side's
                        // best so far refutes it unless the triangle's two
                        // sides are in pencil order
                        const unsigned long long o = S.best[wib][slot ^ 32];
                        if (o != ~0ull) y = (int)(o & 0xffffffffull);
                    }
                    const float4 by = sb[y];
                    if (y != c && surely_in_window(sphere.x, sphere.y, sphere.z, by.x, by.y, by.z,
                                                   0.99f * G.step)) {
                        float pa[3] = {B1.x, B1.y, B1.z}, pb[3] = {B2.x, B2.y, B2.z};
                        float pc[3] = {B3.x, B3.y, B3.z}, pd[3] = {B4.x, B4.y, B4.z};
                        float pe[3] = {by.x, by.y, by.z};
                        const float wa = wt<V>(B1.r), wb = wt<V>(B2.r), wc = wt<V>(B3.r),
                                    wd = wt<V>(B4.r);
                        const float ori = dec_orient<V>(pa, pb, pc, pd, wa, wb, wc, wd, tally);
                        const float res = dec_insphere<V>(pa, pb, pc, pd, pe, wa, wb, wc, wd,
                                                          wt<V>(by.w), tally);
                        ktest_acc++;
                        if (ori < 0 ? (res < 0) : (res > 0)) {
                            keep = false;
                            kill_acc++;
                        }
                    }
                }
            }
            queue_append(Q, A.ctr, qr, keep,
                         make_uint4(p, v2, act ? N[b] : 0u, act ? N[c] : 0u), sphere);
        }
        __syncwarp();
    }
    __syncwarp();
}

// k_tets_enum: one warp per ball (KW = 1: balls of at most 64 upper
// neighbours, taken from a counter over the chunk [lo, hi)) or per group of
// A.unit_rows rows of a larger ball (KW = kMaxW: units from the prefix uoff of
// k_heavy_rows over [lo, hi)).  The ball's neighbours, their balls and cells
// (and, for KW = 1, its link rows) are staged in shared memory.
template <int V, int KW>
__global__ void __launch_bounds__(EnumSmem<KW>::kWarps * 32, KW == 1 ? 3 : 4)
    k_tets_enum(TetArgs A, TetQueue Q, uint64_t lo, uint64_t hi, const uint64_t *uoff) {
    // more than the 48 KB of static shared memory: dynamic, opted in by
    // enum_smem_optin()
    extern __shared__ __align__(16) unsigned char enum_smem[];
    EnumSmem<KW> &S = *reinterpret_cast<EnumSmem<KW> *>(enum_smem);
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned long long cand_acc = 0, alpha_acc = 0, kill_acc = 0, ktest_acc = 0;
    Tally tally;
    QRes qr{0, 0};
    const uint64_t u0 = KW == 1 ? lo : uoff[lo], u1 = KW == 1 ? hi : uoff[hi];
    while (true) {
        uint64_t u = 0;
        if (lane == 0) {
            // stop handing out work once the queue has overflowed: the chunk
            // is rerun smaller
            u = (*(volatile unsigned long long *)&A.ctr[C_SURV] > Q.cap)
                    ? u1
                    : u0 + atomicAdd(&A.ctr[C_NEXT], 1ull);
        }
        u = __shfl_sync(kFull, u, 0);
        if (u >= u1) break;
        uint64_t p = u;
        int a0 = 0;
        if constexpr (KW != 1) {
            uint64_t pl = lo, ph = hi;  // uoff[pl] <= u < uoff[ph]
            while (ph - pl > 1) {
                const uint64_t mid = (pl + ph) >> 1;
                if (uoff[mid] <= u) pl = mid;
                else ph = mid;
            }
            p = pl;
            a0 = (int)(u - uoff[p]) * A.unit_rows;
        }
        const uint64_t e0 = A.eoff[p];
        const int deg = (int)(A.eoff[p + 1] - e0);
        if (KW == 1 && (deg < 3 || deg > 64)) continue;  // the heavy kernel takes the larger balls
        const int W = (deg + 63) >> 6;
        const uint32_t *Ng = A.ER + e0;
        const uint64_t *Lg = A.link + A.loff[p];
        const MolGrid G = A.grids[mol_of(A.mol, p)];
        const bool refute = A.refute && G.gx <= 16384 && G.gy <= 16384 && G.gz <= 16384;
        for (int c = a0 + lane; c < deg; c += 32) {
            const uint32_t x = __ldg(&Ng[c]);
            S.sN[wib][c] = x;
            S.sb[wib][c] = __ldg(&A.at[x]);
            if constexpr (KW == 1) {
                S.sL[wib][c] = Lg[c];
                const uint64_t e2 = A.eoff[x];
                S.sE2[wib][c] = e2;
                S.sD2[wib][c] = (uint16_t)(A.eoff[x + 1] - e2);
                S.sLo[wib][c] = A.loff[x];
            }
        }
        const Ball B1 = pac::ld_ball(&A.at[p]);
        __syncwarp();
        if constexpr (KW == 1) {
            // the rows with at least two link bits, each one's v2 fetched
            // while the one before it is worked on
            const int a1 = deg - 2;
            uint64_t rows = 0;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int a = 32 * h + lane;
                const bool use = a < a1 && __popcll(S.sL[wib][a]) >= 2;
                rows |= (uint64_t)__ballot_sync(kFull, use) << (32 * h);
            }
            int buf = 0;
            if (rows) row_fetch(A, S, wib, __ffsll((long long)rows) - 1, 0);
            while (rows) {
                const int a = __ffsll((long long)rows) - 1;
                rows &= rows - 1;
                if (rows) {
                    row_fetch(A, S, wib, __ffsll((long long)rows) - 1, buf ^ 1);
                    cp_async_wait<1>();
                } else {
                    cp_async_wait<0>();
                }
                __syncwarp();
                tet_row<V, KW>(A, Q, S, wib, qr, (uint32_t)p, a, buf, RowSrc{}, RowSrc{}, deg, W,
                               S.sL[wib], B1, G, refute, cand_acc, alpha_acc, kill_acc, ktest_acc,
                               tally);
                __syncwarp();
                buf ^= 1;
            }
        } else {
            const int a1 = min(a0 + A.unit_rows, deg - 2);
            if constexpr (KW == kMaxW) {
                // each row's v2 neighbours fetched while the row before
                // is worked on (tet_row keeps the cp.async pipeline)
                RowSrc cur = a0 < a1 ? row_src(A, S.sN[wib][a0]) : RowSrc{};
                int buf = 0;
                heavy_fetch_n2(A, S, wib, cur, buf);
                for (int a = a0; a < a1; a++) {
                    const RowSrc nxt = a + 1 < a1 ? row_src(A, S.sN[wib][a + 1]) : RowSrc{};
                    tet_row<V, KW>(A, Q, S, wib, qr, (uint32_t)p, a, buf, cur, nxt, deg, W, Lg,
                                   B1, G, refute, cand_acc, alpha_acc, kill_acc, ktest_acc, tally);
                    cur = nxt;
                    buf ^= 1;
                }
                cp_async_wait<0>();
                __syncwarp();
            }
        }
        __syncwarp();
    }
    queue_close(Q, qr);
    // into the chunk's counters: the host adds them to the pass's only when
    // the chunk is accepted (an overflowing chunk is rerun smaller)
    flush_tally<V>(tally, A.ctr);
    if (lane == 0) {
        bump(A.ctr, C_CAND_Q, cand_acc);
        bump(A.ctr, C_ALPHA_Q, alpha_acc);
    }
    kill_acc = warp_sum(kill_acc);
    ktest_acc = warp_sum(ktest_acc);
    if (lane == 0) {
        bump(A.ctr, C_KILLED, kill_acc);
        bump(A.ctr, C_KTESTS, ktest_acc);
    }
}

// Exact-mode tallies and early-refutation counts of an accepted enumeration
// chunk into the pass's counters.
__global__ void k_add_tally(const unsigned long long *chunk, unsigned long long *pass) {
    const int k = threadIdx.x;
    int which = -1;
    if (k == 0) which = C_FILTER;
    else if (k == 1) which = C_FALLBACK;
    else if (k == 2) which = C_SOS_RANGE;
    else if (k == 3) which = C_KILLED;
    else if (k == 4) which = C_KTESTS;
    if (which >= 0 && chunk[which]) pass[which] += chunk[which];
}

// Work units of the heavy enumeration per ball: ceil((deg - 2) / unit_rows)
// groups of rows for a ball with more than 64 upper neighbours, 0 for the
// others.
__global__ void k_heavy_rows(uint64_t n, const uint64_t *eoff, int unit_rows, uint32_t *rows) {
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint64_t deg = eoff[p + 1] - eoff[p];
    rows[p] = deg > 64 ? (uint32_t)((deg - 2 + unit_rows - 1) / unit_rows) : 0u;
}

constexpr int kScanStep = 4;
constexpr int kScanRefill = 16;  // idle lanes that trigger a refill

// k_tets_scan: the empty-orthosphere test (checkTetsOrthosphere,
// AlphaComplexLargeData.cu:606-734) of the queued tetrahedra.  Each lane
// owns one tetrahedron at a time and tests kScanStep window balls per step; a warp
// claims a range of queue entries at a time and a lane takes the next
// unclaimed one as soon as its own is decided (claims of A.scan_claim
// entries: one counter serves every warp).  Each (tetrahedron, ball)
// decision is taken by the certified filter of certify.cuh when it can
// prove the reference's binary32 outcome, else by replaying that
// arithmetic; A.verify replays every certified decision too and counts
// disagreements (C_CERT_BAD).  Survivors are recorded and mark their faces.
template <int V>
__global__ void __launch_bounds__(256, V == pac::kExact ? 2 : 4) k_tets_scan(TetArgs A, TetQueue Q, uint64_t nq,
                                                      unsigned long long *claim) {
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1;
    unsigned long long evals = 0, oob = 0, certd = 0, bad = 0;
    Tally tally;
    uint64_t head = 0, tail = 0;  // this warp's claimed range (warp-uniform)
    bool have = false, more = true;
    uint32_t p = 0, v2 = 0, v3 = 0, v4 = 0;
    float ax = 0, ay = 0, az = 0, bx = 0, by = 0, bz = 0, cx = 0, cy = 0, cz = 0, dx = 0, dy = 0,
          dz = 0, wa = 0, wb = 0, wc = 0, wd = 0, orientation = 0;
    pac::cert::Insphere ct{};
    int gX = 0, gY = 0, gZ = 0, q = 0;
    uint32_t e = 0, end = 0;
    bool zero = false;
    const MolGrid *G = A.grids;
    while (true) {
        // claim: idle lanes take the next entries of the warp's range
        // idle lanes take new tetrahedra together, once enough of them
        // wait (or none works): the setup then runs for many lanes at once
        unsigned want = __ballot_sync(kFull, !have);
        if (!(__popc(want) >= kScanRefill || want == kFull)) want = 0u;
        if (want && head >= tail && more) {
            uint64_t b = 0;
            if (lane == 0) b = atomicAdd(claim, (unsigned long long)A.scan_claim);
            b = __shfl_sync(kFull, b, 0);
            head = b;
            tail = min(nq, b + (uint64_t)A.scan_claim);
            if (head >= tail) more = false;
            for (uint64_t k = head + 4 * lane; k < tail; k += 128) {
                asm volatile("prefetch.global.L2 [%0];" ::"l"(Q.vid + k));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(Q.sph + k));
            }
        }
        if (want && head < tail) {
            const int r = __popc(want & lt_mask);
            if (!have && head + r < tail) {
                const uint64_t idx = head + r;
                const uint4 vv = Q.vid[idx];
                if (vv.x != kNoTet) {
                    const float4 sph = Q.sph[idx];
                    p = vv.x, v2 = vv.y, v3 = vv.z, v4 = vv.w;
                    G = A.grids + mol_of(A.mol, p);
                    const Ball a1 = pac::ld_ball(&A.at[p]), a2 = pac::ld_ball(&A.at[v2]),
                               a3 = pac::ld_ball(&A.at[v3]), a4 = pac::ld_ball(&A.at[v4]);
                    ax = a1.x, ay = a1.y, az = a1.z, wa = wt<V>(a1.r);
                    bx = a2.x, by = a2.y, bz = a2.z, wb = wt<V>(a2.r);
                    cx = a3.x, cy = a3.y, cz = a3.z, wc = wt<V>(a3.r);
                    dx = a4.x, dy = a4.y, dz = a4.z, wd = wt<V>(a4.r);
                    {
                        const float pa[3] = {ax, ay, az}, pb[3] = {bx, by, bz}, pc[3] = {cx, cy, cz},
                                    pd[3] = {dx, dy, dz};
                        orientation = dec_orient<V>(pa, pb, pc, pd, wa, wb, wc, wd, tally);
                    }
                    if constexpr (V != pac::kExact)
                        ct = pac::cert::setup(ax, ay, az, wa, bx, by, bz, wb, cx, cy, cz, wc, dx, dy,
                                              dz, wd, orientation, sph.x, sph.y, sph.z, G->wmax);
                    const int4 cl = window_cell(*G, sph.x, sph.y, sph.z);
                    gX = cl.x, gY = cl.y, gZ = cl.z;
                    q = 0;
                    zero = false;
                    window_centre(*G, A.cellbeg, cl, e, end, oob);
                    have = true;
                }
            }
            head = min(tail, head + (uint64_t)__popc(want));
        }
        if (!__any_sync(kFull, have)) {
            if (!more) break;
            continue;
        }
        if (!have) continue;
        if (e < end) {
            // kScanStep window balls per step: their loads overlap, and the
            // warp-wide bookkeeping above runs once per step
            const uint32_t cnt = min(end - e, (uint32_t)kScanStep);
            Ball bq[kScanStep];
#pragma unroll
            for (int t = 0; t < kScanStep; t++)
                bq[t] = pac::ld_ball(&A.at[e + min((uint32_t)t, cnt - 1)]);
            const uint32_t x0 = e;
            e += cnt;
            bool viol = false;
#pragma unroll
            for (int t = 0; t < kScanStep; t++) {
                const uint32_t x = x0 + t;
                const Ball bb = bq[t];
                if ((uint32_t)t >= cnt || viol || x == p || x == v2 || x == v3 || x == v4) continue;
                const float we = wt<V>(bb.r);
                int dec = -1;
                if constexpr (V != pac::kExact) dec = pac::cert::test(ct, bb.x, bb.y, bb.z, we);
                evals++;
                if (dec >= 0) certd++;
                if (dec < 0 || A.verify) {
                    const float pa[3] = {ax, ay, az}, pb[3] = {bx, by, bz}, pc[3] = {cx, cy, cz},
                                pd[3] = {dx, dy, dz}, pe[3] = {bb.x, bb.y, bb.z};
                    const float res =
                        dec_insphere<V>(pa, pb, pc, pd, pe, wa, wb, wc, wd, we, tally);
                    const int rdec = (orientation < 0 ? (res < 0) : (res > 0)) ? 1 : 0;
                    if (dec >= 0 && dec != rdec) bad++;
                    if (dec < 0) {
                        dec = rdec;
                        if (res == 0) zero = true;
                    }
                }
                viol = dec == 1;
            }
            if (viol) have = false;
            continue;
        }
        bool found = false;
        while (q < kWindowParts && !found) found = window_part(*G, A.cellbeg, gX, gY, gZ, q++, e, end);
        if (!found) {
            emit_survivor(A.eoff, A.ER, A.loff, A.faces, A.surv, A.surv_cap, A.pend, A.pend_cap,
                          A.ctr, A.tcount, p, v2, v3, v4, zero);
            have = false;
        }
    }
    evals = warp_sum(evals);
    oob = warp_sum(oob);
    certd = warp_sum(certd);
    bad = warp_sum(bad);
    flush_tally<V>(tally, A.ctr);
    if (lane == 0) {
        bump(A.ctr, C_INSPHERE, evals);
        bump(A.ctr, C_OOB, oob);
        bump(A.ctr, C_CERT, certd);
        bump(A.ctr, C_CERT_BAD, bad);
    }
}

// Tetrahedra whose window holds an insphere value of exactly 0: the test
// again, with the reference's simulation of simplicity for those balls
// (AlphaComplexLargeData.cu:645-652, 659-667).
template <int V>
__global__ void k_sos_resolve(TetArgs A, uint64_t npend) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npend) return;
    uint2 pk = A.pend[t];
    uint64_t p = pk.x;
    int a = pk.y & 0xff, b = (pk.y >> 8) & 0xff, c = (pk.y >> 16) & 0xff;
    const uint64_t e0 = A.eoff[p];
    const int deg = (int)(A.eoff[p + 1] - e0);
    const int W = (deg + 63) >> 6;
    const uint32_t *N = A.ER + e0;
    uint32_t v[4] = {(uint32_t)p, N[a], N[b], N[c]};
    Ball B[4];
    for (int k = 0; k < 4; k++) B[k] = pac::ld_ball(&A.at[v[k]]);
    Tally tally;
    float4 sphere;
    dec_tet<V>(B[0], B[1], B[2], B[3], A.alpha, sphere, tally);
    const MolGrid G = A.grids[mol_of(A.mol, p)];
    float pts[5][3], ws[5];
    int idx[5];
    for (int k = 0; k < 4; k++) {
        pts[k][0] = B[k].x;
        pts[k][1] = B[k].y;
        pts[k][2] = B[k].z;
        ws[k] = wt<V>(B[k].r);
        idx[k] = (int)A.orig[v[k]] + 1;
    }
    float orientation = dec_orient<V>(pts[0], pts[1], pts[2], pts[3], ws[0], ws[1], ws[2], ws[3],
                                      tally);
    int gridX = pac::cell_coord(sphere.x, G.minx, G.step);
    int gridY = pac::cell_coord(sphere.y, G.miny, G.step);
    int gridZ = pac::cell_coord(sphere.z, G.minz, G.step);
    int cc = lin3(gridX, gridY, gridZ, G.gx, G.gy);
    bool viol = false;
    for (int q = 0; q < 27 && !viol; q++) {
        uint32_t beg, end;
        if (q == 0) {
            if (cc < 0 || (uint64_t)cc >= G.ncell) continue;
            beg = A.cellbeg[G.cell_base + cc];
            end = A.cellbeg[G.cell_base + cc + 1];
        } else {
            int r = q - 1 + (q >= 14 ? 1 : 0);
            int i = r / 9 - 1, j = (r / 3) % 3 - 1, k = r % 3 - 1;
            int zz = (int)((unsigned)gridZ + (unsigned)i), yy = (int)((unsigned)gridY + (unsigned)j),
                xx = (int)((unsigned)gridX + (unsigned)k);
            if ((zz >= G.gz) || (yy >= G.gy) || (xx >= G.gx)) continue;
            if ((zz < 0) || (yy < 0) || (xx < 0)) continue;
            uint64_t gc = G.cell_base + (uint64_t)lin3(xx, yy, zz, G.gx, G.gy);
            beg = A.cellbeg[gc];
            end = A.cellbeg[gc + 1];
        }
        for (uint32_t e = beg; e < end && !viol; e++) {
            if (e == v[0] || e == v[1] || e == v[2] || e == v[3]) continue;
            const Ball atom = pac::ld_ball(&A.at[e]);
            pts[4][0] = atom.x;
            pts[4][1] = atom.y;
            pts[4][2] = atom.z;
            ws[4] = wt<V>(atom.r);
            float result = dec_insphere<V>(pts[0], pts[1], pts[2], pts[3], pts[4], ws[0], ws[1],
                                           ws[2], ws[3], ws[4], tally);
            if (result == 0) {
                idx[4] = (int)A.orig[e] + 1;
                int status = 0;
                result = (float)pac::sos_orientation(pts, ws, idx, &status, V == pac::kExact);
                atomicAdd(&A.ctr[C_SOS], 1ull);
                if (status == 1) atomicAdd(&A.ctr[C_SOS_RANGE], 1ull);
            }
            viol = orientation < 0 ? (result < 0) : (result > 0);
        }
    }
    flush_tally_thread<V>(tally, A.ctr);
    if (viol) return;
    unsigned long long q = atomicAdd(&A.ctr[C_SURV], 1ull);
    if (q < A.surv_cap) A.surv[q] = pk;
    atomicAdd(&A.tcount[p], 1u);
    const uint64_t lp = A.loff[p];
    mark_face(A.faces, lp, W, a, b);
    mark_face(A.faces, lp, W, a, c);
    mark_face(A.faces, lp, W, b, c);
    const uint32_t v2 = v[1];
    const uint64_t e2 = A.eoff[v2];
    const int deg2 = (int)(A.eoff[v2 + 1] - e2);
    const int mb = lbound(A.ER + e2, deg2, v[2]), mc = lbound(A.ER + e2, deg2, v[3]);
    mark_face(A.faces, A.loff[v2], (deg2 + 63) >> 6, mb, mc);
}

// Survivors to per-ball rows: scatter, then order each ball's rows by
// (a, b, c) -- the order in which the reference enumerates them.
__global__ void k_tet_scatter(const uint2 *surv, uint64_t ns, const uint64_t *toff,
                              uint32_t *cursor, uint32_t *keys, uint64_t p_lo, uint64_t p_hi) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ns) return;
    uint2 s = surv[t];
    if (s.x < p_lo || s.x >= p_hi) return;  // a slab's halo: not this pass's output
    keys[toff[s.x] + atomicAdd(&cursor[s.x], 1u)] = s.y;
}
__global__ void k_tet_sort_emit(uint64_t n, const uint64_t *toff, uint32_t *keys,
                                const uint64_t *eoff, const uint32_t *ER, const uint32_t *orig,
                                uint32_t *out) {
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    uint64_t b = toff[p], e = toff[p + 1];
    for (uint64_t i = b + 1; i < e; i++) {
        uint32_t v = keys[i];
        uint32_t vk = ((v & 0xff) << 16) | (v & 0xff00) | ((v >> 16) & 0xff);
        uint64_t j = i;
        while (j > b) {
            uint32_t u = keys[j - 1];
            uint32_t uk = ((u & 0xff) << 16) | (u & 0xff00) | ((u >> 16) & 0xff);
            if (uk <= vk) break;
            keys[j] = u;
            j--;
        }
        keys[j] = v;
    }
    const uint32_t *N = ER + eoff[p];
    const uint32_t o1 = orig[p];
    for (uint64_t i = b; i < e; i++) {
        uint32_t k = keys[i];
        uint4 t = make_uint4(o1, orig[N[k & 0xff]], orig[N[(k >> 8) & 0xff]],
                             orig[N[(k >> 16) & 0xff]]);
        *(uint4 *)&out[4 * i] = t;
    }
}
__global__ void k_map4(uint64_t nq, const uint32_t *orig, uint32_t *tets) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nq) return;
    uint4 v = *(uint4 *)&tets[4 * t];
    *(uint4 *)&tets[4 * t] = make_uint4(orig[v.x], orig[v.y], orig[v.z], orig[v.w]);
}

// ------------------------------------------------------------------ attachment
// Final triangles of ball v1: tetrahedron faces, plus the alpha triangles
// that are not faces and whose orthosphere no other ball of the 27-cell
// window reaches (checkDanglingTris, AlphaComplexLargeData.cu:798-872).
// Work stealing: one warp per ball v1, balls handed out from a counter.  The alpha triangles
// of v1 that are not tetrahedron faces are queued in shared memory row by
// row; each lane takes one, recomputes its orthosphere (markRealTriangles)
// and tests one window ball per step (checkDanglingTris,
// AlphaComplexLargeData.cu:798-872), taking the next queued triangle as soon
// as its own is decided.  An unattached triangle sets its bit in `faces`.
// Then the warp counts v1's final triangles and marks their edges.
constexpr int kTQCap = 256;
constexpr int kTARefill = 24;  // idle lanes that trigger a refill

template <int V>
__global__ void __launch_bounds__(256, 4) k_tri_attach(uint64_t p_lo, uint64_t n,
                                                       const float4 *__restrict__ at,
                                                       const uint64_t *__restrict__ eoff,
                                                       const uint32_t *__restrict__ ER,
                                                       const uint64_t *__restrict__ loff,
                                                       const uint64_t *__restrict__ link,
                                                       uint64_t *faces, uint32_t *tricount,
                                                       uint8_t *eflag, const uint32_t *cellbeg,
                                                       const uint32_t *mol, const MolGrid *grids,
                                                       float alpha, unsigned long long *ctr) {
    __shared__ uint16_t qa[8][kTQCap], qb[8][kTQCap];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1;
    unsigned long long oob = 0;
    Tally tally;
    while (true) {
        uint64_t p = 0;
        if (lane == 0) p = p_lo + atomicAdd(&ctr[C_NEXT], 1ull);
        p = __shfl_sync(kFull, p, 0);
        if (p >= n) break;
        const uint64_t e0 = eoff[p];
        const int deg = (int)(eoff[p + 1] - e0);
        uint32_t count = 0;
        if (deg >= 2) {
            const int W = (deg + 63) >> 6;
            const uint32_t *N = ER + e0;
            const uint64_t lp = loff[p];
            const Ball A0 = pac::ld_ball(&at[p]);
            const MolGrid *G = grids + mol_of(mol, p);
            int row = 0;       // next row to queue (warp-uniform)
            uint64_t rbits[kMaxW];  // unqueued candidate bits of `row`
            bool rloaded = false;
            // lane state
            bool have = false;
            int ta = 0, tb = 0;
            uint32_t v1 = 0, v2 = 0;
            float px = 0, py = 0, pz = 0, cur = 0;
            int gX = 0, gY = 0, gZ = 0, q = 0;
            uint32_t e = 0, end = 0;
            int qn = 0, head = 0;  // shared queue (warp-uniform)
            while (true) {
                // refill the queue from the remaining rows
                if (head >= qn) {
                    qn = 0;
                    head = 0;
                    while (row < deg - 1 && qn < kTQCap - 64) {
                        if (!rloaded) {
#pragma unroll
                            for (int w = 0; w < kMaxW; w++)
                                rbits[w] = w < W ? (link[lp + (uint64_t)row * W + w] &
                                                    ~faces[lp + (uint64_t)row * W + w])
                                                 : 0;
                            rloaded = true;
                        }
                        int nc = 0;
#pragma unroll
                        for (int w = 0; w < kMaxW; w++) nc += __popcll(rbits[w]);
                        int take = min(nc, kTQCap - qn);
                        for (int k0 = 0; k0 < take; k0 += 32) {
                            int k = k0 + lane;
                            if (k < take) {
                                qa[wib][qn + k] = (uint16_t)row;
                                qb[wib][qn + k] = (uint16_t)select_bit(rbits, W, k);
                            }
                        }
                        qn += take;
                        if (take == nc) {
                            row++;
                            rloaded = false;
                        } else {
                            // drop the queued bits from the row, keep the rest
                            for (int k = 0; k < take; k++) {
                                int b = select_bit(rbits, W, 0);
                                rbits[b >> 6] &= ~(1ull << (b & 63));
                            }
                        }
                    }
                    __syncwarp();
                }
                // idle lanes take new triangles together, once enough of
                // them wait (or none works): the setup runs for many lanes
                // at a time instead of for a few in every step
                unsigned want = __ballot_sync(kFull, !have);
                if (want && head < qn && (__popc(want) >= kTARefill || want == kFull)) {
                    int r = __popc(want & lt_mask);
                    if (!have && head + r < qn) {
                        ta = qa[wib][head + r];
                        tb = qb[wib][head + r];
                        v1 = N[ta];
                        v2 = N[tb];
                        const float4 p1 =
                            tri_sphere<V>(A0, pac::ld_ball(&at[v1]), pac::ld_ball(&at[v2]), alpha);
                        px = p1.x;
                        py = p1.y;
                        pz = p1.z;
                        cur = p1.w;
                        gX = pac::cell_coord(p1.x, G->minx, G->step);
                        gY = pac::cell_coord(p1.y, G->miny, G->step);
                        gZ = pac::cell_coord(p1.z, G->minz, G->step);
                        q = 0;
                        window_centre(*G, cellbeg, make_int4(gX, gY, gZ, lin3(gX, gY, gZ, G->gx, G->gy)),
                                      e, end, oob);
                        have = true;
                    }
                    head = min(qn, head + __popc(want));
                }
                if (!__any_sync(kFull, have)) {
                    if (head >= qn && row >= deg - 1) break;
                    continue;
                }
                if (!have) continue;
                if (e < end) {
                    if constexpr (V != pac::kExact) {
                        // two window balls per step (independent loads)
                        const uint32_t x0 = e, x1 = (e + 1 < end) ? e + 1 : e;
                        e = x1 + 1;
                        const bool ok0 = !(x0 == (uint32_t)p || x0 == v1 || x0 == v2);
                        const bool ok1 = x1 != x0 && !(x1 == (uint32_t)p || x1 == v1 || x1 == v2);
                        const Ball b0 = pac::ld_ball(&at[x0]), b1 = pac::ld_ball(&at[x1]);
                        const bool t0 = pac::attached(b0, px, py, pz, cur);
                        const bool t1 = pac::attached(b1, px, py, pz, cur);
                        if ((ok0 && t0) || (ok1 && t1)) have = false;
                    } else {
                        uint32_t x = e++;
                        if (x == (uint32_t)p || x == v1 || x == v2) continue;
                        if (dec_tri_attached<V>(A0, at, v1, v2, pac::ld_ball(&at[x]), px, py, pz,
                                                cur, tally))
                            have = false;
                    }
                    continue;
                }
                bool found = false;
                while (q < kWindowParts && !found)
                    found = window_part(*G, cellbeg, gX, gY, gZ, q++, e, end);
                if (!found) {
                    atomicOr((unsigned long long *)&faces[lp + (uint64_t)ta * W + (tb >> 6)],
                             1ull << (tb & 63));
                    have = false;
                }
            }
            __syncwarp();
            __threadfence_block();
            // count the final triangles and mark their edges: a lane per
            // row, 32 rows at a time
            for (int a0 = 0; a0 < deg - 1; a0 += 32) {
                const int a = a0 + lane;
                uint64_t fin[kMaxW];
                int nf = 0;
#pragma unroll
                for (int w = 0; w < kMaxW; w++) {
                    fin[w] = (a < deg - 1 && w < W) ? faces[lp + (uint64_t)a * W + w] : 0;
                    nf += __popcll(fin[w]);
                }
                count += (uint32_t)warp_sum((unsigned long long)nf);
                if (!nf) continue;
                eflag[e0 + a] = 1;
                const uint32_t va = N[a];
                const uint64_t e1 = eoff[va];
                const int deg1 = (int)(eoff[va + 1] - e1);
#pragma unroll
                for (int w = 0; w < kMaxW; w++) {
                    uint64_t bits = fin[w];
                    while (bits) {
                        const int b = w * 64 + __ffsll((long long)bits) - 1;
                        bits &= bits - 1;
                        eflag[e0 + b] = 1;
                        const uint32_t vb = N[b];
                        const int pos = lbound(ER + e1, deg1, vb);
                        if (pos < deg1 && ER[e1 + pos] == vb) eflag[e1 + pos] = 1;
                    }
                }
            }
        }
        if (lane == 0) tricount[p] = count;
    }
    oob = warp_sum(oob);
    flush_tally<V>(tally, ctr);
    if (lane == 0) bump(ctr, C_OOB, oob);
}

// Final edges: edges of final triangles, plus the alpha edges whose radical
// foot no other ball reaches (checkDanglingEdges, AlphaComplexLargeData.cu:924-1011).
template <int V>
__global__ void __launch_bounds__(256) k_edge_final(uint64_t p_lo, uint64_t n,
                                                    const float4 *__restrict__ at,
                                                    const uint64_t *__restrict__ eoff,
                                                    const uint32_t *__restrict__ ER,
                                                    uint8_t *eflag, const uint32_t *cellbeg,
                                                    const uint32_t *mol, const MolGrid *grids,
                                                    unsigned long long *ctr) {
    const int lane = threadIdx.x & 31;
    unsigned long long oob = 0;
    Tally tally;
    // balls handed out by a counter (persistent warps)
    for (;;) {
        uint64_t p = 0;
        if (lane == 0) p = p_lo + atomicAdd(&ctr[C_NEXT], 1ull);
        p = __shfl_sync(kFull, p, 0);
        if (p >= n) break;
        const uint64_t e0 = eoff[p];
        const int deg = (int)(eoff[p + 1] - e0);
        if (!deg) continue;
        const Ball a1 = pac::ld_ball(&at[p]);
        const MolGrid G = grids[mol_of(mol, p)];
        for (int k = lane; k < deg; k += 32) {
            if (eflag[e0 + k]) continue;
            const uint32_t v2 = ER[e0 + k];
            float px, py, pz, currentDist;
            const Ball a2 = pac::ld_ball(&at[v2]);
            edge_sphere<V>(a1, a2, px, py, pz, currentDist);
            int gridX = pac::cell_coord(px, G.minx, G.step);
            int gridY = pac::cell_coord(py, G.miny, G.step);
            int gridZ = pac::cell_coord(pz, G.minz, G.step);
            int cc = lin3(gridX, gridY, gridZ, G.gx, G.gy);
            bool att = false;
            for (int q = 0; q < 27 && !att; q++) {
                uint32_t beg, end;
                if (q == 0) {
                    if (cc < 0 || (uint64_t)cc >= G.ncell) {
                        oob++;
                        continue;
                    }
                    beg = cellbeg[G.cell_base + cc];
                    end = cellbeg[G.cell_base + cc + 1];
                } else {
                    int r = q - 1 + (q >= 14 ? 1 : 0);
                    int i = r / 9 - 1, j = (r / 3) % 3 - 1, kk = r % 3 - 1;
                    int zz = (int)((unsigned)gridZ + (unsigned)i),
                        yy = (int)((unsigned)gridY + (unsigned)j),
                        xx = (int)((unsigned)gridX + (unsigned)kk);
                    if ((zz >= G.gz) || (yy >= G.gy) || (xx >= G.gx)) continue;
                    if ((zz < 0) || (yy < 0) || (xx < 0)) continue;
                    uint64_t gc = G.cell_base + (uint64_t)lin3(xx, yy, zz, G.gx, G.gy);
                    beg = cellbeg[gc];
                    end = cellbeg[gc + 1];
                }
                for (uint32_t e = beg; e < end; e++) {
                    if (e == p || e == v2) continue;
                    if (dec_edge_attached<V>(a1, a2, pac::ld_ball(&at[e]), px, py, pz,
                                             currentDist, tally)) {
                        att = true;
                        break;
                    }
                }
            }
            if (!att) eflag[e0 + k] = 1;
        }
    }
    oob = warp_sum(oob);
    flush_tally<V>(tally, ctr);
    if (lane == 0) bump(ctr, C_OOB, oob);
}

// ------------------------------------------------------------------ emission
__global__ void k_emit_edges(uint64_t n, const uint64_t *eoff, const uint32_t *ER,
                             const uint8_t *eflag, const uint64_t *epos, const uint32_t *orig,
                             uint32_t *out) {
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    uint32_t o = orig[p];
    for (uint64_t k = eoff[p]; k < eoff[p + 1]; k++)
        if (eflag[k]) {
            uint64_t q = epos[k];
            out[2 * q] = o;
            out[2 * q + 1] = orig[ER[k]];
        }
}
__global__ void __launch_bounds__(256) k_emit_tris(uint64_t p_lo, uint64_t n, const uint64_t *eoff,
                                                   const uint32_t *ER, const uint64_t *loff,
                                                   const uint64_t *faces, const uint64_t *tpos,
                                                   const uint32_t *orig, uint32_t *out) {
    const int lane = threadIdx.x & 31;
    uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t p = p_lo + warp; p < n; p += nwarps) {
        const int deg = (int)(eoff[p + 1] - eoff[p]);
        if (deg < 2) continue;
        const int W = (deg + 63) >> 6;
        const uint32_t *N = ER + eoff[p];
        const uint32_t o0 = orig[p];
        const uint64_t lp = loff[p];
        uint64_t q = tpos[p];
        // a lane per row, 32 rows at a time; rows in order, b ascending
        // within a row
        for (int a0 = 0; a0 < deg - 1; a0 += 32) {
            const int a = a0 + lane;
            uint64_t f[kMaxW];
            int nf = 0;
#pragma unroll
            for (int w = 0; w < kMaxW; w++) {
                f[w] = (a < deg - 1 && w < W) ? faces[lp + (uint64_t)a * W + w] : 0;
                nf += __popcll(f[w]);
            }
            int incl = nf;
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += v;
            }
            const int total = __shfl_sync(kFull, incl, 31);
            if (nf) {
                const uint32_t o1 = orig[N[a]];
                uint64_t at = q + (uint64_t)(incl - nf);
#pragma unroll
                for (int w = 0; w < kMaxW; w++) {
                    uint64_t bits = f[w];
                    while (bits) {
                        const int b = w * 64 + __ffsll((long long)bits) - 1;
                        bits &= bits - 1;
                        out[3 * at] = o0;
                        out[3 * at + 1] = o1;
                        out[3 * at + 2] = orig[N[b]];
                        at++;
                    }
                }
            }
            q += (uint64_t)total;
        }
    }
}
// first output row of every molecule (and the totals at m = n_mol)
__global__ void k_mol_rows(uint32_t n_mol, const uint64_t *ball_off, uint64_t n,
                           const uint64_t *eoff, const uint64_t *epos, const uint64_t *tpos,
                           const uint64_t *toff, uint64_t *rows) {
    uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m > n_mol) return;
    uint64_t b = m < n_mol ? ball_off[m] : n;
    rows[m] = epos[eoff[b]];
    rows[(n_mol + 1) + m] = tpos[b];
    rows[2 * (n_mol + 1) + m] = toff[b];
}

// ------------------------------------------------------------------ host
// The enumeration kernels' shared memory exceeds the static 48 KB: allow it
// (once per device and flavour; the attribute belongs to the kernel).
template <int V>
static int enum_smem_optin(pac::Ctx &ctx) {
    static bool done[64] = {};
    if (ctx.device >= 0 && ctx.device < 64 && done[ctx.device]) return PAC_OK;
    CK(cudaFuncSetAttribute(k_tets_enum<V, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)sizeof(EnumSmem<1>)));
    CK(cudaFuncSetAttribute(k_tets_enum<V, kMaxW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)sizeof(EnumSmem<kMaxW>)));
    if (ctx.device >= 0 && ctx.device < 64) done[ctx.device] = true;
    return PAC_OK;
}

struct Timer {
    pac::Ctx &ctx;
    int i = 0;
    explicit Timer(pac::Ctx &c) : ctx(c) {}
    void mark() {  // events 0..13 (14 and 15 time the orthosphere test)
        if (i < 14) cudaEventRecord(ctx.ev[i++], ctx.stream);
    }
    double ms(int a, int b) {
        float f = 0;
        if (a < i && b < i) cudaEventElapsedTime(&f, ctx.ev[a], ctx.ev[b]);
        return f;
    }
};

static unsigned blocks_for(uint64_t n, unsigned threads) {
    uint64_t b = (n + threads - 1) / threads;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(b, 0x7fffffffu));
}
static unsigned warp_blocks(uint64_t items) {
    // 8 warps per block, grid-stride: enough blocks to fill 148 SMs many times
    uint64_t b = (items + 7) / 8;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(b, 148ull * 64));
}

template <int V>
static int run_pass_v(pac::Ctx &ctx, const pac::PipelineConfig &cfg, const pac::PassInput &in,
                      pac::PassOutput &out, pac_stats *st) {
    cudaStream_t s = ctx.stream;
    pac::Arena &ar = ctx.arena;
    const uint64_t n = in.n;
    const uint32_t nm = in.n_mol;
    Timer tm(ctx);
    tm.mark();  // 0

    unsigned long long *ctr = ar.alloc_n<unsigned long long>(C_NCOUNTERS);
    int *mm = ar.alloc_n<int>(8 * (size_t)nm);
    MolGrid *grids = ar.alloc_n<MolGrid>(nm);
    uint64_t *ncell_d = ar.alloc_n<uint64_t>(nm);
    uint64_t *d_off = ar.alloc_n<uint64_t>(nm + 1);
    uint32_t *mol = nullptr;
    if (!ctr || !mm || !grids || !ncell_d || !d_off) return PAC_ERR_OOM;
    CK(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long) * C_NCOUNTERS, s));
    {
        std::vector<int> init(8 * (size_t)nm);
        for (uint32_t m = 0; m < nm; m++)
            for (int q = 0; q < 4; q++) {
                init[8 * m + q] = 0x7fffffff;
                init[8 * m + 4 + q] = (int)0x80000000;
            }
        CK(cudaMemcpyAsync(mm, init.data(), sizeof(int) * init.size(), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(d_off, in.h_offsets, sizeof(uint64_t) * (nm + 1),
                           cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));  // `init` leaves scope
    }
    if (nm > 1) {
        mol = ar.alloc_n<uint32_t>(n);
        if (!mol) return PAC_ERR_OOM;
        k_mol_ids<<<nm, 256, 0, s>>>(d_off, nm, mol);
        LAUNCH_CHECK(ctx);
    }
    k_bbox<<<blocks_for(n, 256), 256, 0, s>>>(in.d_balls, n, mol, mm);
    LAUNCH_CHECK(ctx);
    k_grid<<<blocks_for(nm, 128), 128, 0, s>>>(mm, nm, in.sol, in.alpha, grids, ncell_d);
    LAUNCH_CHECK(ctx);
    std::vector<MolGrid> hg(nm);
    CK(cudaMemcpyAsync(hg.data(), grids, sizeof(MolGrid) * nm, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    uint64_t total_cells = 0;
    for (uint32_t m = 0; m < nm; m++) {
        if (hg[m].gx <= 0 || hg[m].gy <= 0 || hg[m].gz <= 0 || hg[m].ncell > 0x7fffffffull)
            return pac::set_error(PAC_ERR_CAPACITY,
                                  "grid of molecule " + std::to_string(m) +
                                      " exceeds the reference's int cell index range");
        hg[m].cell_base = total_cells;
        hg[m].atom_base = in.h_offsets[m];
        total_cells += hg[m].ncell;
    }
    if (total_cells >= 0xffffffffull)
        return pac::set_error(PAC_ERR_CAPACITY, "more than 2^32 cells in one pass");
    CK(cudaMemcpyAsync(grids, hg.data(), sizeof(MolGrid) * nm, cudaMemcpyHostToDevice, s));

    // ---- binning
    uint32_t *gcell = ar.alloc_n<uint32_t>(n), *slot = ar.alloc_n<uint32_t>(n);
    uint32_t *cellcnt = ar.alloc_n<uint32_t>(total_cells);
    uint32_t *cellbeg = ar.alloc_n<uint32_t>(total_cells + 1);
    uint32_t *perm = ar.alloc_n<uint32_t>(n);
    float4 *at = ar.alloc_n<float4>(n);
    uint32_t *orig = ar.alloc_n<uint32_t>(n), *cellof = ar.alloc_n<uint32_t>(n);
    if (!gcell || !slot || !cellcnt || !cellbeg || !perm || !at || !orig || !cellof)
        return PAC_ERR_OOM;
    CK(cudaMemsetAsync(cellcnt, 0, sizeof(uint32_t) * total_cells, s));
    k_cellkey<<<blocks_for(n, 256), 256, 0, s>>>(in.d_balls, n, mol, grids, gcell, slot, cellcnt);
    LAUNCH_CHECK(ctx);
    int rc = exclusive_scan(ctx, cellcnt, total_cells, cellbeg);
    if (rc) return rc;
    k_scatter<<<blocks_for(n, 256), 256, 0, s>>>(n, gcell, slot, cellbeg, perm);
    LAUNCH_CHECK(ctx);
    k_cellsort<<<blocks_for(total_cells, 256), 256, 0, s>>>(total_cells, cellbeg, perm);
    LAUNCH_CHECK(ctx);
    k_gather<<<blocks_for(n, 256), 256, 0, s>>>(n, perm, in.d_balls, in.sol, gcell, mol, grids,
                                                at, orig, cellof);
    LAUNCH_CHECK(ctx);
    tm.mark();  // 1

    // ---- a slab of one molecule (cfg.slab_world > 1): this pass emits the
    // simplices whose smallest vertex in cell order lies in [own_lo, own_hi)
    // -- balls n r / world .. n (r + 1) / world rounded down to cell starts --
    // and computes the tetrahedron and triangle stages from work_lo, two cell
    // layers lower: every vertex of an alpha simplex lies in a cell adjacent
    // to its smallest vertex's (alpha edges join adjacent cells), so the
    // tetrahedra whose faces decide the owned triangles, and the triangles
    // whose edges decide the owned edges, all start at or above work_lo.
    uint64_t own_lo = 0, own_hi = n, work_lo = 0;
    if (cfg.slab_world > 1) {
        if (nm != 1)
            return pac::set_error(PAC_ERR_INVALID_ARG, "a slab pass takes one molecule");
        if (cfg.tet_mode != PAC_TETS_AS_WRITTEN)
            return pac::set_error(PAC_ERR_INVALID_ARG, "a slab pass applies the orthosphere test");
        if (cfg.slab_rank < 0 || cfg.slab_rank >= cfg.slab_world)
            return pac::set_error(PAC_ERR_INVALID_ARG, "slab rank out of range");
        auto cell_start = [&](uint64_t ball, uint64_t &out) -> int {
            if (ball >= n) {
                out = n;
                return PAC_OK;
            }
            uint32_t c = 0, b = 0;
            CK(cudaMemcpyAsync(&c, cellof + ball, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            CK(cudaMemcpyAsync(&b, cellbeg + c, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            out = b;
            return PAC_OK;
        };
        const uint64_t r = (uint64_t)cfg.slab_rank, w = (uint64_t)cfg.slab_world;
        if (r > 0 && (rc = cell_start(n * r / w, own_lo))) return rc;
        if (r + 1 < w && (rc = cell_start(n * (r + 1) / w, own_hi))) return rc;
        if (own_hi < own_lo) own_hi = own_lo;
        if (own_lo > 0) {
            uint32_t c = 0, b = 0;
            CK(cudaMemcpyAsync(&c, cellof + own_lo, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            const uint64_t layer = (uint64_t)hg[0].gx * hg[0].gy + hg[0].gx + 1;
            const uint64_t c0 = c > 2 * layer ? c - 2 * layer : 0;
            CK(cudaMemcpyAsync(&b, cellbeg + c0, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            work_lo = b;
        }
    }

    // ---- alpha edges
    uint32_t *ecount = ar.alloc_n<uint32_t>(n);
    uint64_t *eoff = ar.alloc_n<uint64_t>(n + 1);
    if (!ecount || !eoff) return PAC_ERR_OOM;
    k_edges<V, false><<<warp_blocks(n), 256, 0, s>>>(n, at, cellof, cellbeg, mol, grids, in.alpha,
                                                     ecount, nullptr, nullptr, ctr);
    LAUNCH_CHECK(ctx);
    rc = exclusive_scan(ctx, ecount, n, eoff);
    if (rc) return rc;
    uint64_t nE = 0;
    CK(cudaMemcpyAsync(&nE, eoff + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    uint32_t *ER = ar.alloc_n<uint32_t>(nE);
    uint8_t *eflag = ar.alloc_n<uint8_t>(nE);
    uint64_t *lsize = ar.alloc_n<uint64_t>(n), *loff = ar.alloc_n<uint64_t>(n + 1);
    if (!ER || !eflag || !lsize || !loff) return PAC_ERR_OOM;
    k_edges<V, true><<<warp_blocks(n), 256, 0, s>>>(n, at, cellof, cellbeg, mol, grids, in.alpha,
                                                    nullptr, eoff, ER, ctr);
    LAUNCH_CHECK(ctx);
    CK(cudaMemsetAsync(eflag, 0, nE ? nE : 1, s));
    k_link_size<<<blocks_for(n, 256), 256, 0, s>>>(n, eoff, lsize, ctr);
    LAUNCH_CHECK(ctx);
    rc = exclusive_scan(ctx, lsize, n, loff);
    if (rc) return rc;
    uint64_t nL = 0;
    unsigned long long maxdeg = 0;
    CK(cudaMemcpyAsync(&nL, loff + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&maxdeg, ctr + C_MAXDEG, sizeof(maxdeg), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (maxdeg > (unsigned long long)kMaxDeg)
        return pac::set_error(PAC_ERR_CAPACITY, "a ball has " + std::to_string(maxdeg) +
                                                    " alpha edges to higher balls; the limit is " +
                                                    std::to_string(kMaxDeg));
    tm.mark();  // 2

    // ---- alpha triangles (link matrices)
    uint64_t *link = ar.alloc_n<uint64_t>(nL), *faces = ar.alloc_n<uint64_t>(nL);
    if (!link || !faces) return PAC_ERR_OOM;
    CK(cudaMemsetAsync(faces, 0, sizeof(uint64_t) * (nL ? nL : 1), s));
    CK(cudaMemsetAsync(ctr + C_NEXT, 0, sizeof(unsigned long long), s));
    k_link<V><<<std::min<unsigned>(warp_blocks(n), 148 * 4), 256, 0, s>>>(n, at, eoff, ER, loff,
                                                                          link, in.alpha, ctr);
    LAUNCH_CHECK(ctx);
    tm.mark();  // 3

    // ---- tetrahedra
    TetArgs T{};
    T.n = n;
    T.at = at;
    T.orig = orig;
    T.eoff = eoff;
    T.ER = ER;
    T.loff = loff;
    T.link = link;
    T.faces = faces;
    T.cellbeg = cellbeg;
    T.mol = mol;
    T.grids = grids;
    T.alpha = in.alpha;
    T.ctr = ctr;
    T.cellof = cellof;
    T.refute = cfg.refute ? 1 : 0;
    T.verify = cfg.verify ? 1 : 0;
    T.unit_rows = std::max(1, cfg.unit_rows);
    T.scan_claim = std::max(32, cfg.scan_claim);
    T.tcount = ar.alloc_n<uint32_t>(n);
    uint64_t *toff = ar.alloc_n<uint64_t>(n + 1);
    if (!T.tcount || !toff) return PAC_ERR_OOM;
    uint64_t nQ = 0;      // tetrahedra output
    uint64_t nQ_all = 0;  // survivors, a slab's halo included
    uint32_t *tets_sorted = nullptr;
    if (cfg.tet_mode == PAC_TETS_AS_RUN) {
        k_tets<V, 1><<<warp_blocks(n), 256, 0, s>>>(T);
        LAUNCH_CHECK(ctx);
        rc = exclusive_scan(ctx, T.tcount, n, toff);
        if (rc) return rc;
        CK(cudaMemcpyAsync(&nQ, toff + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        tets_sorted = ar.alloc_n<uint32_t>(4 * nQ);
        if (!tets_sorted) return PAC_ERR_OOM;
        T.toff = toff;
        T.tets_out = tets_sorted;
        // the second sweep counts candidates again: reset those counters
        CK(cudaMemsetAsync(ctr + C_CAND_Q, 0, 2 * sizeof(unsigned long long), s));
        k_tets<V, 2><<<warp_blocks(n), 256, 0, s>>>(T);
        LAUNCH_CHECK(ctx);
    } else {
        // queue of alpha tetrahedra in HBM, processed in chunks of balls
        const uint64_t qcap = std::max<uint64_t>(1 << 16, cfg.queue_entries);
        TetQueue Q;
        Q.vid = ar.alloc_n<uint4>(qcap);
        Q.sph = ar.alloc_n<float4>(qcap);
        Q.cap = qcap;
        uint64_t scap = std::max<uint64_t>(1024, 16 * n);
        T.surv = ar.alloc_n<uint2>(scap);
        T.surv_cap = scap;
        T.pend = ar.alloc_n<uint2>(scap / 4 + 1024);
        T.pend_cap = scap / 4 + 1024;
        unsigned long long *claim = ar.alloc_n<unsigned long long>(1);
        unsigned long long *ctrA = ar.alloc_n<unsigned long long>(C_NCOUNTERS);
        if (!Q.vid || !Q.sph || !T.surv || !T.pend || !claim || !ctrA) return PAC_ERR_OOM;
        CK(cudaMemsetAsync(ctr + C_SURV, 0, 2 * sizeof(unsigned long long), s));
        CK(cudaMemsetAsync(ctr + C_INSPHERE, 0, sizeof(unsigned long long), s));
        CK(cudaMemsetAsync(faces, 0, sizeof(uint64_t) * (nL ? nL : 1), s));
        CK(cudaMemsetAsync(T.tcount, 0, sizeof(uint32_t) * n, s));
        // work units of the balls with more than 64 upper neighbours
        uint32_t *hrows = ar.alloc_n<uint32_t>(n);
        uint64_t *uoff = ar.alloc_n<uint64_t>(n + 1);
        if (!hrows || !uoff) return PAC_ERR_OOM;
        uint64_t heavy_units = 0;
        if (maxdeg > 64) {
            k_heavy_rows<<<blocks_for(n, 256), 256, 0, s>>>(n, eoff, T.unit_rows, hrows);
            LAUNCH_CHECK(ctx);
            rc = exclusive_scan(ctx, hrows, n, uoff);
            if (rc) return rc;
            CK(cudaMemcpyAsync(&heavy_units, uoff + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
        }
        rc = enum_smem_optin<V>(ctx);
        if (rc) return rc;
        // the empty-orthosphere test's share of the stage: ev[14], ev[15]
        // around each scan, read once the stream has passed them
        double ortho_ms = 0.0;
        bool ortho_pending = false;
        auto ortho_collect = [&]() {
            if (!ortho_pending) return;
            float f = 0.f;
            if (cudaEventElapsedTime(&f, ctx.ev[14], ctx.ev[15]) == cudaSuccess) ortho_ms += f;
            ortho_pending = false;
        };
        unsigned long long cand_total = 0, alpha_total = 0;
        uint64_t lo = work_lo, chunk = n;
        {
            // first chunk: the whole range when its queue demand (a few
            // entries per alpha triangle) clearly fits, else a probe of 1/32
            // whose fill sizes the next chunks -- an overflowing chunk is
            // enumerated again, smaller
            unsigned long long atri = 0;
            CK(cudaMemcpyAsync(&atri, ctr + C_ALPHA_T, sizeof(atri), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            const double span = (double)(own_hi - work_lo), share = span / (double)std::max<uint64_t>(1, n);
            if (2.0 * (double)atri * share > 0.85 * (double)qcap)
                chunk = std::max<uint64_t>(1, (uint64_t)(span / 32.0));
        }
        // verbose: per-chunk enumeration and scan times
        cudaEvent_t vev[3] = {nullptr, nullptr, nullptr};
        if (cfg.verbose)
            for (auto &e : vev) CK(cudaEventCreate(&e));
        const unsigned enum_blocks = 148u * (unsigned)std::max(1, cfg.enum_blocks);
        const unsigned heavy_blocks = 148u * (unsigned)std::max(1, cfg.heavy_blocks);
        while (lo < own_hi) {
            const uint64_t hi = std::min<uint64_t>(own_hi, lo + chunk);
            TetArgs TA = T;
            TA.ctr = ctrA;
            if (cfg.verbose) CK(cudaEventRecord(vev[0], s));
            CK(cudaMemsetAsync(ctrA, 0, sizeof(unsigned long long) * C_NCOUNTERS, s));
            k_tets_enum<V, 1><<<(unsigned)std::min<uint64_t>(enum_blocks, (hi - lo + 7) / 8),
                                EnumSmem<1>::kWarps * 32, sizeof(EnumSmem<1>), s>>>(TA, Q, lo, hi,
                                                                                   nullptr);
            LAUNCH_CHECK(ctx);
            if (heavy_units) {  // balls with more than 64 upper neighbours, by rows
                CK(cudaMemsetAsync(ctrA + C_NEXT, 0, sizeof(unsigned long long), s));
                k_tets_enum<V, kMaxW><<<heavy_blocks, EnumSmem<kMaxW>::kWarps * 32,
                                        sizeof(EnumSmem<kMaxW>), s>>>(TA, Q, lo, hi, uoff);
                LAUNCH_CHECK(ctx);
            }
            if (cfg.verbose) CK(cudaEventRecord(vev[1], s));
            unsigned long long ha[C_NCOUNTERS], used[2];
            CK(cudaMemcpyAsync(ha, ctrA, sizeof(ha), cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(used, ctr + C_SURV, sizeof(used), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            ortho_collect();
            const unsigned long long queued = ha[C_SURV];
            if (queued > qcap) {
                if (hi - lo == 1)
                    return pac::set_error(PAC_ERR_CAPACITY,
                                          "the alpha tetrahedra of one ball exceed the queue");
                chunk = std::max<uint64_t>(1, (uint64_t)((double)(hi - lo) * 0.5));
                continue;
            }
            // every queued tetrahedron becomes at most one survivor or one
            // pending entry: grow either list (keeping its entries) first
            if (used[0] + queued > T.surv_cap) {
                const uint64_t nc = std::max<uint64_t>(2 * T.surv_cap, used[0] + queued);
                uint2 *nb = ar.alloc_n<uint2>(nc);
                if (!nb) return PAC_ERR_OOM;
                if (used[0])
                    CK(cudaMemcpyAsync(nb, T.surv, sizeof(uint2) * used[0],
                                       cudaMemcpyDeviceToDevice, s));
                T.surv = nb;
                T.surv_cap = nc;
            }
            if (used[1] + queued > T.pend_cap) {
                const uint64_t nc = std::max<uint64_t>(2 * T.pend_cap, used[1] + queued);
                uint2 *nb = ar.alloc_n<uint2>(nc);
                if (!nb) return PAC_ERR_OOM;
                if (used[1])
                    CK(cudaMemcpyAsync(nb, T.pend, sizeof(uint2) * used[1],
                                       cudaMemcpyDeviceToDevice, s));
                T.pend = nb;
                T.pend_cap = nc;
            }
            cand_total += ha[C_CAND_Q];
            alpha_total += ha[C_ALPHA_Q];
            if (ha[C_FILTER] || ha[C_FALLBACK] || ha[C_SOS_RANGE] || ha[C_KILLED] || ha[C_KTESTS]) {
                k_add_tally<<<1, 32, 0, s>>>(ctrA, ctr);
                LAUNCH_CHECK(ctx);
            }
            CK(cudaMemsetAsync(claim, 0, sizeof(unsigned long long), s));
            if (queued) {
                CK(cudaEventRecord(ctx.ev[14], s));
                k_tets_scan<V><<<148 * std::max(1, cfg.scan_blocks), 256, 0, s>>>(T, Q, queued, claim);
                LAUNCH_CHECK(ctx);
                CK(cudaEventRecord(ctx.ev[15], s));
                ortho_pending = true;
            }
            if (cfg.verbose) {
                float me = 0.f, ms = 0.f;
                CK(cudaEventRecord(vev[2], s));
                CK(cudaEventSynchronize(vev[2]));
                CK(cudaEventElapsedTime(&me, vev[0], vev[1]));
                CK(cudaEventElapsedTime(&ms, vev[1], vev[2]));
                std::fprintf(stderr,
                             "[pac] tetrahedra of balls [%llu, %llu): %llu candidates, %llu alpha, "
                             "%llu refuted early, %llu queued; enumeration %.3f ms, scan %.3f ms\n",
                             (unsigned long long)lo, (unsigned long long)hi, ha[C_CAND_Q],
                             ha[C_ALPHA_Q], ha[C_KILLED], queued, me, ms);
            }
            // next chunk sized from this one's queue fill
            if (queued)
                chunk = std::max<uint64_t>(
                    1, (uint64_t)(0.85 * (double)qcap * (double)(hi - lo) / (double)queued));
            else
                chunk = n;
            lo = hi;
        }
        if (cfg.verbose)
            for (auto &e : vev) cudaEventDestroy(e);
        {
            unsigned long long cq[2] = {cand_total, alpha_total};
            CK(cudaMemcpyAsync(ctr + C_CAND_Q, cq, sizeof(cq), cudaMemcpyHostToDevice, s));
        }
        unsigned long long sp[2];
        CK(cudaMemcpyAsync(sp, ctr + C_SURV, sizeof(sp), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        ortho_collect();
        if (sp[0] > T.surv_cap || sp[1] > T.pend_cap)
            return pac::set_error(PAC_ERR_CAPACITY, "tetrahedron survivor buffer overflow");
        if (sp[1] && sp[0] + sp[1] > T.surv_cap) {  // resolved entries join the survivors
            uint2 *nb = ar.alloc_n<uint2>(sp[0] + sp[1]);
            if (!nb) return PAC_ERR_OOM;
            if (sp[0])
                CK(cudaMemcpyAsync(nb, T.surv, sizeof(uint2) * sp[0], cudaMemcpyDeviceToDevice, s));
            T.surv = nb;
            T.surv_cap = sp[0] + sp[1];
        }
        if (sp[1]) {
            CK(cudaEventRecord(ctx.ev[14], s));
            k_sos_resolve<V><<<blocks_for(sp[1], 64), 64, 0, s>>>(T, sp[1]);
            LAUNCH_CHECK(ctx);
            CK(cudaEventRecord(ctx.ev[15], s));
            ortho_pending = true;
            CK(cudaMemcpyAsync(sp, ctr + C_SURV, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            ortho_collect();
        }
        if (st) st->ms_tet_orthosphere = ortho_ms;
        nQ = sp[0];
        if (cfg.slab_world > 1 && own_lo > 0)  // the halo's tetrahedra are not output
            CK(cudaMemsetAsync(T.tcount, 0, sizeof(uint32_t) * own_lo, s));
        rc = exclusive_scan(ctx, T.tcount, n, toff);
        if (rc) return rc;
        if (cfg.slab_world > 1) {
            nQ_all = nQ;
            CK(cudaMemcpyAsync(&nQ, toff + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
        }
    }
    tm.mark();  // 4

    // ---- emission of the tetrahedra: final now, so with to_host their copy
    // crosses PCIe while the triangles and edges are decided
    out.d_tets = ar.alloc_n<uint32_t>(4 * nQ);
    if (!out.d_tets) return PAC_ERR_OOM;
    if (cfg.tet_mode == PAC_TETS_AS_RUN) {
        CK(cudaMemcpyAsync(out.d_tets, tets_sorted, sizeof(uint32_t) * 4 * (nQ ? nQ : 1),
                           cudaMemcpyDeviceToDevice, s));
        k_map4<<<blocks_for(nQ, 256), 256, 0, s>>>(nQ, orig, out.d_tets);
        LAUNCH_CHECK(ctx);
    } else {
        uint32_t *cursor = ar.alloc_n<uint32_t>(n), *keys = ar.alloc_n<uint32_t>(nQ);
        if (!cursor || !keys) return PAC_ERR_OOM;
        CK(cudaMemsetAsync(cursor, 0, sizeof(uint32_t) * n, s));
        const uint64_t ns = std::max(nQ, nQ_all);
        k_tet_scatter<<<blocks_for(ns, 256), 256, 0, s>>>(T.surv, ns, toff, cursor, keys, own_lo,
                                                          own_hi);
        LAUNCH_CHECK(ctx);
        k_tet_sort_emit<<<blocks_for(n, 128), 128, 0, s>>>(n, toff, keys, eoff, ER, orig,
                                                           out.d_tets);
        LAUNCH_CHECK(ctx);
    }
    if (in.to_host && (rc = pac::list_to_host_async(ctx, 2, out.d_tets, 4 * nQ, &out.h_tets)))
        return rc;
    tm.mark();  // 5

    // ---- final triangles
    uint32_t *tricount = ar.alloc_n<uint32_t>(n);
    uint64_t *tpos = ar.alloc_n<uint64_t>(n + 1);
    uint64_t *epos = ar.alloc_n<uint64_t>(nE + 1);
    if (!tricount || !tpos || !epos) return PAC_ERR_OOM;
    CK(cudaMemsetAsync(ctr + C_NEXT, 0, sizeof(unsigned long long), s));
    if (cfg.slab_world > 1) CK(cudaMemsetAsync(tricount, 0, sizeof(uint32_t) * n, s));
    k_tri_attach<V><<<std::min<unsigned>(warp_blocks(own_hi - work_lo), 148 * 4), 256, 0, s>>>(
        work_lo, own_hi, at, eoff, ER, loff, link, faces, tricount, eflag, cellbeg, mol, grids,
        in.alpha, ctr);
    LAUNCH_CHECK(ctx);
    tm.mark();  // 6
    // only the owned balls' triangles are output
    if (cfg.slab_world > 1 && own_lo > work_lo)
        CK(cudaMemsetAsync(tricount + work_lo, 0, sizeof(uint32_t) * (own_lo - work_lo), s));
    rc = exclusive_scan(ctx, tricount, n, tpos);
    if (rc) return rc;
    uint64_t nT = 0;
    CK(cudaMemcpyAsync(&nT, tpos + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    out.d_tris = ar.alloc_n<uint32_t>(3 * nT);
    if (!out.d_tris) return PAC_ERR_OOM;
    k_emit_tris<<<warp_blocks(own_hi - own_lo), 256, 0, s>>>(own_lo, own_hi, eoff, ER, loff, faces,
                                                            tpos, orig, out.d_tris);
    LAUNCH_CHECK(ctx);
    if (in.to_host && (rc = pac::list_to_host_async(ctx, 1, out.d_tris, 3 * nT, &out.h_tris)))
        return rc;
    tm.mark();  // 7

    // ---- final edges
    CK(cudaMemsetAsync(ctr + C_NEXT, 0, sizeof(unsigned long long), s));
    k_edge_final<V><<<std::min<unsigned>(warp_blocks(own_hi - own_lo), 148 * 5), 256, 0, s>>>(
        own_lo, own_hi, at, eoff, ER, eflag, cellbeg, mol, grids, ctr);
    LAUNCH_CHECK(ctx);
    if (cfg.slab_world > 1) {
        // only the owned balls' edges are output
        uint64_t eb[2] = {0, 0};
        CK(cudaMemcpyAsync(&eb[0], eoff + own_lo, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&eb[1], eoff + own_hi, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (eb[0]) CK(cudaMemsetAsync(eflag, 0, eb[0], s));
        if (nE > eb[1]) CK(cudaMemsetAsync(eflag + eb[1], 0, nE - eb[1], s));
    }
    tm.mark();  // 8
    rc = exclusive_scan(ctx, eflag, nE, epos);
    if (rc) return rc;
    uint64_t nEf = 0;
    CK(cudaMemcpyAsync(&nEf, epos + nE, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    out.d_edges = ar.alloc_n<uint32_t>(2 * nEf);
    if (!out.d_edges) return PAC_ERR_OOM;
    k_emit_edges<<<blocks_for(n, 256), 256, 0, s>>>(n, eoff, ER, eflag, epos, orig, out.d_edges);
    LAUNCH_CHECK(ctx);
    if (in.to_host && (rc = pac::list_to_host_async(ctx, 0, out.d_edges, 2 * nEf, &out.h_edges)))
        return rc;
    out.n_edges = nEf;
    out.n_tris = nT;
    out.n_tets = nQ;
    // per-molecule row offsets
    out.edge_off.assign(nm + 1, 0);
    out.tri_off.assign(nm + 1, 0);
    out.tet_off.assign(nm + 1, 0);
    if (nm == 1) {
        out.edge_off[1] = nEf;
        out.tri_off[1] = nT;
        out.tet_off[1] = nQ;
    } else {
        uint64_t *rows = ar.alloc_n<uint64_t>(3 * (size_t)(nm + 1));
        if (!rows) return PAC_ERR_OOM;
        k_mol_rows<<<blocks_for(nm + 1, 128), 128, 0, s>>>(nm, d_off, n, eoff, epos, tpos, toff,
                                                          rows);
        LAUNCH_CHECK(ctx);
        std::vector<uint64_t> h(3 * (size_t)(nm + 1));
        CK(cudaMemcpyAsync(h.data(), rows, sizeof(uint64_t) * h.size(), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (uint32_t m = 0; m <= nm; m++) {
            out.edge_off[m] = h[m];
            out.tri_off[m] = h[(nm + 1) + m];
            out.tet_off[m] = h[2 * (nm + 1) + m];
        }
    }
    tm.mark();  // 9
    // the lists' copies that did not finish under the later stages
    if (in.to_host && (rc = pac::copies_join(ctx))) return rc;
    tm.mark();  // 10
    unsigned long long hc[C_NCOUNTERS];
    CK(cudaMemcpyAsync(hc, ctr, sizeof(hc), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (hc[C_SOS_RANGE])
        return pac::set_error(PAC_ERR_EXACT_RANGE,
                              "coordinate range too wide for the exact SoS integers");
    if (st) {
        st->n_balls = n;
        st->n_cells = total_cells;
        st->cand_edges = hc[C_CAND_E];
        st->alpha_edges = hc[C_ALPHA_E];
        st->cand_tris = hc[C_CAND_T];
        st->alpha_tris = hc[C_ALPHA_T];
        st->cand_tets = hc[C_CAND_Q];
        st->alpha_tets = hc[C_ALPHA_Q];
        st->final_edges = nEf;
        st->final_tris = nT;
        st->final_tets = nQ;
        st->insphere_evals = hc[C_INSPHERE];
        st->sos_calls = hc[C_SOS];
        st->filter_evals = hc[C_FILTER];
        st->exact_fallbacks = hc[C_FALLBACK];
        st->early_refuted = hc[C_KILLED];
        st->early_tests = hc[C_KTESTS];
        st->cert_decisions = hc[C_CERT];
        st->cert_disagreements = hc[C_CERT_BAD];
        st->ortho_out_of_grid = hc[C_OOB];
        st->max_degree = maxdeg;
        st->ms_grid = tm.ms(0, 1);
        st->ms_edges = tm.ms(1, 2);
        st->ms_tris = tm.ms(2, 3);
        st->ms_tets = tm.ms(3, 4);
        st->ms_tri_attach = tm.ms(5, 6);
        st->ms_edge_attach = tm.ms(7, 8);
        st->ms_emit = tm.ms(4, 5) + tm.ms(6, 7) + tm.ms(8, 9);
        if (in.to_host) st->ms_d2h = tm.ms(9, 10);
        // the reference's data movement for this pass: balls in, lists out,
        // and every candidate list (edges 8 B, triangles 12 B + 16 B
        // orthosphere, tetrahedra 16 B + 16 B orthosphere) written and read
        // once -- independent of how this engine avoids storing them
        st->bytes_model = 16 * n + 8 * st->final_edges + 12 * st->final_tris +
                          16 * st->final_tets +
                          2 * (8 * st->cand_edges + 28 * st->cand_tris + 32 * st->cand_tets);
        if (nm == 1) {
            st->grid[0] = hg[0].gx;
            st->grid[1] = hg[0].gy;
            st->grid[2] = hg[0].gz;
            st->step = hg[0].step;
        }
    }
    if (cfg.verbose)
        std::fprintf(stderr,
                     "[pac] %llu balls: grid %.3f, edges %.3f, triangles %.3f, tetrahedra %.3f, "
                     "triangle attachment %.3f, edge attachment %.3f, emission %.3f ms\n",
                     (unsigned long long)n, tm.ms(0, 1), tm.ms(1, 2), tm.ms(2, 3), tm.ms(3, 4),
                     tm.ms(5, 6), tm.ms(7, 8), tm.ms(4, 5) + tm.ms(6, 7) + tm.ms(8, 9));
    return PAC_OK;
}

int run_pass(pac::Ctx &ctx, const pac::PipelineConfig &cfg, const pac::PassInput &in,
             pac::PassOutput &out, pac_stats *st) {
    if (cfg.exact) {
#if PAC_WITH_EXACT
        return run_pass_v<pac::kExact>(ctx, cfg, in, out, st);
#else
        return pac::set_error(PAC_ERR_INVALID_ARG, "exact predicates are built in the strict flavour");
#endif
    }
    if (cfg.formula == PAC_FORMULA_PLAIN_XMP) return run_pass_v<pac::kPlainXmp>(ctx, cfg, in, out, st);
    return run_pass_v<pac::kUpstream>(ctx, cfg, in, out, st);
}

}  // namespace PAC_NS
