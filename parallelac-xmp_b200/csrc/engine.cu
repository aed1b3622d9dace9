// engine.cu -- the extern "C" API of libpac.so (declared in include/pac.h):
// context and device memory pool, the host/device/batched entry points,
// CRD input and the reference's text output format.
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pac_internal.h"

struct pac_ctx {
    pac::Ctx c;
};

pac::Ctx &pac_ctx_internal(pac_ctx *ctx) { return ctx->c; }

namespace pac {

static thread_local std::string g_last_error;

int set_error(int status, const std::string &msg) {
    g_last_error = msg;
    return status;
}

int list_to_host_async(Ctx &c, int which, const uint32_t *src, size_t count, uint32_t **dst) {
    *dst = nullptr;
    if (!c.copy_stream) {
        if (cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
            c.copy_stream = nullptr;
            return set_error(PAC_ERR_CUDA, "cudaStreamCreate (copy stream) failed");
        }
        for (auto &ev : c.copy_ev)
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
                return set_error(PAC_ERR_CUDA, "cudaEventCreate (copy stream) failed");
    }
    if (count == 0) return PAC_OK;
    const size_t need = sizeof(uint32_t) * count;
    if (need > c.pinned_size[which]) {
        // nothing may still be copying into the old region
        cudaStreamSynchronize(c.copy_stream);
        if (c.pinned[which]) cudaFreeHost(c.pinned[which]);
        c.pinned[which] = nullptr;
        c.pinned_size[which] = 0;
        const size_t sz = std::max(need + need / 4, size_t(1) << 20);
        if (cudaMallocHost(&c.pinned[which], sz) != cudaSuccess) {
            c.pinned[which] = nullptr;
            cudaGetLastError();
            return set_error(PAC_ERR_OOM, "cudaMallocHost for the output lists failed");
        }
        c.pinned_size[which] = sz;
    }
    cudaError_t e = cudaEventRecord(c.copy_ev[which], c.stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c.copy_stream, c.copy_ev[which], 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c.pinned[which], src, need, cudaMemcpyDeviceToHost, c.copy_stream);
    if (e != cudaSuccess) return set_error(PAC_ERR_CUDA, std::string("D2H: ") + cudaGetErrorString(e));
    *dst = static_cast<uint32_t *>(c.pinned[which]);
    return PAC_OK;
}

int copies_join(Ctx &c) {
    if (!c.copy_stream) return PAC_OK;
    cudaError_t e = cudaEventRecord(c.copy_ev[3], c.copy_stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c.stream, c.copy_ev[3], 0);
    if (e != cudaSuccess) return set_error(PAC_ERR_CUDA, std::string("D2H: ") + cudaGetErrorString(e));
    return PAC_OK;
}

Arena::~Arena() {
    for (auto &b : blocks_) cudaFree(b.base);
}

void *Arena::alloc(size_t bytes) {
    bytes = (bytes + 255) & ~size_t(255);
    while (cur_ < blocks_.size()) {
        Block &b = blocks_[cur_];
        if (b.used + bytes <= b.size) {
            void *p = b.base + b.used;
            b.used += bytes;
            return p;
        }
        cur_++;
    }
    size_t sz = std::max<size_t>(bytes, size_t(256) << 20);
    char *p = nullptr;
    cudaError_t e = cudaMalloc(&p, sz);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(PAC_ERR_OOM, std::string("cudaMalloc(") + std::to_string(sz) +
                                   "): " + cudaGetErrorString(e));
        return nullptr;
    }
    blocks_.push_back(Block{p, sz, bytes});
    cur_ = blocks_.size() - 1;
    return p;
}

void Arena::reset() {
    // merge: if more than one block was needed, replace them by one block
    // large enough for the whole previous call, so later calls are served
    // from a single region
    if (blocks_.size() > 1) {
        size_t total = 0;
        for (auto &b : blocks_) total += b.size;
        for (auto &b : blocks_) cudaFree(b.base);
        blocks_.clear();
        char *p = nullptr;
        if (cudaMalloc(&p, total) == cudaSuccess)
            blocks_.push_back(Block{p, total, 0});
        else
            cudaGetLastError();
    }
    for (auto &b : blocks_) b.used = 0;
    cur_ = 0;
}

Arena::Mark Arena::mark() const {
    if (cur_ >= blocks_.size()) return Mark{cur_, 0};
    return Mark{cur_, blocks_[cur_].used};
}

void Arena::rewind(const Mark &m) {
    // blocks past the mark's were empty when it was taken (alloc only moves
    // forward and fresh or reset blocks start empty); blocks added since
    // stay reserved for the next call
    for (size_t k = m.block + 1; k < blocks_.size(); k++) blocks_[k].used = 0;
    if (m.block < blocks_.size()) blocks_[m.block].used = m.used;
    cur_ = std::min(m.block, blocks_.size());
}

size_t Arena::reserved() const {
    size_t t = 0;
    for (auto &b : blocks_) t += b.size;
    return t;
}

}  // namespace pac

// ----------------------------------------------------------------- helpers
namespace {

// Timing events of one host entry point call, destroyed on every return path.
struct EventSet {
    cudaEvent_t e[3]{};
    EventSet() {
        for (auto &x : e) cudaEventCreate(&x);
    }
    ~EventSet() {
        for (auto &x : e)
            if (x) cudaEventDestroy(x);
    }
    EventSet(const EventSet &) = delete;
    EventSet &operator=(const EventSet &) = delete;
};

__global__ void k_check_finite(const float4 *b, uint64_t n, int *bad) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = b[i];
    if (!isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z) || !isfinite(v.w)) *bad = 1;
}

// Launch shapes for the autotuner (pac_options.autotune): blocks per SM of
// the two tetrahedron enumeration kernels and of the orthosphere scan, the
// rows of a large ball per enumeration work unit, and the queue entries a
// scan warp claims at a time.  The first is the default.  None of them
// changes the output.
constexpr pac::LaunchShape kShapes[] = {
    {4, 4, 4, 8, 256},  {3, 4, 4, 8, 256}, {2, 4, 4, 8, 256},  {4, 3, 4, 8, 256},
    {4, 4, 3, 8, 256},  {4, 4, 6, 8, 256}, {4, 4, 4, 4, 256},  {4, 4, 4, 16, 256},
    {4, 4, 4, 8, 512},  {4, 4, 4, 8, 2048}, {2, 2, 2, 8, 256}, {4, 2, 4, 4, 256}};
constexpr int kNumShapes = (int)(sizeof(kShapes) / sizeof(kShapes[0]));
static_assert(kNumShapes <= 16, "Tuner holds 16 timings");

// One pass; with to_host the lists are copied into the context's pinned
// host memory while the pass runs (out.h_*), complete on return.
int run(pac_ctx *ctx, const float4 *d_balls, uint64_t n, uint32_t n_mol,
        const uint64_t *h_off, float sol, float alpha, pac::PassOutput &out, pac_stats *st,
        bool to_host = false) {
    pac::Ctx &c = ctx->c;
    if (!std::isfinite(sol) || !std::isfinite(alpha))
        return pac::set_error(PAC_ERR_INVALID_ARG, "sol_rad and alpha must be finite");
    int *bad = c.arena.alloc_n<int>(1);
    if (!bad) return PAC_ERR_OOM;
    cudaMemsetAsync(bad, 0, sizeof(int), c.stream);
    k_check_finite<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(d_balls, n, bad);
    int hbad = 0;
    cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, c.stream);
    cudaError_t e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess)
        return pac::set_error(PAC_ERR_CUDA, std::string("input check: ") + cudaGetErrorString(e));
    if (hbad) return pac::set_error(PAC_ERR_INVALID_ARG, "non-finite ball coordinate or radius");
    // the alpha-tetrahedron queue: a quarter of the free memory at the
    // context's first pass, at most 12 GiB (32 B per entry); a pass whose
    // queued tetrahedra exceed it runs in chunks
    if (!c.queue_bytes) {
        size_t freeb = 0, totalb = 0;
        cudaMemGetInfo(&freeb, &totalb);
        c.queue_bytes = std::max<uint64_t>(std::min<uint64_t>(freeb / 4, 12ull << 30), 32ull << 16);
    }
    uint64_t qbytes = c.queue_bytes;
    if (c.opt.reserved_u[0]) qbytes = c.opt.reserved_u[0] * 32ull;  // test hook: entries
    const pac::LaunchShape *shape = &kShapes[0];
    // launch shapes: the caller's overrides, else the autotuner's current
    // candidate or its choice, else the defaults
    bool overridden = false;
    for (int k = 0; k < 5; k++) overridden |= c.opt.reserved_i[k] > 0;
    int cand = -1;
    if (c.opt.autotune && !overridden) {
        cand = c.tuner.best >= 0 ? c.tuner.best : c.tuner.next;
        shape = &kShapes[cand];
    }
    pac::PipelineConfig cfg{};
    cfg.formula = c.opt.formula;
    cfg.tet_mode = c.opt.tet_mode;
    cfg.verbose = c.opt.verbose;
    cfg.queue_entries = qbytes / 32;
    cfg.exact = c.opt.predicates == PAC_PRED_EXACT;
    cfg.refute = c.opt.reserved_i[5] != 1;
    cfg.slab_world = c.opt.reserved_i[7] > 1 ? c.opt.reserved_i[7] : 1;
    cfg.slab_rank = c.opt.reserved_i[8];
    cfg.verify = c.opt.reserved_i[6] == 1;
    cfg.enum_blocks = c.opt.reserved_i[0] > 0 ? c.opt.reserved_i[0] : shape->enum_blocks;
    cfg.scan_blocks = c.opt.reserved_i[1] > 0 ? c.opt.reserved_i[1] : shape->scan_blocks;
    cfg.heavy_blocks = c.opt.reserved_i[2] > 0 ? c.opt.reserved_i[2] : shape->heavy_blocks;
    cfg.unit_rows = c.opt.reserved_i[3] > 0 ? c.opt.reserved_i[3] : shape->unit_rows;
    cfg.scan_claim = c.opt.reserved_i[4] > 0 ? c.opt.reserved_i[4] : shape->scan_claim;
    pac_stats local;
    pac_stats *sp = st ? st : &local;
    pac::PassInput in{d_balls, n, n_mol, h_off, sol, alpha};
    in.to_host = to_host;
    int rc = (c.opt.predicates == PAC_PRED_REFCOMPAT_FMA)
                 ? pac_fma::run_pass(c, cfg, in, out, sp)
                 : pac_strict::run_pass(c, cfg, in, out, sp);
    // a pass that stopped early may have list copies in flight: they end
    // before the pool or the pinned regions are reused
    if (rc != PAC_OK && c.copy_stream) cudaStreamSynchronize(c.copy_stream);
    if (rc == PAC_OK && cand >= 0 && c.tuner.best < 0) {
        // every candidate gives the same lists; keep the fastest tetrahedron
        // stage once each has run on this context's work
        c.tuner.ms[cand] = sp->ms_tets;
        if (++c.tuner.next == kNumShapes) {
            int b = 0;
            for (int k = 1; k < kNumShapes; k++)
                if (c.tuner.ms[k] < c.tuner.ms[b]) b = k;
            c.tuner.best = b;
        }
    }
    if (rc == PAC_OK) {
        e = cudaStreamSynchronize(c.stream);
        if (e != cudaSuccess)
            return pac::set_error(PAC_ERR_CUDA, std::string("pass: ") + cudaGetErrorString(e));
    }
    return rc;
}

int validate_opts(const pac_options &o) {
    if (o.formula != PAC_FORMULA_UPSTREAM && o.formula != PAC_FORMULA_PLAIN_XMP)
        return pac::set_error(PAC_ERR_INVALID_ARG, "unknown formula");
    if (o.tet_mode != PAC_TETS_AS_WRITTEN && o.tet_mode != PAC_TETS_AS_RUN)
        return pac::set_error(PAC_ERR_INVALID_ARG, "unknown tet_mode");
    if (o.predicates != PAC_PRED_REFCOMPAT && o.predicates != PAC_PRED_REFCOMPAT_FMA &&
        o.predicates != PAC_PRED_EXACT)
        return pac::set_error(PAC_ERR_INVALID_ARG, "unknown predicate mode");
    if (o.order != PAC_ORDER_REFERENCE && o.order != PAC_ORDER_CANONICAL)
        return pac::set_error(PAC_ERR_INVALID_ARG, "unknown order");
    return PAC_OK;
}

// in-place canonical order on the host copy: ascending vertices within each
// simplex, rows sorted lexicographically
template <int K>
void canonicalise(uint32_t *rows, uint64_t nrows) {
    struct Row {
        uint32_t v[K];
        bool operator<(const Row &o) const {
            for (int i = 0; i < K; i++)
                if (v[i] != o.v[i]) return v[i] < o.v[i];
            return false;
        }
    };
    Row *r = reinterpret_cast<Row *>(rows);
    for (uint64_t i = 0; i < nrows; i++) {
        for (int a = 1; a < K; a++)
            for (int b = a; b > 0 && r[i].v[b] < r[i].v[b - 1]; b--) {
                uint32_t t = r[i].v[b];
                r[i].v[b] = r[i].v[b - 1];
                r[i].v[b - 1] = t;
            }
    }
    std::sort(r, r + nrows);
}

}  // namespace

// ----------------------------------------------------------------- C ABI
extern "C" {

int pac_abi_version(void) { return PAC_ABI_VERSION; }

void pac_default_options(pac_options *opt) {
    if (!opt) return;
    std::memset(opt, 0, sizeof(*opt));
    opt->device = 0;
    opt->formula = PAC_FORMULA_UPSTREAM;
    opt->tet_mode = PAC_TETS_AS_WRITTEN;
    opt->predicates = PAC_PRED_REFCOMPAT;
    opt->order = PAC_ORDER_REFERENCE;
}

int pac_create(pac_ctx **out, const pac_options *opt) {
    if (!out) return pac::set_error(PAC_ERR_INVALID_ARG, "ctx is null");
    *out = nullptr;
    pac_options o;
    pac_default_options(&o);
    if (opt) o = *opt;
    int rc = validate_opts(o);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return pac::set_error(PAC_ERR_NO_DEVICE, "no CUDA device");
    }
    if (o.device < 0 || o.device >= ndev)
        return pac::set_error(PAC_ERR_INVALID_ARG, "device ordinal out of range");
    cudaError_t e = cudaSetDevice(o.device);
    if (e != cudaSuccess)
        return pac::set_error(PAC_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    pac_ctx *c = new pac_ctx();
    c->c.device = o.device;
    c->c.opt = o;
    if (cudaStreamCreateWithFlags(&c->c.stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return pac::set_error(PAC_ERR_CUDA, "cudaStreamCreate failed");
    }
    for (auto &ev : c->c.ev) cudaEventCreate(&ev);
    *out = c;
    return PAC_OK;
}

int pac_destroy(pac_ctx *ctx) {
    if (!ctx) return PAC_OK;
    cudaSetDevice(ctx->c.device);
    cudaStreamSynchronize(ctx->c.stream);
    for (auto &ev : ctx->c.ev)
        if (ev) cudaEventDestroy(ev);
    if (ctx->c.copy_stream) {
        cudaStreamSynchronize(ctx->c.copy_stream);
        for (auto &ev : ctx->c.copy_ev)
            if (ev) cudaEventDestroy(ev);
        cudaStreamDestroy(ctx->c.copy_stream);
    }
    for (void *p : ctx->c.pinned)
        if (p) cudaFreeHost(p);
    cudaStreamDestroy(ctx->c.stream);
    delete ctx;
    return PAC_OK;
}

void *pac_cuda_stream(pac_ctx *ctx) { return ctx ? (void *)ctx->c.stream : nullptr; }

int pac_alpha_complex_device(pac_ctx *ctx, const pac_ball *d_balls, uint32_t n, float sol_rad,
                             float alpha, pac_complex *out, pac_stats *st) {
    if (!ctx || !out || (n && !d_balls))
        return pac::set_error(PAC_ERR_INVALID_ARG, "null argument");
    std::memset(out, 0, sizeof(*out));
    out->n_vertices = n;
    out->on_device = 1;
    if (st) std::memset(st, 0, sizeof(*st));
    if (n == 0) return PAC_OK;
    pac::Ctx &c = ctx->c;
    cudaSetDevice(c.device);
    c.arena.reset();
    c.launches = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, c.stream);
    uint64_t off[2] = {0, n};
    pac::PassOutput po;
    int rc = run(ctx, reinterpret_cast<const float4 *>(d_balls), n, 1, off, sol_rad, alpha, po, st);
    cudaEventRecord(e1, c.stream);
    cudaEventSynchronize(e1);
    if (st && !rc) {
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        st->ms_total = t;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    out->n_edges = po.n_edges;
    out->n_tris = po.n_tris;
    out->n_tets = po.n_tets;
    out->edges = po.d_edges;
    out->tris = po.d_tris;
    out->tets = po.d_tets;
    if (st) st->kernels_launched = (uint32_t)c.launches;
    return PAC_OK;
}

int pac_alpha_complex(pac_ctx *ctx, const pac_ball *balls, uint32_t n, float sol_rad, float alpha,
                      pac_complex *out, pac_stats *st) {
    if (!ctx || !out || (n && !balls)) return pac::set_error(PAC_ERR_INVALID_ARG, "null argument");
    std::memset(out, 0, sizeof(*out));
    out->n_vertices = n;
    if (st) std::memset(st, 0, sizeof(*st));
    if (n == 0) return PAC_OK;
    pac::Ctx &c = ctx->c;
    cudaSetDevice(c.device);
    c.arena.reset();
    c.launches = 0;
    EventSet ev;
    cudaEventRecord(ev.e[0], c.stream);
    float4 *d = c.arena.alloc_n<float4>(n);
    if (!d) return PAC_ERR_OOM;
    cudaError_t e = cudaMemcpyAsync(d, balls, sizeof(float4) * n, cudaMemcpyHostToDevice, c.stream);
    if (e != cudaSuccess)
        return pac::set_error(PAC_ERR_CUDA, std::string("H2D: ") + cudaGetErrorString(e));
    cudaEventRecord(ev.e[1], c.stream);
    uint64_t off[2] = {0, n};
    pac::PassOutput po;
    // the lists reach the context's pinned memory during the pass
    int rc = run(ctx, d, n, 1, off, sol_rad, alpha, po, st, true);
    if (rc) return rc;
    cudaEventRecord(ev.e[2], c.stream);
    e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess)
        return pac::set_error(PAC_ERR_CUDA, std::string("D2H: ") + cudaGetErrorString(e));
    out->n_edges = po.n_edges;
    out->n_tris = po.n_tris;
    out->n_tets = po.n_tets;
    out->on_device = 3;  // context-owned pinned host memory
    out->edges = po.h_edges;
    out->tris = po.h_tris;
    out->tets = po.h_tets;
    if (c.opt.order == PAC_ORDER_CANONICAL) {
        canonicalise<2>(out->edges, out->n_edges);
        canonicalise<3>(out->tris, out->n_tris);
        canonicalise<4>(out->tets, out->n_tets);
    }
    if (st) {
        float a = 0, t = 0;
        cudaEventElapsedTime(&a, ev.e[0], ev.e[1]);
        cudaEventElapsedTime(&t, ev.e[0], ev.e[2]);
        st->ms_h2d = a;  // ms_d2h: set by the pass
        st->ms_total = t;
        st->kernels_launched = (uint32_t)c.launches;
    }
    return PAC_OK;
}

int pac_alpha_complex_batch(pac_ctx *ctx, const pac_ball *balls, const uint64_t *offsets,
                            uint32_t n_mol, float sol_rad, float alpha, pac_batch_complex *out,
                            pac_stats *st) {
    if (!ctx || !out || !offsets || n_mol == 0)
        return pac::set_error(PAC_ERR_INVALID_ARG, "null argument or no molecules");
    std::memset(out, 0, sizeof(*out));
    if (st) std::memset(st, 0, sizeof(*st));
    if (offsets[0] != 0) return pac::set_error(PAC_ERR_INVALID_ARG, "offsets[0] must be 0");
    if (ctx->c.opt.reserved_i[7] > 1)
        return pac::set_error(PAC_ERR_INVALID_ARG, "slab passes take one molecule");
    for (uint32_t m = 0; m < n_mol; m++)
        if (offsets[m + 1] < offsets[m])
            return pac::set_error(PAC_ERR_INVALID_ARG, "offsets must be non-decreasing");
    uint64_t n = offsets[n_mol];
    if (n >= 0xffffffffull) return pac::set_error(PAC_ERR_CAPACITY, "more than 2^32-1 balls");
    if (n && !balls) return pac::set_error(PAC_ERR_INVALID_ARG, "balls is null");
    // empty molecules are carried as zero-length ranges; the pass itself
    // needs at least one ball per molecule, so drop them and re-expand
    std::vector<uint32_t> keep;
    std::vector<uint64_t> koff(1, 0);
    for (uint32_t m = 0; m < n_mol; m++)
        if (offsets[m + 1] > offsets[m]) {
            keep.push_back(m);
            koff.push_back(offsets[m + 1]);
        }
    out->n_mol = n_mol;
    out->on_device = 3;
    out->edge_off = (uint64_t *)std::calloc(n_mol + 1, sizeof(uint64_t));
    out->tri_off = (uint64_t *)std::calloc(n_mol + 1, sizeof(uint64_t));
    out->tet_off = (uint64_t *)std::calloc(n_mol + 1, sizeof(uint64_t));
    if (!out->edge_off || !out->tri_off || !out->tet_off) {
        pac_free_batch_complex(out);
        return pac::set_error(PAC_ERR_OOM, "host allocation failed");
    }
    if (keep.empty()) return PAC_OK;
    pac::Ctx &c = ctx->c;
    cudaSetDevice(c.device);
    c.arena.reset();
    c.launches = 0;
    EventSet ev;
    cudaEventRecord(ev.e[0], c.stream);
    float4 *d = c.arena.alloc_n<float4>(n);
    if (!d) {
        pac_free_batch_complex(out);
        return PAC_ERR_OOM;
    }
    cudaMemcpyAsync(d, balls, sizeof(float4) * n, cudaMemcpyHostToDevice, c.stream);
    cudaEventRecord(ev.e[1], c.stream);
    pac::PassOutput po;
    // the lists reach the context's pinned memory during the pass
    int rc = run(ctx, d, n, (uint32_t)keep.size(), koff.data(), sol_rad, alpha, po, st, true);
    if (rc) {
        pac_free_batch_complex(out);
        return rc;
    }
    out->on_device = 3;
    out->edges = po.h_edges;
    out->tris = po.h_tris;
    out->tets = po.h_tets;
    cudaEventRecord(ev.e[2], c.stream);
    cudaError_t e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess) {
        pac_free_batch_complex(out);
        return pac::set_error(PAC_ERR_CUDA, std::string("batch: ") + cudaGetErrorString(e));
    }
    // re-expand the row offsets over all molecules
    size_t k = 0;
    for (uint32_t m = 0; m <= n_mol; m++) {
        while (k < keep.size() && keep[k] < m) k++;
        out->edge_off[m] = po.edge_off[k];
        out->tri_off[m] = po.tri_off[k];
        out->tet_off[m] = po.tet_off[k];
    }
    if (c.opt.order == PAC_ORDER_CANONICAL)
        for (uint32_t m = 0; m < n_mol; m++) {
            canonicalise<2>(out->edges + 2 * out->edge_off[m], out->edge_off[m + 1] - out->edge_off[m]);
            canonicalise<3>(out->tris + 3 * out->tri_off[m], out->tri_off[m + 1] - out->tri_off[m]);
            canonicalise<4>(out->tets + 4 * out->tet_off[m], out->tet_off[m + 1] - out->tet_off[m]);
        }
    if (st) {
        float a = 0, t = 0;
        cudaEventElapsedTime(&a, ev.e[0], ev.e[1]);
        cudaEventElapsedTime(&t, ev.e[0], ev.e[2]);
        st->ms_h2d = a;  // ms_d2h: set by the pass
        st->ms_total = t;
        st->kernels_launched = (uint32_t)c.launches;
    }
    return PAC_OK;
}

int pac_union_measure(pac_ctx *ctx, const double *xyzr, uint32_t n, const pac_complex *cx,
                      double *vol, double *area, double *dvol, double *darea) {
    if (!ctx || !cx || (n && !xyzr)) return pac::set_error(PAC_ERR_INVALID_ARG, "null argument");
    if (cx->n_vertices && cx->n_vertices != n)
        return pac::set_error(PAC_ERR_INVALID_ARG, "complex and balls differ in size");
    if (cx->on_device == 1 &&
        ((cx->n_edges && !cx->edges) || (cx->n_tris && !cx->tris) || (cx->n_tets && !cx->tets)))
        return pac::set_error(PAC_ERR_INVALID_ARG, "a non-empty list has a null pointer");
    pac::Ctx &c = ctx->c;
    cudaSetDevice(c.device);
    // no arena reset: a device complex from the previous call may live
    // there; this call's copies and scratch go back to the pool on return,
    // so repeated calls do not grow it
    pac::ArenaRewind rewind(c.arena);
    double4 *d = c.arena.alloc_n<double4>(n);
    if (!d) return PAC_ERR_OOM;
    cudaMemcpyAsync(d, xyzr, sizeof(double4) * n, cudaMemcpyHostToDevice, c.stream);
    const uint32_t *l[3] = {cx->edges, cx->tris, cx->tets};
    uint64_t cnt[3] = {cx->n_edges, cx->n_tris, cx->n_tets};
    const uint32_t *dl[3];
    for (int k = 0; k < 3; k++) {
        if (cx->on_device == 1 || !cnt[k]) {
            dl[k] = l[k];
            continue;
        }
        uint32_t *p = c.arena.alloc_n<uint32_t>((k + 2) * cnt[k]);
        if (!p) return PAC_ERR_OOM;
        cudaMemcpyAsync(p, l[k], sizeof(uint32_t) * (k + 2) * cnt[k], cudaMemcpyHostToDevice,
                        c.stream);
        dl[k] = p;
    }
    double *dV = nullptr, *dA = nullptr;
    if (dvol) dV = c.arena.alloc_n<double>(4 * (size_t)n);
    if (darea) dA = c.arena.alloc_n<double>(4 * (size_t)n);
    if ((dvol && !dV) || (darea && !dA)) return PAC_ERR_OOM;
    if ((dvol && !darea) || (darea && !dvol)) {
        // the kernel fills both when either is wanted
        if (!dV) dV = c.arena.alloc_n<double>(4 * (size_t)n);
        if (!dA) dA = c.arena.alloc_n<double>(4 * (size_t)n);
    }
    int rc = pac::union_measure_device(c, d, n, dl[0], cnt[0], dl[1], cnt[1], dl[2], cnt[2], vol,
                                       area, dV, dA, nullptr);
    if (rc) return rc;
    if (dvol) cudaMemcpyAsync(dvol, dV, 4 * sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream);
    if (darea) cudaMemcpyAsync(darea, dA, 4 * sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream);
    cudaError_t e = cudaStreamSynchronize(c.stream);
    if (e != cudaSuccess)
        return pac::set_error(PAC_ERR_CUDA, std::string("union measure: ") + cudaGetErrorString(e));
    return PAC_OK;
}

int pac_union_measure_device(pac_ctx *ctx, const double *d_xyzr, uint32_t n, const pac_complex *cx,
                             double *vol, double *area, double *d_dvol, double *d_darea) {
    if (!ctx || !cx || (n && !d_xyzr)) return pac::set_error(PAC_ERR_INVALID_ARG, "null argument");
    if (cx->on_device != 1)
        return pac::set_error(PAC_ERR_INVALID_ARG, "pac_union_measure_device needs device lists");
    if (cx->n_vertices && cx->n_vertices != n)
        return pac::set_error(PAC_ERR_INVALID_ARG, "complex and balls differ in size");
    if ((cx->n_edges && !cx->edges) || (cx->n_tris && !cx->tris) || (cx->n_tets && !cx->tets))
        return pac::set_error(PAC_ERR_INVALID_ARG, "a non-empty list has a null pointer");
    pac::Ctx &c = ctx->c;
    cudaSetDevice(c.device);
    // scratch of this call (partial sums, gradients not passed) is handed
    // back to the pool on return: repeated calls do not grow it
    pac::ArenaRewind rewind(c.arena);
    return pac::union_measure_device(c, reinterpret_cast<const double4 *>(d_xyzr), n, cx->edges,
                                     cx->n_edges, cx->tris, cx->n_tris, cx->tets, cx->n_tets, vol,
                                     area, d_dvol, d_darea, nullptr);
}

void pac_free_complex(pac_complex *cx) {
    if (!cx) return;
    if (cx->on_device == 2) {
        if (cx->edges) cudaFreeHost(cx->edges);
        if (cx->tris) cudaFreeHost(cx->tris);
        if (cx->tets) cudaFreeHost(cx->tets);
    } else if (cx->on_device == 0) {
        std::free(cx->edges);
        std::free(cx->tris);
        std::free(cx->tets);
    }
    // on_device == 1 (device pool) or 3 (pinned host buffer): the lists
    // belong to the context and stay valid until its next call
    cx->edges = cx->tris = cx->tets = nullptr;
    cx->n_edges = cx->n_tris = cx->n_tets = 0;
}

void pac_free_batch_complex(pac_batch_complex *cx) {
    if (!cx) return;
    std::free(cx->edge_off);
    std::free(cx->tri_off);
    std::free(cx->tet_off);
    std::memset(cx, 0, sizeof(*cx));
}

const char *pac_status_string(int status) {
    switch (status) {
        case PAC_OK: return "ok";
        case PAC_ERR_INVALID_ARG: return "invalid argument";
        case PAC_ERR_CUDA: return "CUDA error";
        case PAC_ERR_CAPACITY: return "capacity exceeded";
        case PAC_ERR_TIMEOUT: return "device wait timed out";
        case PAC_ERR_NO_DEVICE: return "no CUDA device";
        case PAC_ERR_EXACT_RANGE: return "exact arithmetic range exceeded";
        case PAC_ERR_OOM: return "out of memory";
        case PAC_ERR_IO: return "I/O error";
        default: return "unknown status";
    }
}

const char *pac_last_error(void) { return pac::g_last_error.c_str(); }

// pac_read_crd and pac_write_complex: textio.cpp.

}  // extern "C"
