// pac_internal.h -- types shared by the C ABI layer (engine.cu) and the
// pipeline translation unit (pipeline.cu, compiled once per arithmetic
// flavour).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/pac.h"

namespace pac {

// Device memory pool: a list of large blocks handed out by bumping an
// offset; reset() makes everything reusable without freeing, so repeated
// calls on a context allocate nothing after the first.
class Arena {
   public:
    ~Arena();
    // 256-byte aligned; returns nullptr and records the error on failure
    void *alloc(size_t bytes);
    template <class T>
    T *alloc_n(size_t n) {
        return static_cast<T *>(alloc(sizeof(T) * (n ? n : 1)));
    }
    void reset();
    size_t reserved() const;
    // A position in the pool: rewind() releases everything allocated after
    // mark() was taken, keeping what came before (e.g. a complex that the
    // caller still holds).  The memory released must no longer be in use by
    // queued work other than on the context's own stream.
    struct Mark {
        size_t block, used;
    };
    Mark mark() const;
    void rewind(const Mark &m);

   private:
    struct Block {
        char *base;
        size_t size, used;
    };
    std::vector<Block> blocks_;
    size_t cur_ = 0;
};

// Rewinds the pool to where it was at construction, on every return path.
struct ArenaRewind {
    Arena &a;
    Arena::Mark m;
    explicit ArenaRewind(Arena &arena) : a(arena), m(arena.mark()) {}
    ~ArenaRewind() { a.rewind(m); }
    ArenaRewind(const ArenaRewind &) = delete;
    ArenaRewind &operator=(const ArenaRewind &) = delete;
};

struct PipelineConfig {
    int formula;    // pac_formula
    int tet_mode;   // pac_tet_mode
    int verbose;
    uint64_t queue_entries;  // alpha tetrahedra queued per chunk (32 B each)
    bool exact;              // decision-exact predicates (strict flavour only)
    int slab_rank, slab_world;  // one slab of a partition by cell order (world > 1)
    bool refute;             // early refutation in the tetrahedron enumeration
    bool verify;             // replay every certified insphere decision (debug)
    // launch shapes (the output does not depend on them)
    int enum_blocks;   // k_tets_enum<.., 1> blocks per SM
    int heavy_blocks;  // k_tets_enum<.., kMaxW> blocks per SM
    int scan_blocks;   // k_tets_scan blocks per SM
    int unit_rows;     // rows of a ball of more than 64 upper neighbours per work unit
    int scan_claim;    // queue entries a scan warp claims at a time
};

// Launch shapes the autotuner tries, and its state per context.
struct LaunchShape {
    int enum_blocks, heavy_blocks, scan_blocks, unit_rows, scan_claim;
};
struct Tuner {
    int next = 0;          // next candidate to measure
    int best = -1;         // chosen candidate once all are measured
    double ms[16] = {0};   // tetrahedron-stage time of each candidate
};

// Inputs of one device pass over one or more molecules.
struct PassInput {
    const float4 *d_balls;      // n x (x, y, z, raw r), molecules back to back
    uint64_t n;                 // total balls
    uint32_t n_mol;             // molecules
    const uint64_t *h_offsets;  // n_mol + 1 (host)
    float sol, alpha;
    // copy each list into the context's pinned host memory as soon as it is
    // emitted (on the copy stream, while the later stages run)
    bool to_host = false;
};

// Device-resident result of a pass: lists in reference order with
// molecule-local 0-based input indices, and per-molecule row offsets.
struct PassOutput {
    uint32_t *d_edges = nullptr, *d_tris = nullptr, *d_tets = nullptr;
    uint64_t n_edges = 0, n_tris = 0, n_tets = 0;
    std::vector<uint64_t> edge_off, tri_off, tet_off;  // n_mol + 1 (host)
    // PassInput::to_host: the lists in the context's pinned host memory
    uint32_t *h_edges = nullptr, *h_tris = nullptr, *h_tets = nullptr;
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    Arena arena;
    pac_options opt{};
    cudaEvent_t ev[16]{};
    int launches = 0;
    // pinned host memory for the lists returned by the host entry points,
    // one region per list (edges, triangles, tetrahedra); each grows, never
    // shrinks, and is reused by every call
    void *pinned[3] = {nullptr, nullptr, nullptr};
    size_t pinned_size[3] = {0, 0, 0};
    // device-to-host copies of the lists run on their own stream, so that a
    // list emitted early crosses PCIe while the later stages compute
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copy_ev[4]{};
    // bytes for the alpha-tetrahedron queue, fixed at the context's first
    // pass (a quarter of the memory free then, at most 12 GiB), so that later
    // passes lay out the pool the same way
    uint64_t queue_bytes = 0;
    Tuner tuner;
};

int union_measure_device(Ctx &ctx, const double4 *d_balls, uint32_t n, const uint32_t *d_edges,
                         uint64_t ne, const uint32_t *d_tris, uint64_t nt, const uint32_t *d_tets,
                         uint64_t nq, double *vol, double *area, double *d_dV, double *d_dA,
                         float *ms);

// Starts copying count words of the device list src into the context's
// pinned region `which` (0 edges, 1 triangles, 2 tetrahedra) on the copy
// stream, after the work queued so far on the context's stream; *dst gets
// the host address (nullptr when count is 0).  The copy is complete once
// copies_join's wait has passed on the context's stream.
int list_to_host_async(Ctx &c, int which, const uint32_t *src, size_t count, uint32_t **dst);
// Makes the context's stream wait for every copy started so far.
int copies_join(Ctx &c);

// Sets the thread-local error detail; returns status.
int set_error(int status, const std::string &msg);

}  // namespace pac

// The context behind a pac_ctx handle (defined in engine.cu).
pac::Ctx &pac_ctx_internal(pac_ctx *ctx);

namespace pac_strict {
int run_pass(pac::Ctx &ctx, const pac::PipelineConfig &cfg, const pac::PassInput &in,
             pac::PassOutput &out, pac_stats *st);
}
namespace pac_fma {
int run_pass(pac::Ctx &ctx, const pac::PipelineConfig &cfg, const pac::PassInput &in,
             pac::PassOutput &out, pac_stats *st);
}
