/*
 * pac.h -- C ABI of the B200 weighted alpha complex engine (libpac.so).
 *
 * The reference (forest113/ParallelAC-xmp) has no library interface: its
 * only boundary is the process CLI
 *     parallelac <crd> <out> <sol-rad> <alpha>              (AlphaComplexParallel.cu:1053-1057)
 *     parallelac-largeData <crd> <out> <sol-rad> <alpha> <chunk-size>
 *                                                           (AlphaComplexLargeData.cu:1049-1058)
 * and each main() runs the whole pipeline inline.  The entry points below
 * are what an FFI (ctypes, cgo, JNI) binds to run that same pipeline without
 * the process boundary; the two CLIs shipped with this library are thin
 * callers of them.  Each declaration names the reference code it replaces.
 *
 * Conventions
 *   - Every entry point returns a pac_status (0 = PAC_OK, negative = error)
 *     and never exits the process.
 *   - A pac_ctx owns one CUDA stream and a device memory pool; it is not
 *     thread-safe.  Use one context per host thread.
 *   - Balls are float4 (x, y, z, raw radius) in input order; the solvent
 *     radius is added on the device (AlphaComplexLargeData.cu:1085).
 *   - Output vertex indices are 0-based input indices.  With
 *     PAC_ORDER_REFERENCE the lists come in the reference binary's file order
 *     (AlphaComplexLargeData.cu:2036-2050); with PAC_ORDER_CANONICAL every
 *     simplex is sorted ascending and each list is sorted lexicographically.
 */
#ifndef PAC_H
#define PAC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PAC_ABI_VERSION 2

typedef enum {
    PAC_OK = 0,
    PAC_ERR_INVALID_ARG = -1, /* null pointer, NaN/inf input, bad option */
    PAC_ERR_CUDA = -2,        /* a CUDA call failed; see pac_last_error() */
    PAC_ERR_CAPACITY = -3,    /* an internal limit was exceeded (e.g. degree) */
    PAC_ERR_TIMEOUT = -4,     /* a bounded device wait gave up */
    PAC_ERR_NO_DEVICE = -5,   /* no CUDA device / extension not usable */
    PAC_ERR_EXACT_RANGE = -6, /* exact arithmetic width exceeded */
    PAC_ERR_OOM = -7,         /* device or host allocation failed */
    PAC_ERR_IO = -8           /* file could not be read or written */
} pac_status;

/* Which of the reference's two formula sets the filters use. */
typedef enum {
    /* AlphaComplexLargeData.cu:167-190, 298-348 (binary parallelac-largeData) */
    PAC_FORMULA_UPSTREAM = 0,
    /* AlphaComplexParallel.cu:203-230, 310-372 (binary parallelac), including
       its division-free edge test and its triangle right-hand side
       `a31*x + a32*y + a33*z*2` (AlphaComplexParallel.cu:344) */
    PAC_FORMULA_PLAIN_XMP = 1
} pac_formula;

/* The empty-orthosphere test of the alpha tetrahedra
   (checkTetsOrthosphere, AlphaComplexLargeData.cu:597-735). */
typedef enum {
    /* Apply it, as the source is written.  This is the weighted alpha
       complex proper. */
    PAC_TETS_AS_WRITTEN = 0,
    /* Skip it, as the reference binary behaves: checkTetsOrthosphere needs
       161 registers per thread for sm_100a and is launched with 512-thread
       blocks (AlphaComplexLargeData.cu:1158, 1492), the launch fails with
       "too many resources requested", the error is only printed
       (AlphaComplexLargeData.cu:51-57), and every alpha-filtered tetrahedron
       is kept.  The shipped golden outputs were produced this way. */
    PAC_TETS_AS_RUN = 1
} pac_tet_mode;

/* Arithmetic of the predicates. */
typedef enum {
    /* Single-precision operations in the reference's order, without FMA
       contraction (= the reference built with nvcc -fmad=false); exact
       simulation of simplicity on an insphere result of exactly zero
       (predicates.h:4669-5462). */
    PAC_PRED_REFCOMPAT = 0,
    /* Same, but every operation that the reference leaves to nvcc's default
       FMA contraction is compiled with contraction enabled (nvcc -fmad=true),
       to follow the reference binary built with default flags. */
    PAC_PRED_REFCOMPAT_FMA = 1,
    /* Exact decisions (no counterpart in the reference, which has no
       working exact fallback): every edge/triangle/tetrahedron alpha test,
       orientation, insphere and attachment test is the exact sign of its
       polynomial in the binary32 inputs, weights (r + sol)^2 taken exactly.
       Each is decided by a double-precision filter with a running error
       bound, and by 640-bit integer arithmetic when the filter cannot tell
       (pac_stats.filter_evals / exact_fallbacks).  Exact zeros of insphere
       go to the simulation of simplicity as in the reference.  Candidate
       sets and windows are the reference's; window centres are computed in
       double precision.  The formula option has no effect.  Inputs whose
       binary exponents span too widely for the integers give
       PAC_ERR_EXACT_RANGE. */
    PAC_PRED_EXACT = 2
} pac_pred_mode;

typedef enum { PAC_ORDER_REFERENCE = 0, PAC_ORDER_CANONICAL = 1 } pac_order;

typedef struct {
    int device;      /* CUDA device ordinal, default 0 */
    int formula;     /* pac_formula, default PAC_FORMULA_UPSTREAM */
    int tet_mode;    /* pac_tet_mode, default PAC_TETS_AS_WRITTEN */
    int predicates;  /* pac_pred_mode, default PAC_PRED_REFCOMPAT */
    int order;       /* pac_order, default PAC_ORDER_REFERENCE */
    /* 1: pick launch shapes by measurement.  The context's first passes
       each try one candidate shape (blocks per SM of the tetrahedron
       enumeration and scan kernels, rows of a large ball per enumeration
       work unit, queue entries a scan warp claims; 12 candidates), timing
       the tetrahedron stage; later passes use the fastest.  Every shape
       gives the same lists, so tuning passes return correct results too. */
    int autotune;
    int verbose;     /* 1: print per-stage timings of each pass and, per chunk of
                        the tetrahedron stage, its counts and times to stderr */
    /* Launch-shape overrides, each used when > 0 (any of them turns the
       autotuner off): reserved_i[0] blocks per SM of the enumeration of
       balls with at most 64 upper neighbours (default 4), [1] of the
       orthosphere scan (4), [2] of the enumeration of larger balls (4),
       [3] rows of a large ball per work unit (8), [4] queue entries a scan
       warp claims (256).
       reserved_i[5] = 1: no early refutation in the enumeration (every
       alpha tetrahedron goes to the scan; same lists).
       reserved_i[6] = 1: verify mode -- the scan also replays the
       reference's arithmetic for every decision the certified filter takes
       and counts disagreements (pac_stats.cert_disagreements; 0 expected).
       reserved_i[7] = W > 1, reserved_i[8] = r: slab r of W of one molecule
       (as written only): the pass outputs the simplices whose smallest
       vertex in cell order lies in the r-th of W contiguous ranges of the
       cell-sorted balls (cut at cell starts), in the reference's order, so
       that the W outputs concatenated in rank order are the whole complex.
       Every rank holds all balls and computes the tetrahedron and triangle
       stages from two cell layers below its range; no data is exchanged.
       The stage counters then count the slab's work, halo included. */
    int reserved_i[9];
    /* reserved_u[0]: if nonzero, the number of alpha tetrahedra the pass
       queues per chunk (default: a quarter of free device memory, at most
       12 GiB, 32 B per entry).  Smaller values force more chunks. */
    uint64_t reserved_u[8];
} pac_options;

typedef struct {
    float x, y, z, r;
} pac_ball;

/* One complex.  on_device says where the three lists live:
     0  host memory allocated by the caller (e.g. for pac_write_complex)
     1  device memory of the context (pac_alpha_complex_device)
     3  pinned host memory of the context (pac_alpha_complex)
   Lists of kinds 1 and 3 belong to the context and stay valid until its next
   call or pac_destroy; copy them to keep them longer.  pac_free_complex()
   resets the struct (and frees nothing for those kinds). */
typedef struct {
    uint32_t n_vertices;
    uint32_t on_device;
    uint64_t n_edges, n_tris, n_tets;
    uint32_t *edges; /* 2 * n_edges */
    uint32_t *tris;  /* 3 * n_tris */
    uint32_t *tets;  /* 4 * n_tets */
} pac_complex;

/* Many molecules: the lists of molecule m are rows [off[m], off[m+1]) of
   the concatenated lists, with molecule-local vertex indices.  The lists are
   context-owned pinned host memory (on_device = 3, valid until the next call);
   the offset arrays are malloc'ed and freed by pac_free_batch_complex(). */
typedef struct {
    uint32_t n_mol;
    uint32_t on_device;
    uint64_t *edge_off, *tri_off, *tet_off; /* n_mol + 1 each (host) */
    uint32_t *edges, *tris, *tets;
} pac_batch_complex;

/* Stage counters and timings (filled when a non-null pointer is passed). */
typedef struct {
    uint64_t n_balls, n_cells;
    uint64_t cand_edges, alpha_edges;
    uint64_t cand_tris, alpha_tris;
    uint64_t cand_tets, alpha_tets;
    uint64_t final_edges, final_tris, final_tets;
    uint64_t insphere_evals;  /* insphere_w evaluations (as-written mode) */
    uint64_t sos_calls;       /* insphere results of exactly 0 -> SoS */
    uint64_t exact_fallbacks; /* exact-mode: filter failures -> exact kernel */
    uint64_t filter_evals;    /* exact-mode: filtered decisions */
    uint64_t ortho_out_of_grid; /* window centres outside the grid */
    uint64_t max_degree;
    /* stage times (CUDA events).  The host entry points copy each list to
       host memory as soon as it is emitted, on a second stream, while the
       later stages run: ms_d2h is the part of those copies that was left
       after the last kernel. */
    double ms_total, ms_h2d, ms_grid, ms_edges, ms_tris, ms_tets, ms_tri_attach,
        ms_edge_attach, ms_emit, ms_d2h;
    uint64_t bytes_model; /* algorithmic bytes of the pass */
    uint32_t grid[3];
    float step;
    uint32_t kernels_launched;
    /* as-written tetrahedra (ABI version 2): alpha tetrahedra refuted inside
       the enumeration by the best other candidate of their triangle group,
       and the tests made there; orthosphere-scan decisions taken by the
       certified filter (the rest replay the reference's arithmetic), and in
       verify mode the certified decisions the replay disagrees with */
    uint64_t early_refuted, early_tests;
    uint64_t cert_decisions, cert_disagreements;
    /* the part of ms_tets spent in the empty-orthosphere test (the scan and
       the simulation-of-simplicity kernel): the reference's "AC2 test for
       tetrahedra" phase (AlphaComplexLargeData.cu:2014) */
    double ms_tet_orthosphere;
} pac_stats;

/* Version of this ABI (PAC_ABI_VERSION). */
int pac_abi_version(void);

/* Defaults: device 0, upstream formulas, as-written tets, ref-compat
   predicates, reference order. */
void pac_default_options(pac_options *opt);

/* Create / destroy a context.  Replaces the implicit CUDA context, the
   initialize<<<1,1>>>() exactinit() launch and the Thrust allocations of
   AlphaComplexLargeData.cu:1145-1155. */
typedef struct pac_ctx pac_ctx;
int pac_create(pac_ctx **ctx, const pac_options *opt);
int pac_destroy(pac_ctx *ctx);

/* The cudaStream_t (as void*) this context launches on, so a caller can
   order its own work, or record timing events, against the engine's.  No
   reference counterpart (the reference uses the default stream). */
void *pac_cuda_stream(pac_ctx *ctx);

/* Weighted alpha complex of one molecule, host buffers in and out.
   Replaces the pipeline of AlphaComplexParallel.cu:1119-1807 and
   AlphaComplexLargeData.cu:1119-2001 (grid, candidate enumeration, the
   power/orientation/attachment filters and the set differences), run as a
   single device pass without the chunk loop.
   balls: n host balls; sol_rad and alpha as on the reference command line
   (AlphaComplexLargeData.cu:1076-1077). */
int pac_alpha_complex(pac_ctx *ctx, const pac_ball *balls, uint32_t n,
                      float sol_rad, float alpha, pac_complex *out,
                      pac_stats *stats);

/* Same with device-resident input and output (d_balls is a device pointer;
   out->on_device = 1).  Nothing crosses PCIe except a few counters.  The
   engine launches on its own stream (pac_cuda_stream), which does not wait
   for work on other streams: device inputs must be complete when a device
   entry point is called (synchronise, or record an event and make the
   engine's stream wait on it). */
int pac_alpha_complex_device(pac_ctx *ctx, const pac_ball *d_balls,
                             uint32_t n, float sol_rad, float alpha,
                             pac_complex *out, pac_stats *stats);

/* Many independent molecules in one device pass.  balls holds the molecules
   back to back; offsets has n_mol + 1 entries (offsets[0] = 0).  Replaces
   running the reference binary once per molecule. */
int pac_alpha_complex_batch(pac_ctx *ctx, const pac_ball *balls,
                            const uint64_t *offsets, uint32_t n_mol,
                            float sol_rad, float alpha, pac_batch_complex *out,
                            pac_stats *stats);

/* Union-of-balls volume and surface area over a fixed complex by
   inclusion-exclusion, with their gradients by a hand-written adjoint.  No
   reference counterpart: the reference computes only the complex.
   xyzr: n x 4 doubles (x, y, z, R) with R the grown radius sqrt(r^2 + alpha)
   of each ball (r including the solvent radius), in input order.  cx: the
   complex of those balls (host lists, or device lists when cx->on_device ==
   1).  vol/area: totals.  dvol/darea: n x 4 doubles (d/dx, d/dy, d/dz,
   d/dR) each, or NULL.  With the weighted alpha complex of the balls at
   alpha (the dual complex of the grown balls) the totals are the exact
   volume and area of the union; in every case they are the inclusion-
   exclusion sums over cx and the gradients are their exact derivatives with
   cx held fixed.  Gradient sums use floating-point atomics: run-to-run
   differences are at rounding level. */
int pac_union_measure(pac_ctx *ctx, const double *xyzr, uint32_t n,
                      const pac_complex *cx, double *vol, double *area,
                      double *dvol, double *darea);

/* Same with device-resident inputs and gradient outputs (d_xyzr, d_dvol,
   d_darea are device pointers; cx must hold device lists, e.g. from
   pac_alpha_complex_device).  vol/area are host pointers. */
int pac_union_measure_device(pac_ctx *ctx, const double *d_xyzr, uint32_t n,
                             const pac_complex *cx, double *vol, double *area,
                             double *d_dvol, double *d_darea);

/* Same measure for callers that cannot allocate device memory (for example
   when a framework's allocator has reserved the GPU's memory, or in a
   latency-bound loop that cannot take cudaMalloc's implicit
   synchronisation).  No counterpart in the reference.  All arguments are as
   for pac_union_measure_device: device balls, a complex with device lists,
   and device gradient buffers -- both or neither; vol/area are host
   pointers.  Nothing is allocated: the only scratch is a fixed 2 MiB array
   inside the library that every GPU loading it holds until exit.
   Limit: sum over the four lists of ceil(count / 128) <= 65,536 (about 8.4
   million simplices); larger complexes return PAC_ERR_CAPACITY.  The first
   call on a device looks up the array's device address; make that first call
   before any stream capture.  All calls share the one array: calls that
   overlap on the GPU (two contexts, two streams) race and must be serialised
   by the caller. */
int pac_union_measure_noalloc(pac_ctx *ctx, const double *d_xyzr, uint32_t n,
                              const pac_complex *cx, double *vol, double *area,
                              double *d_dvol, double *d_darea);

void pac_free_complex(pac_complex *cx);
void pac_free_batch_complex(pac_batch_complex *cx);

/* Read a CRD file (count, then x y z r per line, parsed as %f).
   Replaces AlphaComplexLargeData.cu:1067-1112.  *balls is malloc'ed. */
int pac_read_crd(const char *path, pac_ball **balls, uint32_t *n);

/* Write the reference's output file format (AlphaComplexLargeData.cu:2028-2050):
   header "V E T Tet", V lines "%9.5lf" x4 (radius including sol_rad), then
   the edge, triangle and tetrahedron lines with "%9d" fields. */
int pac_write_complex(const char *path, const pac_ball *balls, uint32_t n,
                      float sol_rad, const pac_complex *cx);

const char *pac_status_string(int status);
/* Detail of the last error on this host thread ("" if none). */
const char *pac_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* PAC_H */
