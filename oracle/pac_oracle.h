/*
 * pac_oracle.h -- CPU restatement of the ParallelAC weighted alpha complex
 * pipeline.  TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the
 * bench's CPU-baseline leg link this library as the checker.  The product
 * path (libpac) never calls it.
 *
 * The restatement follows AlphaComplexLargeData.cu (formula variant
 * ORC_UPSTREAM) and AlphaComplexParallel.cu (variant ORC_PLAIN_XMP), with
 * every single-precision operation performed in the reference's order and
 * without contraction (build with -ffp-contract=off).  Exact predicates
 * (the SoS fallback of predicates.h:4669-5462) use multi-word integers.
 */
#ifndef PAC_ORACLE_H
#define PAC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_UPSTREAM = 0, ORC_PLAIN_XMP = 1 };

/* flags */
enum {
    /* Apply the empty-orthosphere test to the alpha tetrahedra
       (checkTetsOrthosphere, LD:597-735) as the source is written.  Without
       this flag the restatement follows the reference binary as it runs:
       that kernel needs more registers than a 512-thread block can hold
       (161 per thread for sm_100a), its launch fails, and every
       alpha-filtered tetrahedron is kept. */
    ORC_TET_ORTHO = 1,
    /* Decision-exact predicates: every edge/triangle/tetrahedron alpha
       test, orientation, insphere and attachment test is the exact sign of
       its polynomial in the binary32 inputs (weights r^2 exact), evaluated
       in multi-word integers; windows are centred at FP64 orthocentres.
       The formula variant does not matter in this mode.  status = -6 when
       an input's range exceeds the integers' width. */
    ORC_EXACT = 2
};

typedef struct {
    /* final complex in the reference binary's output order, 0-based
       original indices (AlphaComplexLargeData.cu:2036-2050) */
    uint64_t n_edges, n_tris, n_tets;
    uint32_t *edges; /* 2 per edge */
    uint32_t *tris;  /* 3 per triangle */
    uint32_t *tets;  /* 4 per tetrahedron */
    /* stage counts */
    uint64_t cand_edges, alpha_edges;
    uint64_t cand_tris, alpha_tris;
    uint64_t cand_tets, alpha_tets;
    uint64_t tris_in_tets, edges_in_tris;
    uint64_t insphere_evals, sos_calls, sos_exhausted;
    uint64_t ortho_out_of_grid;
    int32_t grid[3];
    float step;
    int status; /* 0 ok, <0 error */
} orc_result;

/* xyzr: n x 4 floats (x, y, z, raw radius) in input order. */
int orc_alpha_complex(const float *xyzr, uint32_t n, float sol_rad,
                      float alpha, int variant, int flags, int threads,
                      orc_result *res);
void orc_free(orc_result *res);

/* Single predicates, exposed so the tests can pin them against the
   reference's own predicates.h compiled for the host. */
float orc_orient3d(const float *pa, const float *pb, const float *pc,
                   const float *pd);
float orc_insphere_w(const float *pa, const float *pb, const float *pc,
                     const float *pd, const float *pe, float wa, float wb,
                     float wc, float wd, float we);
/* Single decision-exact predicates on balls (x, y, z, r) with weights
   r^2 (see ORC_EXACT): kind 0 edge alpha (2 balls), 1 triangle alpha (3),
   2 tetrahedron alpha (4; 2 when flat), 3 orient3d sign (4), 4 insphere
   sign (5), 5 edge attached by the last ball (3), 6 triangle attached by
   the last ball (4).  Returns the decision (0/1/2) or the sign. */
int orc_exact_pred(int kind, const float *balls, float alpha);

/* returns the SoS sign (+1/-1); *depth receives the SoS depth reached */
int orc_sos4(const float *p0, const float *p1, const float *p2,
             const float *p3, const float *p4, float w0, float w1, float w2,
             float w3, float w4, int i0, int i1, int i2, int i3, int i4,
             int *depth);

/* FP64 union-of-balls volume and area over a fixed complex by
   inclusion-exclusion, gradients by forward-mode automatic differentiation
   (union_oracle.cpp).  xyzr: n x 4 (x, y, z, radius); dvol/darea: n x 4. */
int orc_union_measure(const double *xyzr, uint32_t n, const uint32_t *edges,
                      uint64_t ne, const uint32_t *tris, uint64_t nt,
                      const uint32_t *tets, uint64_t nq, double *vol,
                      double *area, double *dvol, double *darea);

#ifdef __cplusplus
}
#endif
#endif
