/*
 * synth.c -- seeded synthetic molecule generators for the benchmark and
 * parity workloads (host code, C99).
 *
 * A molecule is a self-avoiding random walk with 1.5 A steps whose atoms
 * keep at least 1.2 A from every non-bonded atom, confined by rejection to
 * a ball (or a cube) sized for 0.05 atoms/A^3.  Radii are drawn from the
 * C/N/O/S set {1.70, 1.55, 1.52, 1.80} with p = {0.63, 0.17, 0.19, 0.01}.
 * Coordinates are generated in double and stored as float.  The random
 * stream is splitmix64, so the same seed gives the same balls everywhere.
 *
 * Output layout: n x float4 (x, y, z, raw radius) -- the layout the engine
 * takes as input.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint64_t s;
} rng_t;

static uint64_t rng_next(rng_t *r) {
    uint64_t z = (r->s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double rng_unit(rng_t *r) { return (double)(rng_next(r) >> 11) * 0x1.0p-53; }

static void rng_dir(rng_t *r, double *d) {
    double z = 2.0 * rng_unit(r) - 1.0;
    double phi = 6.283185307179586 * rng_unit(r);
    double s = sqrt(fmax(0.0, 1.0 - z * z));
    d[0] = s * cos(phi);
    d[1] = s * sin(phi);
    d[2] = z;
}

static float pick_radius(rng_t *r) {
    double u = rng_unit(r);
    if (u < 0.63) return 1.70f;
    if (u < 0.80) return 1.55f;
    if (u < 0.99) return 1.52f;
    return 1.80f;
}

/* spatial hash of placed atoms, cell = 1.2 A */
typedef struct {
    int64_t *head;
    int64_t *next;
    uint64_t mask;
} hgrid;

static uint64_t hkey(int64_t a, int64_t b, int64_t c) {
    uint64_t h = (uint64_t)a * 73856093ull ^ (uint64_t)b * 19349663ull ^
                 (uint64_t)c * 83492791ull;
    return h * 0x9E3779B97F4A7C15ull;
}

#define SEP 1.2
#define STEP 1.5

static int too_close(const hgrid *g, const double *pos, const double *p,
                     int64_t skip) {
    int64_t cx = (int64_t)floor(p[0] / SEP), cy = (int64_t)floor(p[1] / SEP),
            cz = (int64_t)floor(p[2] / SEP);
    for (int i = -1; i <= 1; i++)
        for (int j = -1; j <= 1; j++)
            for (int k = -1; k <= 1; k++) {
                uint64_t h = hkey(cx + i, cy + j, cz + k) & g->mask;
                for (int64_t a = g->head[h]; a >= 0; a = g->next[a]) {
                    if (a == skip) continue;
                    double dx = pos[3 * a] - p[0], dy = pos[3 * a + 1] - p[1],
                           dz = pos[3 * a + 2] - p[2];
                    if (dx * dx + dy * dy + dz * dz < SEP * SEP) return 1;
                }
            }
    return 0;
}

static void hinsert(hgrid *g, const double *p, int64_t a) {
    int64_t cx = (int64_t)floor(p[0] / SEP), cy = (int64_t)floor(p[1] / SEP),
            cz = (int64_t)floor(p[2] / SEP);
    uint64_t h = hkey(cx, cy, cz) & g->mask;
    g->next[a] = g->head[h];
    g->head[h] = a;
}

/* shape: 0 = ball of radius `extent`, 1 = cube of half-side `extent` */
static int inside(const double *p, int shape, double extent) {
    if (shape == 0) return p[0] * p[0] + p[1] * p[1] + p[2] * p[2] <= extent * extent;
    return fabs(p[0]) <= extent && fabs(p[1]) <= extent && fabs(p[2]) <= extent;
}

static void random_inside(rng_t *r, int shape, double extent, double *p) {
    do {
        for (int k = 0; k < 3; k++) p[k] = (2.0 * rng_unit(r) - 1.0) * extent;
    } while (!inside(p, shape, extent));
}

/* One globule of n balls centred at c. Returns 0 on success. */
static int walk(uint64_t seed, uint32_t n, int shape, double extent,
                const double *c, float *out) {
    rng_t r = {seed};
    double *pos = (double *)malloc(sizeof(double) * 3 * (n ? n : 1));
    uint64_t cap = 1;
    while (cap < 2ull * n) cap <<= 1;
    hgrid g;
    g.head = (int64_t *)malloc(sizeof(int64_t) * cap);
    g.next = (int64_t *)malloc(sizeof(int64_t) * (n ? n : 1));
    g.mask = cap - 1;
    if (!pos || !g.head || !g.next) {
        free(pos); free(g.head); free(g.next);
        return -1;
    }
    for (uint64_t i = 0; i < cap; i++) g.head[i] = -1;
    double p[3] = {0, 0, 0};
    for (uint32_t a = 0; a < n; a++) {
        double q[3];
        int ok = 0;
        if (a > 0) {
            for (int t = 0; t < 64 && !ok; t++) {
                double d[3];
                rng_dir(&r, d);
                for (int k = 0; k < 3; k++) q[k] = p[k] + STEP * d[k];
                ok = inside(q, shape, extent) && !too_close(&g, pos, q, (int64_t)a - 1);
            }
        }
        while (!ok) { /* chain break: restart somewhere free */
            random_inside(&r, shape, extent, q);
            ok = !too_close(&g, pos, q, -1);
        }
        memcpy(&pos[3 * a], q, sizeof(q));
        hinsert(&g, q, a);
        memcpy(p, q, sizeof(q));
        out[4 * a + 0] = (float)(q[0] + c[0]);
        out[4 * a + 1] = (float)(q[1] + c[1]);
        out[4 * a + 2] = (float)(q[2] + c[2]);
        out[4 * a + 3] = pick_radius(&r);
    }
    free(pos); free(g.head); free(g.next);
    return 0;
}

static double globule_radius(uint32_t n) {
    return cbrt(3.0 * (double)n / (4.0 * 3.141592653589793 * 0.05));
}

/* A compact globule of n balls at the origin (the base generator). */
int pac_synth_globule(uint64_t seed, uint32_t n, float *out) {
    double c[3] = {0, 0, 0};
    return walk(seed, n, 0, globule_radius(n), c, out);
}

/* Globule snapped to a `grid` A lattice with radii quantised to `rq` A. */
int pac_synth_snapped(uint64_t seed, uint32_t n, double grid, double rq,
                      float *out) {
    int rc = pac_synth_globule(seed, n, out);
    if (rc) return rc;
    for (uint32_t a = 0; a < n; a++) {
        for (int k = 0; k < 3; k++)
            out[4 * a + k] = (float)(nearbyint((double)out[4 * a + k] / grid) * grid);
        out[4 * a + 3] = (float)(nearbyint((double)out[4 * a + 3] / rq) * rq);
    }
    return 0;
}

/* nx*ny*nz globules of `per` balls, each confined to a cube of side
   `side`, centred on a lattice of pitch `pitch` around the origin. */
int pac_synth_assembly(uint64_t seed, uint32_t nx, uint32_t ny, uint32_t nz,
                       uint32_t per, double pitch, double side, float *out) {
    uint64_t g = 0;
    for (uint32_t k = 0; k < nz; k++)
        for (uint32_t j = 0; j < ny; j++)
            for (uint32_t i = 0; i < nx; i++, g++) {
                double c[3] = {((double)i - 0.5 * (nx - 1)) * pitch,
                               ((double)j - 0.5 * (ny - 1)) * pitch,
                               ((double)k - 0.5 * (nz - 1)) * pitch};
                int rc = walk(seed * 1000003ull + g, per, 1, 0.5 * side, c,
                              out + 4 * per * g);
                if (rc) return rc;
            }
    return 0;
}

/* Sizes of a batch of `count` molecules, log-uniform in [lo, hi]. */
int pac_synth_batch_sizes(uint64_t seed, uint32_t count, uint32_t lo,
                          uint32_t hi, uint32_t *sizes) {
    rng_t r = {seed};
    double a = log((double)lo), b = log((double)hi);
    for (uint32_t i = 0; i < count; i++) {
        uint32_t s = (uint32_t)floor(exp(a + (b - a) * rng_unit(&r)));
        sizes[i] = s < lo ? lo : (s > hi ? hi : s);
    }
    return 0;
}

/* The batch itself: molecule i is a globule with seed (seed, i). */
int pac_synth_batch(uint64_t seed, uint32_t count, const uint32_t *sizes,
                    float *out) {
    uint64_t off = 0;
    for (uint32_t i = 0; i < count; i++) {
        int rc = pac_synth_globule(seed * 1000003ull + i + 1, sizes[i], out + 4 * off);
        if (rc) return rc;
        off += sizes[i];
    }
    return 0;
}

#ifdef __cplusplus
}
#endif
