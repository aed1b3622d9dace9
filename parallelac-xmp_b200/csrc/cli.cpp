// cli.cpp -- the reference's two command lines on top of libpac:
//   parallelac <crd-file> <out-file> <sol-rad> <alpha>
//       (AlphaComplexParallel.cu:1053-1057; plain-xmp formulas)
//   parallelac-largeData <crd-file> <out-file> <sol-rad> <alpha> <chunk-size>
//       (AlphaComplexLargeData.cu:1049-1058; upstream formulas; the chunk size
//        is accepted and reported, the pass itself is never chunked)
// Same argument checks, exit codes, stdout report and output file.  Two
// environment variables choose what the positional interface cannot:
//   PAC_TET_MODE   = as-run (default: the reference binary's output) | as-written
//   PAC_PREDICATES = strict (default) | fma | exact
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/pac.h"

#ifdef PAC_CLI_LARGEDATA
static const int kArgs = 6;
static const char *kUsage =
    "Usage : parallelac-largeData <crd-file> <out-file> <sol-rad> <alpha> <chunk-size>\n";
#else
static const int kArgs = 5;
static const char *kUsage = "Usage : parallelac <crd-file> <out-file> <sol-rad> <alpha>\n";
#endif

int main(int argc, char **argv) {
    if (argc < kArgs) {
        std::printf("%s", kUsage);
        return 1;
    }
    pac_ball *balls = nullptr;
    uint32_t n = 0;
    int rc = pac_read_crd(argv[1], &balls, &n);
    if (rc) {
        std::fprintf(stderr, "parallelac: %s (%s)\n", pac_status_string(rc), pac_last_error());
        return 1;
    }
    float solventRadius = (float)std::atof(argv[3]);
    float alpha = (float)std::atof(argv[4]);
    std::printf("Successfully read the file %s ...\n", argv[1]);
    std::printf(
        "The given file has %d atoms. \n\nStarting alpha complex computation for "
        "alpha = %.3f and solvent radius = %.3f ...\n\n",
        (int)n, alpha, solventRadius);
#ifdef PAC_CLI_LARGEDATA
    // the reference's chunk (512 doubled up to the suggestion) and its
    // per-chunk progress line (AlphaComplexLargeData.cu:1227-1235); the pass
    // itself is one device pass whatever the chunk
    {
        const int suggestion = std::atoi(argv[5]);
        long long chunk = 512;
        while (chunk < suggestion) chunk *= 2;
        for (long long start = 0; start < (long long)n; start += chunk)
            std::printf("Processed %lld atoms ... \n", start);
    }
#endif
    pac_options opt;
    pac_default_options(&opt);
#ifdef PAC_CLI_LARGEDATA
    opt.formula = PAC_FORMULA_UPSTREAM;
#else
    opt.formula = PAC_FORMULA_PLAIN_XMP;
#endif
    const char *tm = std::getenv("PAC_TET_MODE");
    opt.tet_mode = (tm && std::strcmp(tm, "as-written") == 0) ? PAC_TETS_AS_WRITTEN : PAC_TETS_AS_RUN;
    const char *pm = std::getenv("PAC_PREDICATES");
    opt.predicates = (pm && std::strcmp(pm, "fma") == 0)     ? PAC_PRED_REFCOMPAT_FMA
                     : (pm && std::strcmp(pm, "exact") == 0) ? PAC_PRED_EXACT
                                                             : PAC_PRED_REFCOMPAT;
    pac_ctx *ctx = nullptr;
    rc = pac_create(&ctx, &opt);
    pac_complex cx;
    pac_stats st;
    if (!rc) rc = pac_alpha_complex(ctx, balls, n, solventRadius, alpha, &cx, &st);
    if (rc) {
        std::fprintf(stderr, "parallelac: %s (%s)\n", pac_status_string(rc), pac_last_error());
        pac_destroy(ctx);
        std::free(balls);
        return 1;
    }
    std::printf("Alpha complex computed.\n\n");
    std::printf("Number of vertices: %15d\n", (int)n);
    std::printf("Number of edges: %18ld\n", (long)cx.n_edges);
    std::printf("Number of triangles: %14ld\n", (long)cx.n_tris);
    std::printf("Number of tetrahedra: %13ld\n", (long)cx.n_tets);
    std::printf("Total simplices: %18ld\n", (long)(n + cx.n_edges + cx.n_tris + cx.n_tets));
    std::printf(
        "\nTime taken (ms):\nData transfer: %20.3f\nGrid computation: %17.3f\nPotential edges: %18.3f\n"
        "Potential triangles: %14.3f\nPotential tetrahedra: %13.3f\nAC2 test for tetrahedra: %10.3f\n"
        "AC2 test for triangles: %11.3f\nAC2 test for edges: %15.3f\n",
        st.ms_h2d + st.ms_d2h + st.ms_emit, st.ms_grid, st.ms_edges, st.ms_tris,
        st.ms_tets - st.ms_tet_orthosphere, st.ms_tet_orthosphere, st.ms_tri_attach,
        st.ms_edge_attach);
    std::printf("Total time taken (ms): %12.3f\n", st.ms_total);
    std::printf("\nWriting computed alpha complex to the file %s ...\n", argv[2]);
    rc = pac_write_complex(argv[2], balls, n, solventRadius, &cx);
    if (rc) std::fprintf(stderr, "parallelac: %s (%s)\n", pac_status_string(rc), pac_last_error());
    pac_free_complex(&cx);
    pac_destroy(ctx);
    std::free(balls);
    return rc ? 1 : 0;
}
