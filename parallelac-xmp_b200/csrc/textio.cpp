// Text input and output of the reference's file formats, formatted and
// parsed on all host threads.
//
// Output (AlphaComplexLargeData.cu:2028-2050): a header "V E T Tet", V ball
// lines "%9.5lf %9.5lf %9.5lf %9.5lf" (radius including the solvent radius),
// then the edge, triangle and tetrahedron lines with "%9d" fields.  The
// reference writes them with one fprintf per line; here blocks of lines are
// formatted in parallel into per-thread buffers and written in order, so the
// file is byte for byte what printf gives.  The fixed-point conversion is
// exact: a float is M * 2^E with a 24-bit M, so round(|x| * 10^5) is an
// integer division of M * 10^5 by a power of two, rounded half to even on
// the exact value as glibc's printf rounds; values too large for that (|x| of
// 2^40 and more) and non-finite values go through snprintf.
//
// Input (AlphaComplexLargeData.cu:1067-1112): the count, then 4 * count
// whitespace-separated numbers read with "%f".  The body is split at
// whitespace into one range per thread; the tokens of each range are counted,
// a prefix sum places them, and each token is converted with strtof (the
// conversion scanf's %f performs).
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "pac.h"

namespace pac {
int set_error(int status, const std::string &msg);
}

namespace {

int io_threads() {
    unsigned t = std::thread::hardware_concurrency();
    if (t == 0) t = 1;
    if (t > 32) t = 32;
    return (int)t;
}

// Run body(t) for t in [0, T) on T threads (the calling thread takes t = 0).
template <class F>
void run_threads(int T, F body) {
    std::vector<std::thread> th;
    th.reserve(T > 1 ? T - 1 : 0);
    for (int t = 1; t < T; t++) th.emplace_back(body, t);
    body(0);
    for (auto &x : th) x.join();
}

// "%9d": right-aligned in 9 columns, wider when needed.
inline int put_int9(char *o, int v) {
    char d[12];
    int n = 0;
    uint32_t u = v < 0 ? 0u - (uint32_t)v : (uint32_t)v;
    do {
        d[n++] = (char)('0' + u % 10);
        u /= 10;
    } while (u);
    const int w = n + (v < 0);
    int k = 0;
    for (int i = w; i < 9; i++) o[k++] = ' ';
    if (v < 0) o[k++] = '-';
    while (n) o[k++] = d[--n];
    return k;
}

// "%9.5lf" of a float widened to double.
inline int put_fixed5(char *o, float f) {
    uint32_t bits;
    std::memcpy(&bits, &f, 4);
    const bool neg = bits >> 31;
    const int ex = (int)((bits >> 23) & 0xff);
    const uint32_t frac = bits & 0x7fffff;
    if (ex == 0xff || ex >= 127 + 40) {  // non-finite or |f| >= 2^40
        char tmp[64];
        int n = std::snprintf(tmp, sizeof(tmp), "%9.5lf", (double)f);
        std::memcpy(o, tmp, (size_t)n);
        return n;
    }
    // |f| = M * 2^E
    const uint64_t M = ex ? (frac | 0x800000u) : frac;
    const int E = ex ? ex - 150 : -149;
    const uint64_t P = M * 100000ull;  // < 2^41
    uint64_t N;                        // round_half_even(|f| * 10^5)
    if (E >= 0) {
        N = P << E;  // E < 17 here: < 2^58
    } else {
        const int s = -E;
        if (s >= 64) {
            N = 0;  // P < 2^41 < 2^(s-1): below one half
        } else {
            const uint64_t q = P >> s, r = P & ((1ull << s) - 1), half = 1ull << (s - 1);
            N = q + ((r > half || (r == half && (q & 1))) ? 1 : 0);
        }
    }
    const uint64_t ip = N / 100000ull, fp = N % 100000ull;
    char d[24];
    int n = 0;
    uint64_t u = ip;
    do {
        d[n++] = (char)('0' + u % 10);
        u /= 10;
    } while (u);
    const int w = (int)neg + n + 6;  // sign, integer digits, '.', 5 digits
    int k = 0;
    for (int i = w; i < 9; i++) o[k++] = ' ';
    if (neg) o[k++] = '-';
    while (n) o[k++] = d[--n];
    o[k++] = '.';
    uint64_t g = fp;
    for (int i = 4; i >= 0; i--) {
        o[k + i] = (char)('0' + g % 10);
        g /= 10;
    }
    return k + 5;
}

}  // namespace

namespace {

constexpr uint64_t kLinesPerTask = 1 << 16;

// Writes count lines, line i formatted by fmt(i, dst) (at most max_line
// characters), T * kLinesPerTask lines at a time: each thread formats its
// share into its own buffer, then the buffers are written in order.
template <class F>
bool write_lines(FILE *fp, uint64_t count, int max_line, int T, F fmt) {
    std::vector<std::vector<char>> buf(T);
    std::vector<size_t> used(T);
    for (uint64_t base = 0; base < count; base += (uint64_t)T * kLinesPerTask) {
        const uint64_t tasks = (count - base + kLinesPerTask - 1) / kLinesPerTask;
        const int Tb = tasks < (uint64_t)T ? (int)tasks : T;
        for (int t = Tb; t < T; t++) used[t] = 0;
        run_threads(Tb, [&](int t) {
            const uint64_t lo = base + (uint64_t)t * kLinesPerTask;
            const uint64_t hi = lo + kLinesPerTask < count ? lo + kLinesPerTask : count;
            used[t] = 0;
            if (lo >= hi) return;
            std::vector<char> &b = buf[t];
            if (b.size() < (size_t)(hi - lo) * (size_t)max_line) b.resize((size_t)(hi - lo) * max_line);
            char *o = b.data();
            for (uint64_t i = lo; i < hi; i++) o += fmt(i, o);
            used[t] = (size_t)(o - b.data());
        });
        for (int t = 0; t < T; t++)
            if (used[t] && std::fwrite(buf[t].data(), 1, used[t], fp) != used[t]) return false;
    }
    return true;
}

bool is_space(char c) {
    return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f';
}

}  // namespace

extern "C" {

int pac_write_complex(const char *path, const pac_ball *balls, uint32_t n, float sol_rad,
                      const pac_complex *cx) {
    if (!path || !cx || (n && !balls)) return pac::set_error(PAC_ERR_INVALID_ARG, "null argument");
    if (cx->on_device == 1)
        return pac::set_error(PAC_ERR_INVALID_ARG, "complex lists are in device memory");
    FILE *fp = std::fopen(path, "w");
    if (!fp) return pac::set_error(PAC_ERR_IO, std::string("cannot create ") + path);
    const int T = io_threads();
    bool ok = std::fprintf(fp, "%d %ld %ld %ld\n", (int)n, (long)cx->n_edges, (long)cx->n_tris,
                           (long)cx->n_tets) > 0;
    ok = ok && write_lines(fp, n, 4 * 64, T, [&](uint64_t i, char *o) {
        const pac_ball &b = balls[i];
        const float r = b.r + sol_rad;
        int k = put_fixed5(o, b.x);
        o[k++] = ' ';
        k += put_fixed5(o + k, b.y);
        o[k++] = ' ';
        k += put_fixed5(o + k, b.z);
        o[k++] = ' ';
        k += put_fixed5(o + k, r);
        o[k++] = '\n';
        return k;
    });
    const uint32_t *E = cx->edges, *Tr = cx->tris, *Q = cx->tets;
    ok = ok && write_lines(fp, cx->n_edges, 2 * 12, T, [&](uint64_t i, char *o) {
        int k = put_int9(o, (int)E[2 * i]);
        o[k++] = ' ';
        k += put_int9(o + k, (int)E[2 * i + 1]);
        o[k++] = '\n';
        return k;
    });
    ok = ok && write_lines(fp, cx->n_tris, 3 * 12, T, [&](uint64_t i, char *o) {
        int k = 0;
        for (int j = 0; j < 3; j++) {
            k += put_int9(o + k, (int)Tr[3 * i + j]);
            o[k++] = j < 2 ? ' ' : '\n';
        }
        return k;
    });
    ok = ok && write_lines(fp, cx->n_tets, 4 * 12, T, [&](uint64_t i, char *o) {
        int k = 0;
        for (int j = 0; j < 4; j++) {
            k += put_int9(o + k, (int)Q[4 * i + j]);
            o[k++] = j < 3 ? ' ' : '\n';
        }
        return k;
    });
    const bool bad = std::ferror(fp) != 0;
    if (std::fclose(fp) != 0 || bad || !ok)
        return pac::set_error(PAC_ERR_IO, std::string("write failed: ") + path);
    return PAC_OK;
}

int pac_read_crd(const char *path, pac_ball **balls, uint32_t *n) {
    if (!path || !balls || !n) return pac::set_error(PAC_ERR_INVALID_ARG, "null argument");
    *balls = nullptr;
    *n = 0;
    FILE *f = std::fopen(path, "rb");
    if (!f) return pac::set_error(PAC_ERR_IO, std::string("cannot open ") + path);
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<char> buf((size_t)(sz > 0 ? sz : 0) + 1);
    const size_t got = std::fread(buf.data(), 1, (size_t)(sz > 0 ? sz : 0), f);
    std::fclose(f);
    buf[got] = 0;
    char *p = buf.data(), *end = nullptr;
    errno = 0;
    const long cnt = std::strtol(p, &end, 10);
    if (end == p || cnt < 0 || cnt > 0xfffffffeL)
        return pac::set_error(PAC_ERR_IO, std::string("bad ball count in ") + path);
    const uint64_t want = 4ull * (uint64_t)cnt;
    pac_ball *b = (pac_ball *)std::malloc(sizeof(pac_ball) * (size_t)(cnt ? cnt : 1));
    if (!b) return pac::set_error(PAC_ERR_OOM, "host allocation failed");
    // the body [end, stop), split at whitespace into one range per thread
    const char *body = end, *stop = buf.data() + got;
    const size_t len = (size_t)(stop - body);
    int T = io_threads();
    if (len < ((size_t)1 << 20)) T = 1;
    std::vector<const char *> cut(T + 1);
    cut[0] = body;
    cut[T] = stop;
    for (int t = 1; t < T; t++) {
        const char *c = body + len * (size_t)t / (size_t)T;
        if (c < cut[t - 1]) c = cut[t - 1];
        while (c < stop && !is_space(*c)) c++;  // no token is split
        cut[t] = c;
    }
    // tokens per range, then their first index
    std::vector<uint64_t> ntok(T + 1, 0);
    run_threads(T, [&](int t) {
        uint64_t k = 0;
        bool in = false;
        for (const char *c = cut[t]; c < cut[t + 1]; c++) {
            const bool sp = is_space(*c);
            if (!sp && !in) k++;
            in = !sp;
        }
        ntok[t + 1] = k;
    });
    for (int t = 0; t < T; t++) ntok[t + 1] += ntok[t];
    // convert; the first malformed token of each range is recorded
    std::vector<uint64_t> badtok(T, UINT64_MAX);
    run_threads(T, [&](int t) {
        uint64_t k = ntok[t];
        const char *c = cut[t];
        while (k < want) {
            while (c < cut[t + 1] && is_space(*c)) c++;
            if (c >= cut[t + 1]) break;
            const char *e = c;
            while (e < cut[t + 1] && !is_space(*e)) e++;
            char *ce = nullptr;
            const float v = std::strtof(c, &ce);
            if (ce != e) {  // not a whole number token
                badtok[t] = k;
                break;
            }
            (&b[k >> 2].x)[k & 3] = v;
            k++;
            c = e;
        }
    });
    uint64_t bad = ntok[T] < want ? ntok[T] : want;
    for (int t = 0; t < T; t++)
        if (badtok[t] < bad) bad = badtok[t];
    if (bad < want) {
        std::free(b);
        return pac::set_error(PAC_ERR_IO, std::string(path) + ": ball " + std::to_string(bad / 4) +
                                              " is truncated or malformed");
    }
    *balls = b;
    *n = (uint32_t)cnt;
    return PAC_OK;
}

}  // extern "C"
