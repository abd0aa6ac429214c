// generators.cpp — seeded synthetic CSR matrices for the benchmark and test
// configurations (libsbbgen.so; host code, OpenMP).
//
// Every row draws from its own splitmix64 stream keyed by (seed, row), so a
// matrix is identical whatever the thread count.  Generation is two passes:
// pass 1 builds each row to learn its length (row pointer by prefix sum),
// pass 2 rebuilds the row from the same stream and writes it.  Columns are
// sorted and distinct within a row.
//
// The reference's own datasets (SuiteSparse circuit5M, rail4284) are not
// available here; these families stand in for them with their shapes.
#include <omp.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

inline uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t s;
    Rng(uint64_t seed, uint64_t stream) : s(mix64(seed * 0xD1B54A32D192ED03ull ^ mix64(stream))) {}
    uint64_t next()
    {
        s += 0x9E3779B97F4A7C15ull;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uni() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
    long long below(long long n) { return (long long)(uni() * (double)n); }       // [0,n)
};

}  // namespace

extern "C" {

// Family ids.
enum {
    GEN_POWERLAW = 1,   // C1: L ~ density L^-expo on [1, lmax], floor; uniform columns
    GEN_CIRCUIT = 2,    // C2: diag + band(+-hw, keep p) + ceil(Pareto) long range + dense rows
    GEN_SHORTWIDE = 3,  // C3: lognormal L, runs inside 64-aligned column blocks, val = 1
    GEN_BANDED = 4,     // C5 banded: window [i-hw, i+hw]
    GEN_PLFAMILY = 5,   // C5 power-law rows with mean ~ r
    GEN_BLOCKDIAG = 6,  // C5 block-diagonal
    GEN_UNIFORM = 7,    // tests: L uniform in [lmin, lmax], optional empty rows
};

typedef struct {
    unsigned long long seed;
    int family;
    int m, n;
    double expo;       // power-law exponent (density ~ L^-expo)
    double lmin, lmax; // row-length bounds
    double p;          // band keep probability (circuit)
    int hw;            // band half-width
    int block;         // block size (block-diag)
    double r;          // target mean nnz per row (C5 families)
    double mu, sigma;  // lognormal (short-wide)
    int ndense;        // dense rows (circuit)
    double dense_lo, dense_hi, dense_expo;
    double p_empty;    // probability of an empty row (uniform family)
    int unit_values;   // all values 1.0
} sbbgen_params;

}  // extern "C"

namespace {

// Truncated power law with density ~ x^-e on [a, b], continuous inverse CDF.
double powerlaw(Rng &g, double e, double a, double b)
{
    double u = g.uni();
    if (std::fabs(e - 1.0) < 1e-12) return a * std::pow(b / a, u);
    double k = 1.0 - e;
    double A = std::pow(a, k), B = std::pow(b, k);
    return std::pow(A + u * (B - A), 1.0 / k);
}

// L distinct sorted values from [lo, lo+w): selection sampling when dense,
// draw-sort-dedupe with top-ups when sparse.
void distinct_sorted(Rng &g, long long lo, long long w, long long L, std::vector<int> &out)
{
    out.clear();
    if (L <= 0 || w <= 0) return;
    if (L >= w) {
        for (long long i = 0; i < w; i++) out.push_back((int)(lo + i));
        return;
    }
    if (L * 4 >= w) {  // Knuth's algorithm S
        long long need = L;
        for (long long i = 0; i < w && need > 0; i++) {
            if ((double)(w - i) * g.uni() < (double)need) {
                out.push_back((int)(lo + i));
                --need;
            }
        }
        return;
    }
    // Each round draws exactly the deficit, so the set never overshoots L.
    while ((long long)out.size() < L) {
        long long want = L - (long long)out.size();
        for (long long i = 0; i < want; i++) out.push_back((int)(lo + g.below(w)));
        std::sort(out.begin(), out.end());
        out.erase(std::unique(out.begin(), out.end()), out.end());
    }
}

struct RowGen {
    const sbbgen_params &P;
    std::vector<char> dense;  // circuit: dense-row marks
    std::vector<long long> dense_len;

    explicit RowGen(const sbbgen_params &p) : P(p)
    {
        if (P.family == GEN_CIRCUIT && P.ndense > 0) {
            dense.assign(P.m, 0);
            dense_len.assign(P.m, 0);
            Rng g(P.seed, 0xDE05Eull);
            int placed = 0;
            while (placed < P.ndense && placed < P.m) {
                long long r = g.below(P.m);
                if (dense[r]) continue;
                dense[r] = 1;
                double L = placed == 0 ? P.dense_hi : powerlaw(g, P.dense_expo, P.dense_lo, P.dense_hi);
                dense_len[r] = std::min<long long>((long long)L, P.n);
                ++placed;
            }
        }
    }

    void row(long long i, std::vector<int> &cols, std::vector<int> &tmp) const
    {
        Rng g(P.seed, (uint64_t)i + 1);
        cols.clear();
        switch (P.family) {
        case GEN_POWERLAW: {
            long long L = (long long)std::floor(powerlaw(g, P.expo, P.lmin, P.lmax + 1.0));
            L = std::max<long long>(1, std::min<long long>(L, std::min<long long>((long long)P.lmax, P.n)));
            distinct_sorted(g, 0, P.n, L, cols);
            break;
        }
        case GEN_CIRCUIT: {
            if (!dense.empty() && dense[i]) {
                distinct_sorted(g, 0, P.n, dense_len[i], cols);
                break;
            }
            for (int d = -P.hw; d <= P.hw; d++) {
                long long c = i + d;
                bool keep = d == 0 || g.uni() < P.p;
                if (keep && c >= 0 && c < P.n) cols.push_back((int)c);
            }
            long long K = (long long)std::ceil(powerlaw(g, P.expo, P.lmin, P.lmax));
            for (long long k = 0; k < K; k++) cols.push_back((int)g.below(P.n));
            std::sort(cols.begin(), cols.end());
            cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
            break;
        }
        case GEN_SHORTWIDE: {
            double z = 0;  // Box-Muller
            {
                double u1 = g.uni(), u2 = g.uni();
                z = std::sqrt(-2.0 * std::log(1.0 - u1)) * std::cos(6.283185307179586 * u2);
            }
            long long L = (long long)std::llround(std::exp(P.mu + P.sigma * z));
            L = std::max<long long>(1, std::min<long long>(L, P.n));
            long long nblk = P.n / 64;
            long long k = (L + 47) / 48;  // runs of <= 48 columns, one per block
            k = std::min(k, nblk);
            distinct_sorted(g, 0, nblk, k, tmp);
            long long left = L;
            for (size_t b = 0; b < tmp.size(); b++) {
                long long runs_left = (long long)tmp.size() - (long long)b;
                long long len = std::min<long long>(64, (left + runs_left - 1) / runs_left);
                long long off = g.below(64 - len + 1);
                long long base = (long long)tmp[b] * 64 + off;
                for (long long c = 0; c < len && base + c < P.n; c++) cols.push_back((int)(base + c));
                left -= len;
            }
            break;
        }
        case GEN_BANDED: {
            long long lo = std::max<long long>(0, i - P.hw), hi = std::min<long long>(P.n - 1, i + P.hw);
            long long w = hi - lo + 1;
            long long L = (long long)std::llround(P.r * (0.5 + g.uni()));
            L = std::max<long long>(1, std::min(L, w));
            distinct_sorted(g, lo, w, L, cols);
            break;
        }
        case GEN_PLFAMILY: {
            long long L = (long long)std::llround(powerlaw(g, P.expo, P.lmin, P.lmax));
            L = std::max<long long>(1, std::min<long long>(L, P.n));
            distinct_sorted(g, 0, P.n, L, cols);
            break;
        }
        case GEN_BLOCKDIAG: {
            long long b0 = (i / P.block) * P.block;
            long long w = std::min<long long>(P.block, P.n - b0);
            if (w <= 0) break;
            long long L = (long long)std::llround(P.r * (0.5 + g.uni()));
            L = std::max<long long>(1, std::min(L, w));
            distinct_sorted(g, b0, w, L, cols);
            break;
        }
        case GEN_UNIFORM: {
            if (g.uni() < P.p_empty) break;
            long long L = (long long)P.lmin + g.below((long long)(P.lmax - P.lmin + 1));
            L = std::min<long long>(L, P.n);
            distinct_sorted(g, 0, P.n, L, cols);
            break;
        }
        default:
            break;
        }
    }
};

}  // namespace

extern "C" {

// Pass 1: row pointer (m+1 entries); returns nnz.
long long sbbgen_rowptr(const sbbgen_params *P, long long *rowptr)
{
    RowGen G(*P);
    rowptr[0] = 0;
#pragma omp parallel
    {
        std::vector<int> cols, tmp;
#pragma omp for schedule(dynamic, 256)
        for (long long i = 0; i < P->m; i++) {
            G.row(i, cols, tmp);
            rowptr[i + 1] = (long long)cols.size();
        }
    }
    for (long long i = 0; i < P->m; i++) rowptr[i + 1] += rowptr[i];
    return rowptr[P->m];
}

// Pass 2: columns and values (val U(-1,1) from a per-row value stream, or 1.0).
void sbbgen_fill(const sbbgen_params *P, const long long *rowptr, int *col, double *val)
{
    RowGen G(*P);
#pragma omp parallel
    {
        std::vector<int> cols, tmp;
#pragma omp for schedule(dynamic, 256)
        for (long long i = 0; i < P->m; i++) {
            G.row(i, cols, tmp);
            long long b = rowptr[i];
            std::memcpy(col + b, cols.data(), sizeof(int) * cols.size());
            Rng v(P->seed ^ 0x5A17ull, (uint64_t)i);
            for (size_t k = 0; k < cols.size(); k++)
                val[b + k] = P->unit_values ? 1.0 : 2.0 * v.uni() - 1.0;
        }
    }
}

// Dense vector U(lo, hi), one stream per 4096-element chunk.
void sbbgen_uniform(unsigned long long seed, long long n, double lo, double hi, double *out)
{
#pragma omp parallel for schedule(static)
    for (long long c = 0; c < (n + 4095) / 4096; c++) {
        Rng g(seed ^ 0xA5A5ull, (uint64_t)c);
        long long e = std::min(n, (c + 1) * 4096);
        for (long long i = c * 4096; i < e; i++) out[i] = lo + (hi - lo) * g.uni();
    }
}

int sbbgen_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
