// gen.c: seeded synthetic workloads for the semiring SpGEMM path.
//
// Every generator is counter-based (splitmix64 of seed and a draw index), so
// the output is identical for any OpenMP thread count and on any host.  All
// matrices come out as sorted, duplicate-free CSR with int64 row pointers and
// column indices, the layout of a by-row GrB_Matrix in SuiteSparse:GraphBLAS
// (Source/builtin/include/GB_matrix.h:213-235).
//
// Workloads (sizes are chosen by the caller):
//   * R-MAT (a,b,c,d) edge lists, symmetrised, self-loops and duplicates
//     dropped (triangle counting and BFS inputs);
//   * Erdos-Renyi rows with exactly d distinct uniform columns per row and
//     values uniform in [lo,hi] (saxpy3 plus_times input);
//   * Poisson(mean) entries per row, uniform columns, duplicates merged by
//     min (batched min_plus input).

#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static inline uint64_t mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// draw number `ctr` of stream `seed`
static inline uint64_t draw(uint64_t seed, uint64_t ctr)
{
    return mix64(mix64(seed) ^ (ctr * 0xD1B54A32D192ED03ULL));
}

static inline double unif01(uint64_t seed, uint64_t ctr)
{
    return (double)(draw(seed, ctr) >> 11) * 0x1.0p-53;
}

//------------------------------------------------------------------------------
// R-MAT edges: m = ef << scale draws, endpoints u[e], v[e] in [0, 2^scale)
//------------------------------------------------------------------------------

void grbgen_rmat_edges(int scale, int64_t m, double a, double b, double c,
                       uint64_t seed, int32_t *u, int32_t *v)
{
    const double ab = a + b, abc = a + b + c;
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < m; e++)
    {
        uint32_t x = 0, y = 0;
        for (int l = 0; l < scale; l++)
        {
            double r = unif01(seed, (uint64_t)e * (uint64_t)scale + (uint64_t)l);
            uint32_t bx, by;
            if (r < a)        { bx = 0; by = 0; }
            else if (r < ab)  { bx = 0; by = 1; }
            else if (r < abc) { bx = 1; by = 0; }
            else              { bx = 1; by = 1; }
            x = (x << 1) | bx;
            y = (y << 1) | by;
        }
        u[e] = (int32_t)x;
        v[e] = (int32_t)y;
    }
}

static int cmp_i64(const void *p, const void *q)
{
    int64_t a = *(const int64_t *)p, b = *(const int64_t *)q;
    return (a > b) - (a < b);
}

//------------------------------------------------------------------------------
// edge list -> sorted duplicate-free CSR (optionally symmetrised, no self loops)
//------------------------------------------------------------------------------

// Ap has n+1 entries.  Ai must hold (symmetric ? 2m : m) entries.  Returns nnz.
int64_t grbgen_csr_from_edges(int64_t n, int64_t m, const int32_t *u,
                              const int32_t *v, int symmetric, int drop_self,
                              int64_t *Ap, int64_t *Ai)
{
    int64_t *cnt = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    if (!cnt) return -1;
    for (int64_t e = 0; e < m; e++)
    {
        if (drop_self && u[e] == v[e]) continue;
        cnt[u[e]]++;
        if (symmetric) cnt[v[e]]++;
    }
    int64_t *pos = (int64_t *)malloc(((size_t)n + 1) * sizeof(int64_t));
    if (!pos) { free(cnt); return -1; }
    int64_t s = 0;
    for (int64_t r = 0; r < n; r++) { pos[r] = s; s += cnt[r]; }
    pos[n] = s;
    memcpy(Ap, pos, ((size_t)n + 1) * sizeof(int64_t));
    for (int64_t e = 0; e < m; e++)
    {
        if (drop_self && u[e] == v[e]) continue;
        Ai[pos[u[e]]++] = v[e];
        if (symmetric) Ai[pos[v[e]]++] = u[e];
    }
    // sort and deduplicate each row (rows are independent)
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t r = 0; r < n; r++)
    {
        int64_t lo = Ap[r], hi = Ap[r + 1];
        qsort(Ai + lo, (size_t)(hi - lo), sizeof(int64_t), cmp_i64);
        int64_t w = lo;
        for (int64_t p = lo; p < hi; p++)
            if (p == lo || Ai[p] != Ai[p - 1]) Ai[w++] = Ai[p];
        cnt[r] = w - lo;
    }
    // compact rows in place (left shift only, so sequential is safe)
    int64_t w = 0;
    for (int64_t r = 0; r < n; r++)
    {
        int64_t lo = Ap[r];
        if (w != lo) memmove(Ai + w, Ai + lo, (size_t)cnt[r] * sizeof(int64_t));
        Ap[r] = w;
        w += cnt[r];
    }
    Ap[n] = w;
    free(cnt);
    free(pos);
    return w;
}

//------------------------------------------------------------------------------
// strict lower / upper triangles of a sorted CSR matrix
//------------------------------------------------------------------------------

// Lp, Up have n+1 entries; Li, Ui have room for nnz(S) entries.
void grbgen_split_tril_triu(int64_t n, const int64_t *Sp, const int64_t *Si,
                            int64_t *Lp, int64_t *Li, int64_t *Up, int64_t *Ui)
{
    int64_t nl = 0, nu = 0;
    for (int64_t r = 0; r < n; r++)
    {
        Lp[r] = nl; Up[r] = nu;
        for (int64_t p = Sp[r]; p < Sp[r + 1]; p++)
        {
            int64_t c = Si[p];
            if (c < r) Li[nl++] = c;
            else if (c > r) Ui[nu++] = c;
        }
    }
    Lp[n] = nl; Up[n] = nu;
}

//------------------------------------------------------------------------------
// Erdos-Renyi: exactly d distinct uniform columns per row, values U[lo,hi]
//------------------------------------------------------------------------------

// Ap: nrows+1, Ai / Ax: nrows*d.  Value type: fp64 (Ax64) or fp32 (Ax32), one
// of the two may be NULL.
void grbgen_er_fixed(int64_t nrows, int64_t ncols, int d, double lo, double hi,
                     uint64_t seed, int64_t *Ap, int64_t *Ai, double *Ax64,
                     float *Ax32)
{
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < nrows; r++)
    {
        int64_t *row = Ai + r * d;
        uint64_t ctr = (uint64_t)r << 20;
        int got = 0;
        while (got < d)
        {
            int64_t c = (int64_t)(draw(seed, ctr++) % (uint64_t)ncols);
            int dup = 0;
            for (int t = 0; t < got; t++) if (row[t] == c) { dup = 1; break; }
            if (!dup) row[got++] = c;
        }
        qsort(row, (size_t)d, sizeof(int64_t), cmp_i64);
        for (int t = 0; t < d; t++)
        {
            double val = lo + (hi - lo) * unif01(seed ^ 0x5151515151515151ULL,
                                                 (uint64_t)(r * d + t));
            if (Ax64) Ax64[r * d + t] = val;
            if (Ax32) Ax32[r * d + t] = (float)val;
        }
        Ap[r] = r * d;
    }
    Ap[nrows] = nrows * d;
}

//------------------------------------------------------------------------------
// Erdos-Renyi with a per-row count drawn uniformly in [dmin, dmax]
//------------------------------------------------------------------------------

// Pass Ai == NULL to get nnz only (row pointers are always filled).
int64_t grbgen_er_range(int64_t n, int dmin, int dmax, double lo, double hi,
                        uint64_t seed, int64_t *Ap, int64_t *Ai, double *Ax64,
                        float *Ax32)
{
    int64_t s = 0;
    for (int64_t r = 0; r < n; r++)
    {
        int64_t d = dmin + (int64_t)(draw(seed ^ 0xABCDEFULL, (uint64_t)r) %
                                     (uint64_t)(dmax - dmin + 1));
        if (d > n) d = n;
        Ap[r] = s;
        s += d;
    }
    Ap[n] = s;
    if (!Ai) return s;
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; r++)
    {
        int64_t d = Ap[r + 1] - Ap[r];
        int64_t *row = Ai + Ap[r];
        uint64_t ctr = (uint64_t)r << 20;
        int64_t got = 0;
        while (got < d)
        {
            int64_t c = (int64_t)(draw(seed, ctr++) % (uint64_t)n);
            int dup = 0;
            for (int64_t t = 0; t < got; t++) if (row[t] == c) { dup = 1; break; }
            if (!dup) row[got++] = c;
        }
        qsort(row, (size_t)d, sizeof(int64_t), cmp_i64);
        for (int64_t t = 0; t < d; t++)
        {
            double val = lo + (hi - lo) * unif01(seed ^ 0x5151515151515151ULL,
                                                 (uint64_t)(Ap[r] + t));
            if (Ax64) Ax64[Ap[r] + t] = val;
            if (Ax32) Ax32[Ap[r] + t] = (float)val;
        }
    }
    return s;
}

//------------------------------------------------------------------------------
// Poisson(mean) entries per row, uniform columns, duplicates merged by min
//------------------------------------------------------------------------------

static int poisson_draw(double mean, uint64_t seed, uint64_t ctr)
{
    // Knuth's multiplication method: fine for small means
    double L = exp(-mean), p = 1.0;
    int k = 0;
    do { k++; p *= unif01(seed, ctr * 64 + (uint64_t)k); } while (p > L && k < 63);
    return k - 1;
}

typedef struct { int64_t c; float w; } cw_t;

static int cmp_cw(const void *p, const void *q)
{
    const cw_t *a = (const cw_t *)p, *b = (const cw_t *)q;
    if (a->c != b->c) return (a->c > b->c) - (a->c < b->c);
    return (a->w > b->w) - (a->w < b->w);
}

// Pass Ai == NULL to get the number of raw draws (an upper bound on nnz);
// otherwise Ai/Ax need that many entries and the exact nnz is returned.
int64_t grbgen_poisson_minw(int64_t n, double mean, float wlo, float whi,
                            uint64_t seed, int64_t *Ap, int64_t *Ai, float *Ax)
{
    int64_t s = 0;
    for (int64_t r = 0; r < n; r++)
    {
        int d = poisson_draw(mean, seed ^ 0x77ULL, (uint64_t)r);
        Ap[r] = s;
        s += d;
    }
    Ap[n] = s;
    if (!Ai) return s;
    int64_t *cnt = (int64_t *)malloc((size_t)n * sizeof(int64_t));
    if (!cnt) return -1;
    #pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; r++)
    {
        int64_t lo = Ap[r], d = Ap[r + 1] - Ap[r];
        cw_t buf[64];
        for (int64_t t = 0; t < d; t++)
        {
            buf[t].c = (int64_t)(draw(seed, (uint64_t)(lo + t)) % (uint64_t)n);
            buf[t].w = wlo + (whi - wlo) *
                (float)unif01(seed ^ 0x3333ULL, (uint64_t)(lo + t));
        }
        qsort(buf, (size_t)d, sizeof(cw_t), cmp_cw);
        int64_t w = 0;
        for (int64_t t = 0; t < d; t++)
        {
            // sorted by (c, w): the first of each run holds the minimum weight
            if (t > 0 && buf[t].c == buf[t - 1].c) continue;
            Ai[lo + w] = buf[t].c;
            Ax[lo + w] = buf[t].w;
            w++;
        }
        cnt[r] = w;
    }
    int64_t w = 0;
    for (int64_t r = 0; r < n; r++)
    {
        int64_t lo = Ap[r];
        if (w != lo)
        {
            memmove(Ai + w, Ai + lo, (size_t)cnt[r] * sizeof(int64_t));
            memmove(Ax + w, Ax + lo, (size_t)cnt[r] * sizeof(float));
        }
        Ap[r] = w;
        w += cnt[r];
    }
    Ap[n] = w;
    free(cnt);
    return w;
}

//------------------------------------------------------------------------------
// scalar draws for the host side (sizes of batched instances, arrival times)
//------------------------------------------------------------------------------

double grbgen_unif01(uint64_t seed, uint64_t ctr) { return unif01(seed, ctr); }
