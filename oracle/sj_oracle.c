/*
 * sj_oracle.c -- CPU restatement of the reference's grid-indexed epsilon self-join.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: only the tests, the
 * smoke entry point and the CPU-baseline leg of bench.py load it.  The product
 * library (libsj) never links, loads or calls anything in oracle/.
 *
 * Parity pin: the reference ships no tests, golden vectors or known-answer
 * cases.  This restatement is pinned against outputs of the reference itself,
 * built by oracle/build_ref.py from its own sources into oracle/_ref and run on
 * a B200; the resulting pair sets are committed as fixtures under
 * tests/golden/ (see tests/golden/make_golden.py).
 *
 * What it restates (file:line in the reference project):
 *   grid dimensions      main.cu:446-503   min-eps / max+eps, nCells = ceil((max-min)/eps)
 *   cell coordinate      main.cu:263,294   (unsigned)((x - minArr[j]) / eps), FP64
 *   linear cell id       main.cu:423-439   sum idx[j] * prod_{i<j} nCells[i], dim 0 fastest
 *   index arrays         main.cu:240-401   indexLookupArr grouped by cell (ascending id),
 *                                          grid{indexmin,indexmax} inclusive,
 *                                          gridCellLookup sorted by linear id,
 *                                          per-dim non-empty coordinate masks
 *   candidate cells      kernel.cu:1455-1504 + 1076-1093: the 3^k stencil of the query
 *                                          cell, clamped to the grid.  The per-dim mask
 *                                          filter only drops coordinates that no point
 *                                          occupies, so it never changes the pair set.
 *   distance             kernel.cu:344-349  acc += (cand[l]-query[l])^2 over all GPUNUMDIM
 *                                          dims, in dim order, in the exact rounding order
 *                                          of the reference's nvcc build (orc_dist2);
 *                                          emit (query, cand) iff sqrt(acc) <= eps.
 *   output               (key = query id, value = candidate id), self pairs included,
 *                        both orders present; canonical form sorted by (key, value).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAXK 16

typedef struct {
    int D, k;
    double eps;
    double minArr[ORC_MAXK];
    double maxArr[ORC_MAXK];
    unsigned nCells[ORC_MAXK];
    uint64_t mult[ORC_MAXK];
    uint64_t totalCells;
} orc_grid;

typedef struct {
    orc_grid g;
    int64_t n;
    const double *pts;       /* borrowed: n x D, row-major (AoS) */
    uint32_t nNonEmpty;
    uint32_t *lookup;        /* indexLookupArr[n] */
    int32_t *cellMin;        /* grid[].indexmin */
    int32_t *cellMax;        /* grid[].indexmax (inclusive) */
    uint64_t *cellLid;       /* gridCellLookup[].gridLinearID, ascending; idx == position */
    uint32_t *pointCell;     /* non-empty cell index of each point id */
    uint32_t *coords;        /* nNonEmpty x k cell coordinates */
    uint32_t *mask;          /* gridCellNDMask */
    uint32_t maskOffsets[2 * ORC_MAXK];
    uint32_t nMask;
} orc_index;

/* ---------------------------------------------------------------- hashing -- */

/* splitmix64 finaliser (Vigna); the set hash is the wrapping sum over pairs,
 * so it does not depend on the order in which pairs are produced. */
uint64_t orc_pair_hash(int32_t key, int32_t val)
{
    uint64_t z = ((uint64_t)(uint32_t)key << 32) | (uint64_t)(uint32_t)val;
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

uint64_t orc_hash_pairs(const int32_t *keys, const int32_t *vals, int64_t m)
{
    uint64_t h = 0;
    for (int64_t i = 0; i < m; i++) h += orc_pair_hash(keys[i], vals[i]);
    return h;
}

/* ------------------------------------------------------------- predicate -- */

/* kernel.cu:344-349: runningTotalDist += (cand[l] - query[l])^2 over l, from 0.
 * fma_mode 1 (default) is the arithmetic the reference's nvcc build performs,
 * pinned against its own outputs (tests/golden): the compiler drops the
 * initial "0 +" and fuses the FIRST product of the first addition,
 *     acc = fma(d0, d0, d1*d1),  then  acc = fma(dl, dl, acc) for l >= 2
 * (D == 1: acc = d0*d0).  fma_mode 0 rounds every product and sum separately;
 * fma_mode 2 is the plain chain acc = fma(dl, dl, acc) from acc = 0.  Both are
 * kept only to show that the fixtures discriminate between the variants. */
static inline double orc_dist2(const double *cand, const double *query, int D, int fma_mode)
{
    double acc = 0.0;
    if (fma_mode == 1) {
        double d0 = cand[0] - query[0];
        if (D == 1) {
            volatile double sq = d0 * d0;
            return sq;
        }
        double d1 = cand[1] - query[1];
        volatile double sq1 = d1 * d1;
        acc = fma(d0, d0, sq1);
        for (int l = 2; l < D; l++) {
            double d = cand[l] - query[l];
            acc = fma(d, d, acc);
        }
    } else if (fma_mode == 2) {
        for (int l = 0; l < D; l++) {
            double d = cand[l] - query[l];
            acc = fma(d, d, acc);
        }
    } else {
        for (int l = 0; l < D; l++) {
            double d = cand[l] - query[l];
            volatile double sq = d * d; /* forces the separate rounding */
            acc = acc + sq;
        }
    }
    return acc;
}

static inline int orc_within(double acc, double eps) { return sqrt(acc) <= eps; }

/* Largest double T with sqrt(T) <= eps under round-to-nearest sqrt.  Because a
 * correctly rounded sqrt is monotone, sqrt(acc) <= eps  <=>  acc <= T. */
double orc_threshold(double eps)
{
    double t = eps * eps;
    while (sqrt(t) > eps) t = nextafter(t, -INFINITY);
    for (;;) {
        double u = nextafter(t, INFINITY);
        if (sqrt(u) <= eps) t = u; else break;
    }
    return t;
}

/* ------------------------------------------------------------------ grid -- */

static inline unsigned orc_cell_coord(double x, double mn, double eps)
{
    return (unsigned)((x - mn) / eps); /* main.cu:294 */
}

/* main.cu:446-503 */
int orc_grid_dims(const double *pts, int64_t n, int D, int k, double eps, orc_grid *g)
{
    if (n <= 0 || k < 1 || k > ORC_MAXK || k > D) return -1;
    memset(g, 0, sizeof(*g));
    g->D = D; g->k = k; g->eps = eps;
    for (int j = 0; j < k; j++) { g->minArr[j] = pts[j]; g->maxArr[j] = pts[j]; }
    for (int64_t i = 1; i < n; i++)
        for (int j = 0; j < k; j++) {
            double x = pts[i * D + j];
            if (x < g->minArr[j]) g->minArr[j] = x;
            if (x > g->maxArr[j]) g->maxArr[j] = x;
        }
    for (int j = 0; j < k; j++) { g->minArr[j] -= eps; g->maxArr[j] += eps; }
    for (int j = 0; j < k; j++) g->nCells[j] = (unsigned)ceil((g->maxArr[j] - g->minArr[j]) / eps);
    uint64_t m = 1;
    for (int j = 0; j < k; j++) { g->mult[j] = m; m *= g->nCells[j]; }
    g->totalCells = m;
    return 0;
}

/* main.cu:423-439 */
static inline uint64_t orc_linear_id(const unsigned *idx, const orc_grid *g)
{
    uint64_t id = 0, mul = 1;
    for (int j = 0; j < g->k; j++) { id += (uint64_t)idx[j] * mul; mul *= g->nCells[j]; }
    return id;
}

typedef struct { uint64_t lid; uint32_t id; } orc_kv;

static int orc_kv_cmp(const void *a, const void *b)
{
    const orc_kv *x = a, *y = b;
    if (x->lid != y->lid) return x->lid < y->lid ? -1 : 1;
    return x->id < y->id ? -1 : (x->id > y->id);
}

static int orc_u32_cmp(const void *a, const void *b)
{
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return x < y ? -1 : (x > y);
}

/* main.cu:240-401.  Returns NULL on bad input. */
orc_index *orc_index_build(const double *pts, int64_t n, int D, int k, double eps)
{
    orc_index *ix = calloc(1, sizeof(orc_index));
    if (!ix) return NULL;
    if (orc_grid_dims(pts, n, D, k, eps, &ix->g) != 0) { free(ix); return NULL; }
    ix->n = n; ix->pts = pts;
    orc_kv *kv = malloc(sizeof(orc_kv) * (size_t)n);
    for (int64_t i = 0; i < n; i++) {
        unsigned c[ORC_MAXK];
        for (int j = 0; j < k; j++) c[j] = orc_cell_coord(pts[i * D + j], ix->g.minArr[j], eps);
        kv[i].lid = orc_linear_id(c, &ix->g);
        kv[i].id = (uint32_t)i;
    }
    qsort(kv, (size_t)n, sizeof(orc_kv), orc_kv_cmp);
    uint32_t nne = 0;
    for (int64_t i = 0; i < n; i++) if (i == 0 || kv[i].lid != kv[i - 1].lid) nne++;
    ix->nNonEmpty = nne;
    ix->lookup = malloc(sizeof(uint32_t) * (size_t)n);
    ix->cellMin = malloc(sizeof(int32_t) * nne);
    ix->cellMax = malloc(sizeof(int32_t) * nne);
    ix->cellLid = malloc(sizeof(uint64_t) * nne);
    ix->pointCell = malloc(sizeof(uint32_t) * (size_t)n);
    ix->coords = malloc(sizeof(uint32_t) * (size_t)nne * k);
    int64_t c = -1;
    for (int64_t i = 0; i < n; i++) {
        if (i == 0 || kv[i].lid != kv[i - 1].lid) {
            c++;
            ix->cellMin[c] = (int32_t)i;
            ix->cellLid[c] = kv[i].lid;
        }
        ix->cellMax[c] = (int32_t)i;
        ix->lookup[i] = kv[i].id;
        ix->pointCell[kv[i].id] = (uint32_t)c;
    }
    for (uint32_t q = 0; q < nne; q++) {
        uint32_t pid = ix->lookup[ix->cellMin[q]];
        for (int j = 0; j < k; j++)
            ix->coords[(size_t)q * k + j] = orc_cell_coord(pts[(int64_t)pid * D + j], ix->g.minArr[j], eps);
    }
    /* per-dim sorted set of occupied coordinates (main.cu:381-401) */
    uint32_t *tmp = malloc(sizeof(uint32_t) * (nne ? nne : 1));
    ix->mask = malloc(sizeof(uint32_t) * (size_t)nne * k + 4);
    uint32_t off = 0;
    for (int j = 0; j < k; j++) {
        for (uint32_t q = 0; q < nne; q++) tmp[q] = ix->coords[(size_t)q * k + j];
        qsort(tmp, nne, sizeof(uint32_t), orc_u32_cmp);
        ix->maskOffsets[2 * j] = off;
        for (uint32_t q = 0; q < nne; q++)
            if (q == 0 || tmp[q] != tmp[q - 1]) ix->mask[off++] = tmp[q];
        ix->maskOffsets[2 * j + 1] = off - 1;
    }
    ix->nMask = off;
    free(tmp);
    free(kv);
    return ix;
}

void orc_index_free(orc_index *ix)
{
    if (!ix) return;
    free(ix->lookup); free(ix->cellMin); free(ix->cellMax); free(ix->cellLid);
    free(ix->pointCell); free(ix->coords); free(ix->mask); free(ix);
}

void orc_index_sizes(const orc_index *ix, uint32_t *nNonEmpty, uint32_t *nMask, uint64_t *totalCells)
{
    *nNonEmpty = ix->nNonEmpty; *nMask = ix->nMask; *totalCells = ix->g.totalCells;
}

void orc_index_grid(const orc_index *ix, double *minArr, unsigned *nCells)
{
    for (int j = 0; j < ix->g.k; j++) { minArr[j] = ix->g.minArr[j]; nCells[j] = ix->g.nCells[j]; }
}

void orc_index_export(const orc_index *ix, uint32_t *lookup, int32_t *cellMinMax, uint64_t *cellLid,
                      uint32_t *mask, uint32_t *maskOffsets)
{
    memcpy(lookup, ix->lookup, sizeof(uint32_t) * (size_t)ix->n);
    for (uint32_t c = 0; c < ix->nNonEmpty; c++) {
        cellMinMax[2 * c] = ix->cellMin[c];
        cellMinMax[2 * c + 1] = ix->cellMax[c];
    }
    memcpy(cellLid, ix->cellLid, sizeof(uint64_t) * ix->nNonEmpty);
    memcpy(mask, ix->mask, sizeof(uint32_t) * ix->nMask);
    memcpy(maskOffsets, ix->maskOffsets, sizeof(uint32_t) * 2 * ix->g.k);
}

/* Binary search for a linear id among the non-empty cells; -1 when empty. */
static inline int64_t orc_find_cell(const orc_index *ix, uint64_t lid)
{
    int64_t lo = 0, hi = (int64_t)ix->nNonEmpty;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (ix->cellLid[mid] < lid) lo = mid + 1; else hi = mid;
    }
    return (lo < (int64_t)ix->nNonEmpty && ix->cellLid[lo] == lid) ? lo : -1;
}

/* Visits the non-empty cells of the clamped 3^k stencil of cell `c`
 * (kernel.cu:1076-1093).  Writes their indices to out[], returns the count. */
static int orc_stencil(const orc_index *ix, uint32_t c, int64_t *out)
{
    const int k = ix->g.k;
    const uint32_t *a = ix->coords + (size_t)c * k;
    int off[ORC_MAXK];
    for (int j = 0; j < k; j++) off[j] = -1;
    int cnt = 0;
    for (;;) {
        unsigned idx[ORC_MAXK];
        int ok = 1;
        for (int j = 0; j < k; j++) {
            int64_t v = (int64_t)a[j] + off[j];
            if (v < 0 || v >= (int64_t)ix->g.nCells[j]) { ok = 0; break; }
            idx[j] = (unsigned)v;
        }
        if (ok) {
            int64_t b = orc_find_cell(ix, orc_linear_id(idx, &ix->g));
            if (b >= 0) out[cnt++] = b;
        }
        int j = 0;
        while (j < k && off[j] == 1) { off[j] = -1; j++; }
        if (j == k) break;
        off[j]++;
    }
    return cnt;
}

static int64_t orc_stencil_cap(int k)
{
    int64_t s = 1;
    for (int j = 0; j < k; j++) s *= 3;
    return s;
}

/* --------------------------------------------------------------- joins -- */

/* Pair count, set hash and candidate evaluations for the query points with
 * id in {q0, q0+qstride, ...} < q1 (a bounded sample when qstride > 1). */
int orc_join_stats(const orc_index *ix, int fma_mode, int64_t q0, int64_t q1, int64_t qstride,
                   int nthreads, uint64_t *pairs, uint64_t *hash, uint64_t *evals)
{
    const int D = ix->g.D;
    const double eps = ix->g.eps;
    const double *pts = ix->pts;
    if (qstride < 1) qstride = 1;
    if (q1 > ix->n) q1 = ix->n;
    uint64_t P = 0, H = 0, E = 0;
    int64_t cap = orc_stencil_cap(ix->g.k);
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads) reduction(+ : P, H, E)
#endif
    {
        int64_t *nb = malloc(sizeof(int64_t) * (size_t)cap);
        int64_t nq = (q1 - q0 + qstride - 1) / qstride;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
        for (int64_t t = 0; t < nq; t++) {
            int64_t p = q0 + t * qstride;
            const double *qp = pts + p * D;
            int m = orc_stencil(ix, ix->pointCell[p], nb);
            for (int b = 0; b < m; b++)
                for (int32_t s = ix->cellMin[nb[b]]; s <= ix->cellMax[nb[b]]; s++) {
                    uint32_t q = ix->lookup[s];
                    E++;
                    if (orc_within(orc_dist2(pts + (int64_t)q * D, qp, D, fma_mode), eps)) {
                        P++;
                        H += orc_pair_hash((int32_t)p, (int32_t)q);
                    }
                }
        }
        free(nb);
    }
    *pairs = P; *hash = H; *evals = E;
    return 0;
}

/* orc_join_stats under the linear-ID Unicomp ownership (kernel.cu:1529-1534):
 * a sampled point p evaluates the points of its own cell with a larger id and
 * every point of the stencil cells with a larger linear id, and each hit
 * counts both directions, (p,q) and (q,p) (a self pair once).  Over all points
 * the pairs and the set hash equal orc_join_stats's with half the candidate
 * evaluations: the CPU baseline's join (a CPU self-join evaluates each
 * unordered pair once, as the reference's Unicomp kernels do). */
int orc_join_stats_unicomp(const orc_index *ix, int fma_mode, int64_t q0, int64_t q1, int64_t qstride,
                           int nthreads, uint64_t *pairs, uint64_t *hash, uint64_t *evals)
{
    const int D = ix->g.D;
    const double eps = ix->g.eps;
    const double *pts = ix->pts;
    if (qstride < 1) qstride = 1;
    if (q1 > ix->n) q1 = ix->n;
    uint64_t P = 0, H = 0, E = 0;
    int64_t cap = orc_stencil_cap(ix->g.k);
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads) reduction(+ : P, H, E)
#endif
    {
        int64_t *nb = malloc(sizeof(int64_t) * (size_t)cap);
        int64_t nq = (q1 - q0 + qstride - 1) / qstride;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
        for (int64_t t = 0; t < nq; t++) {
            int64_t p = q0 + t * qstride;
            const double *qp = pts + p * D;
            const int64_t c = ix->pointCell[p];
            int m = orc_stencil(ix, (uint32_t)c, nb);
            for (int b = 0; b < m; b++) {
                if (nb[b] < c) continue;   /* owned by the cell with the larger linear id */
                const int home = nb[b] == c;
                for (int32_t s = ix->cellMin[nb[b]]; s <= ix->cellMax[nb[b]]; s++) {
                    uint32_t q = ix->lookup[s];
                    if (home && (int64_t)q < p) continue;
                    E++;
                    if (orc_within(orc_dist2(pts + (int64_t)q * D, qp, D, fma_mode), eps)) {
                        if ((int64_t)q == p) {
                            P += 1;
                            H += orc_pair_hash((int32_t)p, (int32_t)p);
                        } else {
                            P += 2;
                            H += orc_pair_hash((int32_t)p, (int32_t)q) + orc_pair_hash((int32_t)q, (int32_t)p);
                        }
                    }
                }
            }
        }
        free(nb);
    }
    *pairs = P; *hash = H; *evals = E;
    return 0;
}

/* Neighbour count of every point (its row length in the neighbour table). */
int orc_join_degrees(const orc_index *ix, int fma_mode, int nthreads, uint32_t *deg)
{
    const int D = ix->g.D;
    const double eps = ix->g.eps;
    const double *pts = ix->pts;
    int64_t cap = orc_stencil_cap(ix->g.k);
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
    {
        int64_t *nb = malloc(sizeof(int64_t) * (size_t)cap);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
        for (int64_t p = 0; p < ix->n; p++) {
            const double *qp = pts + p * D;
            int m = orc_stencil(ix, ix->pointCell[p], nb);
            uint32_t d = 0;
            for (int b = 0; b < m; b++)
                for (int32_t s = ix->cellMin[nb[b]]; s <= ix->cellMax[nb[b]]; s++)
                    d += orc_within(orc_dist2(pts + (int64_t)ix->lookup[s] * D, qp, D, fma_mode), eps);
            deg[p] = d;
        }
        free(nb);
    }
    return 0;
}

/* Rows of the neighbour table for the query ids qids[0..nq): per query its
 * degree and the set hash of its row (sum of orc_pair_hash(query, value)).
 * With off != NULL and vals != NULL, row i's values (unsorted) are also
 * written to vals[off[i] .. off[i] + deg[i]) when that fits below cap (rows
 * that do not fit leave deg[i] correct and set the return value to 1). */
int orc_query_rows(const orc_index *ix, int fma_mode, const int64_t *qids, int64_t nq, int nthreads,
                   uint32_t *deg, uint64_t *rowHash, const int64_t *off, int32_t *vals, int64_t cap)
{
    const int D = ix->g.D;
    const double eps = ix->g.eps;
    const double *pts = ix->pts;
    int64_t scap = orc_stencil_cap(ix->g.k);
    int overflow = 0;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads) reduction(| : overflow)
#endif
    {
        int64_t *nb = malloc(sizeof(int64_t) * (size_t)scap);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 4)
#endif
        for (int64_t i = 0; i < nq; i++) {
            const int64_t p = qids[i];
            const double *qp = pts + p * D;
            int m = orc_stencil(ix, ix->pointCell[p], nb);
            uint32_t d = 0;
            uint64_t h = 0;
            for (int b = 0; b < m; b++)
                for (int32_t s = ix->cellMin[nb[b]]; s <= ix->cellMax[nb[b]]; s++) {
                    const uint32_t q = ix->lookup[s];
                    if (orc_within(orc_dist2(pts + (int64_t)q * D, qp, D, fma_mode), eps)) {
                        if (off && vals) {
                            if (off[i] + (int64_t)d < cap) vals[off[i] + d] = (int32_t)q;
                            else overflow = 1;
                        }
                        d++;
                        h += orc_pair_hash((int32_t)p, (int32_t)q);
                    }
                }
            deg[i] = d;
            if (rowHash) rowHash[i] = h;
        }
        free(nb);
    }
    return overflow;
}

static int orc_i32_cmp(const void *a, const void *b)
{
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return x < y ? -1 : (x > y);
}

/* All pairs in canonical (key, value) order.  With keys == NULL only counts.
 * Returns the pair count, or -1 when cap is too small. */
int64_t orc_join_pairs(const orc_index *ix, int fma_mode, int32_t *keys, int32_t *vals, int64_t cap)
{
    const int D = ix->g.D;
    const double eps = ix->g.eps;
    const double *pts = ix->pts;
    int64_t scap = orc_stencil_cap(ix->g.k);
    int64_t *nb = malloc(sizeof(int64_t) * (size_t)scap);
    int64_t m = 0;
    for (int64_t p = 0; p < ix->n; p++) {
        const double *qp = pts + p * D;
        int nn = orc_stencil(ix, ix->pointCell[p], nb);
        int64_t start = m;
        for (int b = 0; b < nn; b++)
            for (int32_t s = ix->cellMin[nb[b]]; s <= ix->cellMax[nb[b]]; s++) {
                uint32_t q = ix->lookup[s];
                if (orc_within(orc_dist2(pts + (int64_t)q * D, qp, D, fma_mode), eps)) {
                    if (keys) {
                        if (m >= cap) { free(nb); return -1; }
                        keys[m] = (int32_t)p;
                        vals[m] = (int32_t)q;
                    }
                    m++;
                }
            }
        if (keys) qsort(vals + start, (size_t)(m - start), sizeof(int32_t), orc_i32_cmp);
    }
    free(nb);
    return m;
}

/* O(n^2) brute force with the same predicate and no grid restriction. */
int64_t orc_brute_pairs(const double *pts, int64_t n, int D, double eps, int fma_mode,
                        int32_t *keys, int32_t *vals, int64_t cap)
{
    int64_t m = 0;
    for (int64_t p = 0; p < n; p++)
        for (int64_t q = 0; q < n; q++)
            if (orc_within(orc_dist2(pts + q * D, pts + p * D, D, fma_mode), eps)) {
                if (keys) {
                    if (m >= cap) return -1;
                    keys[m] = (int32_t)p;
                    vals[m] = (int32_t)q;
                }
                m++;
            }
    return m;
}

/* Candidate evaluations of the full-stencil traversal, per non-empty cell:
 * |c| * sum over stencil cells |c'| (the work unit W_dist counts). */
int orc_cell_candidates(const orc_index *ix, uint64_t *cand)
{
    int64_t cap = orc_stencil_cap(ix->g.k);
    int64_t *nb = malloc(sizeof(int64_t) * (size_t)cap);
    for (uint32_t c = 0; c < ix->nNonEmpty; c++) {
        int m = orc_stencil(ix, c, nb);
        uint64_t s = 0;
        for (int b = 0; b < m; b++) s += (uint64_t)(ix->cellMax[nb[b]] - ix->cellMin[nb[b]] + 1);
        cand[c] = s * (uint64_t)(ix->cellMax[c] - ix->cellMin[c] + 1);
    }
    free(nb);
    return 0;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
