// Host engine behind the C ABI (include/sj.h).
//
// Pipeline of one join (replacing distanceTableNDGridBatches, GPU.cu:1297-2569):
//   1. grid index on the device (sj_index.cu)
//   2. owned neighbour-cell lists for the traversal pattern (sj_stencil.cu)
//   3. per-cell hit-rate estimate: sampling (GPU.cu:854-1065 analogue) or the
//      learned MLP (sj_estimate.cu)
//   4. tasks = (query tile of a cell) x (stretch of its candidate stream), with
//      exact evaluation counts and predicted pairs; ordered by predicted cost
//      for the work-queue / sorted modes (kernel.cu:33-250, GPU.cu:1660-1734)
//   5. batches = consecutive tasks whose predicted pairs fit the capacity; per
//      batch: count pass -> exclusive scan over point ids -> (split and retry
//      on overflow) -> fill pass -> delivery (GPU.cu:2101-2377)
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <immintrin.h>
#include <cstring>
#include <mutex>
#include <numeric>
#include <omp.h>
#include <parallel/algorithm>
#include <string>
#include <vector>

#include "sj_internal.h"

namespace sj {
int import_csv(const char *path, int D, std::vector<double> &pts);
}

namespace {

thread_local std::string g_lastError;

void set_error(const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_lastError = buf;
}

#define CK(expr)                                                                      \
    do {                                                                              \
        cudaError_t _e = (expr);                                                      \
        if (_e != cudaSuccess) {                                                      \
            set_error("%s: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__, __LINE__); \
            return (_e == cudaErrorMemoryAllocation) ? SJ_ERR_OOM : SJ_ERR_CUDA;      \
        }                                                                             \
    } while (0)

#define CKS(expr)                                  \
    do {                                           \
        sj_status _s = (expr);                     \
        if (_s != SJ_OK) return _s;                \
    } while (0)

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    ~DevBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t ensure(size_t cnt)
    {
        if (cnt <= n && p) return cudaSuccess;
        release();
        size_t c = cnt ? cnt : 1;
        cudaError_t e = cudaMalloc((void **)&p, c * sizeof(T));
        if (e == cudaSuccess) n = c;
        return e;
    }
    void swap(DevBuf &o)
    {
        std::swap(p, o.p);
        std::swap(n, o.n);
    }
};

struct PinBuf {
    void *p = nullptr;
    size_t bytes = 0;
    ~PinBuf() { release(); }
    void release()
    {
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t ensure(size_t b)
    {
        if (b <= bytes && p) return cudaSuccess;
        release();
        cudaError_t e = cudaMallocHost(&p, b ? b : 1);
        if (e == cudaSuccess) bytes = b ? b : 1;
        return e;
    }
};

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
    Timer()
    {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~Timer()
    {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
    void start(cudaStream_t s) { cudaEventRecord(a, s); }
    float stop(cudaStream_t s)
    {
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    }
};

int pattern_of_mode(int mode)
{
    switch (mode) {
    // mode 8 (kernel.cu:2072-2188: heaviest points first, 1/3 of the batches
    // each with NB_THREAD_THIRD{1,2,3} threads per point) is the full stencil
    // in workload order; the engine's work split is its cost-proportional task
    // chunking (a heavier cell is cut into more tasks), so it runs like 7 / 9
    case 3: case 7: case 8: case 9: return SJ_PAT_FULL;
    case 4: return SJ_PAT_UNICOMP;
    case 5: return SJ_PAT_BUNICOMP;
    case 6: case 10: return SJ_PAT_LID;
    }
    return -1;
}

int padded_dim(int D)
{
    if (D <= 4) return D == 3 ? 3 : D;
    if (D <= 6) return 6;
    if (D <= 8) return 8;
    if (D <= 12) return 12;
    return 16;
}

double eps_threshold(double eps)
{
    double t = eps * eps;
    while (std::sqrt(t) > eps) t = std::nextafter(t, -INFINITY);
    for (;;) {
        double u = std::nextafter(t, INFINITY);
        if (std::sqrt(u) <= eps) t = u; else break;
    }
    return t;
}

// Estimator feature weights: for two points uniform in two eps-wide cells whose
// coordinates differ by one in m of k dimensions and agree in the others, the
// probability that they lie within eps over those k dimensions.  Per dimension,
// u = (difference / eps)^2 has CDF 2 sqrt(v) - v on [0, 1] for a shared cell
// coordinate and v / 2 for adjacent ones; the sum of k such terms is below 1
// with the mass that discretised convolutions (NB bins on [0, 1]) give.  Uniform
// density makes these exact scale-free constants; the estimator learns how the
// data's density departs from them.
void offset_class_weights(int k, float *w)
{
    constexpr int NB = 1024;
    static std::mutex mu;
    static std::vector<float> cache[SJ_MAX_K + 1];
    std::lock_guard<std::mutex> lock(mu);
    if (k < 1 || k > SJ_MAX_K) return;
    if (cache[k].empty()) {
        std::vector<double> p0(NB), p1(NB);
        for (int i = 0; i < NB; i++) {
            const double a = (double)i / NB, b = (double)(i + 1) / NB;
            p0[i] = (2.0 * std::sqrt(b) - b) - (2.0 * std::sqrt(a) - a);
            p1[i] = (b - a) / 2.0;
        }
        auto conv = [](const std::vector<double> &x, const std::vector<double> &y) {
            std::vector<double> z(NB, 0.0);
            for (int i = 0; i < NB; i++) {
                if (x[i] == 0.0) continue;
                for (int j = 0; i + j < NB; j++) z[i + j] += x[i] * y[j];
            }
            return z;
        };
        std::vector<std::vector<double>> pow0(k + 1, std::vector<double>(NB, 0.0)), pow1 = pow0;
        pow0[0][0] = pow1[0][0] = 1.0;   // the sum of no terms: mass 1 at 0
        for (int j = 1; j <= k; j++) {
            pow0[j] = conv(pow0[j - 1], p0);
            pow1[j] = conv(pow1[j - 1], p1);
        }
        cache[k].resize(k + 1);
        for (int m = 0; m <= k; m++) {
            const std::vector<double> z = conv(pow1[m], pow0[k - m]);
            cache[k][m] = (float)std::accumulate(z.begin(), z.end(), 0.0);
        }
    }
    for (int m = 0; m <= k; m++) w[m] = cache[k][m];
}

struct Ctx {
    sj_params p{};
    int dev = 0, numSM = 148;
    cudaStream_t s = nullptr;
    // points
    uint64_t n = 0;
    DevBuf<double> pts;        // n x D as supplied
    bool havePoints = false;
    // index
    bool indexed = false;
    sj_grid_dev g{};
    uint32_t nCells = 0;
    DevBuf<uint32_t> ids;      // cell-sorted point ids
    DevBuf<double> xs;         // cell-sorted coordinates, n x Dp
    DevBuf<uint32_t> cellStart;
    DevBuf<uint64_t> cellLid;
    DevBuf<uint32_t> cellCoord;
    double dataMin[SJ_MAX_DIM], dataMax[SJ_MAX_DIM];
    // neighbour lists
    int nbrPattern = -1;
    uint32_t nbrTotal = 0;
    DevBuf<uint32_t> nbrStart, nbrCell;
    DevBuf<uint32_t> nbrPre;           // per owned-neighbour entry: occupancy prefix within its cell
    DevBuf<double> nbrPreW, cellW;     // occupancy x offset-class weight: per-entry prefix, per-cell total
    DevBuf<float> nbrWt;               // per entry: offset-class weight
    DevBuf<float> exactPred;           // per task: its measured pairs (the exact plan of the statistics)
    bool rateLearned = false;          // c.rate holds the learned estimator's predictions
    DevBuf<uint64_t> candFull;
    DevBuf<float> feat;
    // per-cell predicted hits per evaluation (learned or sampled)
    DevBuf<float> rate;
    // tasks, built on the device (sj_tasks.cu)
    uint32_t nTasks = 0;
    DevBuf<sj_task> dTasks, dTasksAlt;
    DevBuf<float> dTaskPred, dTaskPredAlt;
    DevBuf<uint32_t> tgGroupCnt, tgGroupBase, tgGroupLen, tgPosCnt, tgOrder, tgOrderAlt, tgItemCnt, tgItemStart,
        tgItemTasks, tgItemTaskStart, tgTot32;
    DevBuf<uint64_t> tgKeys, tgKeysAlt;
    DevBuf<unsigned long long> tgPosEv, tgEvExcl, tgTotals, tgScan64;
    DevBuf<uint8_t> tgWorkers;
    // per-task record offsets (exclusive prefix sums, nTasks + 1 each): row-mask
    // words, column-mask words, row offsets, candidate records, emission units,
    // planned pairs, predicted pairs
    DevBuf<unsigned long long> off[7];
    DevBuf<unsigned long long> offTemp;
    // batch plan
    DevBuf<uint32_t> planNext, planStart, planCount;
    DevBuf<unsigned long long> planStats;
    // batch state
    DevBuf<uint32_t> keyCount, keyStart, keyStart2;
    DevBuf<int32_t> outKey, outVal;
    // host delivery: second set of the device buffers a batch's copy reads, so
    // the next batch's kernels need not wait for that copy
    DevBuf<int32_t> outValAlt;
    DevBuf<uint32_t> keyStartAlt;
    std::vector<cudaEvent_t> syncEvents;   // stage boundaries of the synchronous phase
    DevBuf<uint8_t> scanTemp, scanTemp2;
    DevBuf<uint32_t> total, total2;
    DevBuf<unsigned long long> stat;   // see sj_join_args::stat
    DevBuf<uint32_t> queueHead;
    DevBuf<uint32_t> taskHits;
    DevBuf<uint32_t> dTaskEvals, dTaskRefined;   // per task, written by the count pass
    DevBuf<unsigned long long> sums;   // task sums: evaluations, refined, measured pairs
    DevBuf<double> errSum;             // sum over tasks of |predicted - measured pairs|
    // count-pass records for the emission pass: per task, row and column hit
    // masks, per-query row-run offsets and per-position candidate records
    DevBuf<uint32_t> masks, colMasks, rowRel, candId, candRel;
    // the count pass of batch i + 1 writes this second record set while the
    // emission of batch i reads the first (device-fold pipeline)
    DevBuf<uint32_t> masks2, colMasks2, rowRel2, candId2, candRel2;
    DevBuf<uint32_t> emitHead;   // the emission's work counter when it runs beside a count pass
    // device CSR neighbour table under construction (sj_neighbor_csr): the
    // caller's arrays and the rows' fill cursors
    uint64_t *csrRowPtr = nullptr;
    int32_t *csrCols = nullptr;
    uint64_t csrCap = 0;
    DevBuf<uint32_t> csrFill;
    DevBuf<uint4> longRuns;            // key expansion: runs too long for one warp
    DevBuf<uint32_t> foldChunkKey;     // consumer fold: the key at each chunk's first slot
    DevBuf<uint32_t> longCount;
    DevBuf<unsigned long long> batchTot;
    std::vector<cudaEvent_t> events;   // per-batch stage boundaries of the asynchronous phase
    PinBuf pinTotal, pinKey[2], pinVal[2], pinStart[2];
    // host delivery: copy stream and its events (per pinned buffer set: run
    // offsets copied, values copied)
    cudaStream_t cs = nullptr;
    cudaEvent_t evStart[2] = {nullptr, nullptr}, evVals[2] = {nullptr, nullptr}, evEmit = nullptr;
    // estimator
    std::vector<float> mlpW;
    DevBuf<float> dMlpW;
    // grow-only scratch reused by every index build / join (no per-call allocation)
    DevBuf<double> sMinMax;
    DevBuf<uint64_t> sKeys, sKeysAlt;
    DevBuf<uint32_t> sValsAlt, sFlags, sOne, sCnt;
    DevBuf<uint8_t> sTemp;
    DevBuf<float> sMlpOut;
    DevBuf<unsigned long long> sHits, sCands, sScalars;
    DevBuf<unsigned long long> dCellHits;   // measured hits per cell (after sj_degrees)
    bool haveMeas = false;
    bool haveSamples = false;   // sHits / sCands hold the last sampling estimate's per-cell counts
    sj_stats st{};
};


sj_status check_params(const sj_params &p)
{
    if (p.gpunumdim < 1 || p.gpunumdim > SJ_MAX_DIM) {
        set_error("gpunumdim must be in 1..%d", SJ_MAX_DIM);
        return SJ_ERR_BAD_INPUT;
    }
    if (p.numindexeddim < 1 || p.numindexeddim > p.gpunumdim || p.numindexeddim > SJ_MAX_K) {
        set_error("numindexeddim must be in 1..min(gpunumdim, %d)", SJ_MAX_K);
        return SJ_ERR_BAD_INPUT;
    }
    if (!(p.epsilon > 0.0) || !std::isfinite(p.epsilon)) {
        set_error("epsilon must be a positive finite number");
        return SJ_ERR_BAD_INPUT;
    }
    if (pattern_of_mode(p.search_mode) < 0) {
        set_error("search_mode %d not supported (3,4,5,6,7,8,9,10)", p.search_mode);
        return SJ_ERR_BAD_INPUT;
    }
    if (p.search_mode == 5 && p.numindexeddim != 2 && p.numindexeddim != 3) {
        set_error("B-Unicomp (mode 5) is defined for NUMINDEXEDDIM 2 or 3 only");
        return SJ_ERR_BAD_INPUT;
    }
    if (p.precision != SJ_PREC_FP64 && p.precision != SJ_PREC_FP32_REFINE) {
        set_error("unknown precision");
        return SJ_ERR_BAD_INPUT;
    }
    if (p.precision == SJ_PREC_FP32_REFINE && (p.epsilon < 1e-15 || p.epsilon > 1e15)) {
        set_error("FP32 filter needs 1e-15 <= epsilon <= 1e15");
        return SJ_ERR_BAD_INPUT;
    }
    if (p.scheduler != SJ_SCHED_SAMPLING && p.scheduler != SJ_SCHED_LEARNED) {
        set_error("unknown scheduler");
        return SJ_ERR_BAD_INPUT;
    }
    if (p.shard_count < 1 || p.shard_index < 0 || p.shard_index >= p.shard_count) {
        set_error("bad shard_index / shard_count");
        return SJ_ERR_BAD_INPUT;
    }
    if (!(p.sample_rate > 0.0 && p.sample_rate <= 1.0)) {
        set_error("sample_rate must be in (0, 1]");
        return SJ_ERR_BAD_INPUT;
    }
    if (p.batch_capacity_pairs != 0 && p.batch_capacity_pairs < 65536) {
        set_error("batch_capacity_pairs must be 0 (automatic) or at least 65536");
        return SJ_ERR_BAD_INPUT;
    }
    if (p.alpha < 0.0) {
        set_error("alpha must be >= 0");
        return SJ_ERR_BAD_INPUT;
    }
    return SJ_OK;
}

// ---------------------------------------------------------------- index --
sj_status build_index(Ctx &c)
{
    if (!c.havePoints) {
        set_error("no points: call sj_set_points or sj_import_csv first");
        return SJ_ERR_STATE;
    }
    Timer tm;
    tm.start(c.s);
    const int D = c.p.gpunumdim, k = c.p.numindexeddim;
    const uint64_t n = c.n;
    // 1. min / max of every dimension
    DevBuf<double> &mm = c.sMinMax;
    CK(mm.ensure(2 * D + 1));
    CK(sj_launch_minmax(c.pts.p, n, D, mm.p, c.s));
    std::vector<double> hmm(2 * D + 1);
    CK(cudaMemcpyAsync(hmm.data(), mm.p, sizeof(double) * (2 * D + 1), cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    uint64_t badBits;
    memcpy(&badBits, &hmm[2 * D], 8);
    if (badBits) {
        set_error("input contains non-finite coordinates");
        return SJ_ERR_BAD_INPUT;
    }
    sj_grid_dev &g = c.g;
    memset(&g, 0, sizeof(g));
    g.D = D;
    g.Dp = padded_dim(D);
    g.k = k;
    g.eps = c.p.epsilon;
    g.thresh = eps_threshold(c.p.epsilon);
    offset_class_weights(k, g.offW);
    for (int j = 0; j < D; j++) {
        c.dataMin[j] = hmm[2 * j];
        c.dataMax[j] = hmm[2 * j + 1];
        g.center[j] = 0.5 * (c.dataMin[j] + c.dataMax[j]);
    }
    // 2. grid dimensions (main.cu:446-503)
    double total = 1.0;
    unsigned long long mul = 1;
    for (int j = 0; j < k; j++) {
        double mn = c.dataMin[j] - g.eps;
        double mx = c.dataMax[j] + g.eps;
        g.minArr[j] = mn;
        double cells = std::ceil((mx - mn) / g.eps);
        if (!(cells >= 1.0) || cells > 4294967295.0) {
            set_error("dimension %d spans %.3g cells (limit 2^32-1)", j, cells);
            return SJ_ERR_BAD_INPUT;
        }
        g.nCells[j] = (unsigned)cells;
        g.mult[j] = mul;
        mul *= g.nCells[j];
        total *= cells;
    }
    if (total >= 1.8e19) {
        set_error("grid has %.3g cells; linear ids need < 2^64", total);
        return SJ_ERR_BAD_INPUT;
    }
    c.st.total_cells = mul;
    int bits = 1;
    while (bits < 64 && (1ULL << bits) < mul) bits++;
    // 3. keys, stable sort, run-length cells
    DevBuf<uint64_t> &keys = c.sKeys, &keysAlt = c.sKeysAlt;
    DevBuf<uint32_t> &valsAlt = c.sValsAlt, &flags = c.sFlags;
    DevBuf<uint8_t> &tmp = c.sTemp;
    CK(keys.ensure(n));
    CK(keysAlt.ensure(n));
    CK(c.ids.ensure(n));
    CK(valsAlt.ensure(n));
    CK(flags.ensure(n));
    CK(tmp.ensure(std::max(sj_radix_temp_bytes(n), sj_scan_temp_bytes(n))));
    DevBuf<uint32_t> &nne = c.sOne;
    CK(nne.ensure(2));   // [0] non-empty cells, [1] out-of-grid flag
    CK(cudaMemsetAsync(nne.p + 1, 0, sizeof(uint32_t), c.s));
    CK(sj_launch_cell_keys(c.pts.p, n, g, keys.p, c.ids.p, nne.p + 1, c.s));
    int inAlt = 0;
    CK(sj_radix_sort_u64_u32(keys.p, c.ids.p, keysAlt.p, valsAlt.p, n, bits, tmp.p, &inAlt, c.s));
    uint64_t *sk = inAlt ? keysAlt.p : keys.p;
    if (inAlt) CK(cudaMemcpyAsync(c.ids.p, valsAlt.p, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, c.s));
    CK(sj_launch_cell_flags(sk, n, flags.p, c.s));
    CK(sj_exclusive_scan_u32(flags.p, flags.p, n, tmp.p, nne.p, c.s));
    uint32_t hn[2] = {0, 0};
    CK(cudaMemcpyAsync(hn, nne.p, sizeof(hn), cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    if (hn[1]) {
        // a cell coordinate past its dimension's cell count would alias another cell
        set_error("internal: a point's cell coordinate lies outside the grid");
        return SJ_ERR_INTERNAL;
    }
    const uint32_t nCells = hn[0];
    c.nCells = nCells;
    CK(c.cellStart.ensure(nCells + 1));
    CK(c.cellLid.ensure(nCells));
    CK(c.cellCoord.ensure((size_t)nCells * k));
    CK(sj_launch_cell_build(sk, flags.p, n, c.cellStart.p, c.cellLid.p, c.s));
    uint32_t nn = (uint32_t)n;
    CK(cudaMemcpyAsync(c.cellStart.p + nCells, &nn, sizeof(uint32_t), cudaMemcpyHostToDevice, c.s));
    CK(sj_launch_cell_coords(c.cellLid.p, nCells, g, c.cellCoord.p, c.s));
    // 4. cell-sorted coordinates
    CK(c.xs.ensure(n * (uint64_t)g.Dp));
    CK(sj_launch_gather(c.pts.p, c.ids.p, n, D, g.Dp, c.xs.p, c.s));
    c.indexed = true;
    c.nbrPattern = -1;
    c.haveMeas = false;
    c.st.n_points = (uint32_t)n;
    c.st.n_nonempty_cells = nCells;
    c.st.ms_index = tm.stop(c.s);
    return SJ_OK;
}

// ------------------------------------------------------ neighbour lists --
sj_status build_neighbours(Ctx &c, int pattern)
{
    if (c.nbrPattern == pattern) return SJ_OK;
    const uint32_t nc = c.nCells;
    CK(c.nbrStart.ensure(nc + 1));
    CK(c.candFull.ensure(nc));
    CK(c.feat.ensure((size_t)nc * SJ_NFEAT));
    DevBuf<uint32_t> &cnt = c.sCnt;
    CK(cnt.ensure(nc + 1));
    DevBuf<unsigned long long> &sc = c.sScalars;
    CK(sc.ensure(2 + sj_sample_totals_len()));
    CK(cudaMemsetAsync(sc.p, 0, sizeof(unsigned long long), c.s));
    CK(sj_launch_neighbours(c.cellLid.p, c.cellCoord.p, c.cellStart.p, nc, c.g, pattern, nullptr, cnt.p,
                            c.candFull.p, sc.p, c.feat.p, 0, c.s));
    DevBuf<uint8_t> &tmp = c.sTemp;
    CK(tmp.ensure(sj_scan_temp_bytes(nc)));
    CK(sj_exclusive_scan_u32(cnt.p, c.nbrStart.p, nc, tmp.p, c.nbrStart.p + nc, c.s));
    // the list length sizes the list; the candidate total is the work unit
    struct {
        uint32_t total;
        unsigned long long full;
    } h{};
    CK(cudaMemcpyAsync(&h.total, c.nbrStart.p + nc, sizeof(uint32_t), cudaMemcpyDeviceToHost, c.s));
    CK(cudaMemcpyAsync(&h.full, sc.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    CK(c.nbrCell.ensure(h.total));
    CK(sj_launch_neighbours(c.cellLid.p, c.cellCoord.p, c.cellStart.p, nc, c.g, pattern, c.nbrStart.p, c.nbrCell.p,
                            nullptr, nullptr, nullptr, 1, c.s));
    CK(c.nbrPre.ensure(h.total ? h.total : 1));
    CK(c.nbrPreW.ensure(h.total ? h.total : 1));
    CK(c.nbrWt.ensure(h.total ? h.total : 1));
    CK(c.cellW.ensure(nc ? nc : 1));
    CK(sj_nbr_spread(c.cellStart.p, c.cellCoord.p, c.nbrStart.p, c.nbrCell.p, nc, c.g, c.nbrPre.p, c.nbrPreW.p,
                     c.nbrWt.p, c.cellW.p, c.s));
    c.nbrTotal = h.total;
    c.st.full_stencil_calcs = h.full;
    c.nbrPattern = pattern;
    return SJ_OK;
}

void join_args_base(Ctx &c, sj_join_args &a)
{
    memset(&a, 0, sizeof(a));
    a.xs = c.xs.p;
    a.ids = c.ids.p;
    a.cellStart = c.cellStart.p;
    a.nbrStart = c.nbrStart.p;
    a.nbrCell = c.nbrCell.p;
    a.cellCoord = c.cellCoord.p;
}

// FP32 filter bounds.  Queries are taken relative to their home cell's centre
// (indexed dims) or the data centre (others): |a| <= Ra; candidates lie in the
// home cell or a neighbour: |b| <= Rb.  The kernel evaluates in FP32
//     y = fl(|b|^2 - tLo) + sum_l fl(-2 a_l) b_l     (D+2 roundings),
// with tLo = RD(T - |a|^2 - M).  With u = 2^-24 and r = Ra + Rb:
//   * chain rounding <= (D+2) u (r^2 + T + M),
//   * rounding the local coordinates moves |b - a|^2 by <= 2 u r^2,
//   * the FP64 predicate's own rounding (d2 vs the exact |dx|^2) <= 2^-49 r^2,
// so M = 2 (D+4) u (r^2 + T) + 2^-39 (r^2 + T) exceeds their sum: y <= 0 proves
// d2 <= T.  y >= delta proves d2 > T when delta >= 2M + 2u (T + Ra^2 + M) (the
// second term covers rounding tLo down).  Pairs with 0 < y < delta are
// re-evaluated in FP64.
struct FilterBounds {
    double margin;
    float delta;
};

FilterBounds filter_bounds(const Ctx &c)
{
    const sj_grid_dev &g = c.g;
    double ra2 = 0, rb2 = 0;
    for (int j = 0; j < g.D; j++) {
        if (j < g.k) {
            ra2 += (0.5 * g.eps * 1.01) * (0.5 * g.eps * 1.01);
            rb2 += (1.5 * g.eps * 1.01) * (1.5 * g.eps * 1.01);
        } else {
            double h = 0.5 * (c.dataMax[j] - c.dataMin[j]) * 1.01 + 1e-300;
            ra2 += h * h;
            rb2 += h * h;
        }
    }
    const double r = std::sqrt(ra2) + std::sqrt(rb2);
    const double u = std::ldexp(1.0, -24);
    const double T = g.thresh;
    FilterBounds b;
    b.margin = 2.0 * (g.D + 4) * u * (r * r + T) + std::ldexp(r * r + T, -39);
    const double d = (2.0 * b.margin + 2.0 * u * (T + ra2 + b.margin)) * (1.0 + std::ldexp(1.0, -20));
    float df = (float)d;
    if ((double)df < d) df = std::nextafter(df, INFINITY);
    b.delta = df;
    return b;
}

// --------------------------------------------------------------- tasks --
struct BatchRange {
    uint32_t t0, t1;
    double pred;      // planned batch: its predicted pairs; a part re-planned after an overflow: -1
    uint64_t exact;   // a re-planned part: its measured pairs (0 for a planned batch)
};

sj_status run_count(Ctx &c, sj_join_args &a, bool queue, cudaStream_t st = nullptr, int maxCtasPerSM = 0)
{
    if (!st) st = c.s;
    if (queue) CK(cudaMemsetAsync(c.queueHead.p, 0, sizeof(uint32_t), st));
    CK(sj_launch_join(a, c.g, c.p.precision == SJ_PREC_FP32_REFINE ? 1 : 0, queue ? 1 : 0, c.numSM, maxCtasPerSM,
                      st));
    return SJ_OK;
}

// Resident CTAs per SM of the count pass and the emission when they run side by
// side on two streams (0: as many as fit).  Kernels that each fill every SM
// would only take turns; smaller grids let both be resident at once, so the
// emission's memory-latency-bound warps use the issue slots the count pass
// leaves.  SJ_JOIN_CTAS / SJ_EMIT_CTAS override them.
void pipe_ctas(int &join, int &emit)
{
    join = 0;
    emit = 0;
    if (const char *e = getenv("SJ_JOIN_CTAS")) join = atoi(e);
    if (const char *e = getenv("SJ_EMIT_CTAS")) emit = atoi(e);
}

// Hit-mask words (row or column) one batch may record (4 bytes each); a batch
// is also cut when its masks would exceed this.  SJ_MASK_WORDS overrides it
// (a tuning knob, at most 2^31).
uint64_t mask_batch_words()
{
    uint64_t w = 1ULL << 30;
    if (const char *e = getenv("SJ_MASK_WORDS")) {
        const double v = atof(e);
        if (v >= 65536.0 && v <= 2147483648.0) w = (uint64_t)v;
    }
    return w;
}

// The task list, built on the device (sj_tasks.cu): per-cell workload and cost
// key, the cost order (stable radix sort, heaviest first, ties in cell order),
// one work item per (cell, segment group, query tile) and its tasks.  policy:
// 0 cost-proportional stream chunks, 1 fixed chunks, 2 the mode-8 split by
// thirds of the work (0 and 2 predict pairs from c.rate).  sampleRate > 0 builds the sampling
// estimator's tasks.  With `shard`, keeps this context's shard of the list.
// Sets c.nTasks; the tasks are in c.dTasks, their predicted pairs in c.dTaskPred.
sj_status build_tasks_dev(Ctx &c, bool sym, uint64_t cap, bool byCost, int policy, float sampleRate, bool shard)
{
    const uint32_t nc = c.nCells;
    cudaStream_t s = c.s;
    sj_taskgen g{};
    g.cellStart = c.cellStart.p;
    g.nbrStart = c.nbrStart.p;
    g.nbrCell = c.nbrCell.p;
    g.rate = policy == 1 ? nullptr : c.rate.p;   // the split of policy 2 ignores it, its predictions do not
    g.nCells = nc;
    g.tile = SJ_CTA * (uint32_t)sj_query_slots(c.g.Dp, c.p.precision == SJ_PREC_FP32_REFINE);
    g.cap = cap;
    // predicted pairs per task: about 4096 tasks per full batch.  SJ_TASK_PAIRS
    // overrides it (a tuning knob: profiling runs at a reduced batch capacity
    // use it to keep the task shapes of the full-capacity run)
    g.pairsPerTask = std::max(4096.0, (double)cap / 4096.0);
    if (const char *ev = getenv("SJ_TASK_PAIRS")) {
        const double v = atof(ev);
        if (v >= 1.0) g.pairsPerTask = v;
    }
    // evaluations per task at most: about 2 ms of one count-pass CTA, so a
    // batch's tail is short next to its ~10^10 evaluations over ~740 CTAs.
    // SJ_TASK_EVALS overrides it (0: no limit; a tuning knob)
    g.evalsPerTask = 4.0e6;
    if (const char *ev = getenv("SJ_TASK_EVALS")) g.evalsPerTask = std::max(0.0, atof(ev));
    g.sym = sym ? 1 : 0;
    g.policy = policy;
    g.sampleRate = sampleRate;
    // the learned scheduler shares a cell's predicted neighbour pairs among its
    // tasks by the offset-class model its features use; the sampling estimate
    // keeps the cell's mean rate
    g.spread = (c.rateLearned && policy != 1) ? 1 : 0;
    g.nbrPre = c.nbrPre.p;
    g.nbrPreW = c.nbrPreW.p;
    g.nbrWt = c.nbrWt.p;
    g.cellW = c.cellW.p;
    DevBuf<uint8_t> &tmp = c.sTemp;
    CK(tmp.ensure(std::max(sj_scan_temp_bytes(nc + 1), sj_radix_temp_bytes(nc))));
    CK(c.tgTot32.ensure(2));
    CK(c.tgTotals.ensure(4));
    CK(cudaMemsetAsync(c.tgTotals.p, 0, sizeof(unsigned long long) * 4, s));
    // segment groups of every cell and their slots (at most one group per
    // SJ_MAX_SEG owned neighbours, plus one per cell)
    CK(c.tgGroupCnt.ensure(nc + 1));
    CK(c.tgGroupBase.ensure(nc + 1));
    CK(c.tgGroupLen.ensure((size_t)nc + c.nbrTotal / SJ_MAX_SEG + 1));
    CK(sj_tg_groups(g, c.tgGroupCnt.p, s));
    CK(sj_exclusive_scan_u32(c.tgGroupCnt.p, c.tgGroupBase.p, nc, tmp.p, c.tgTot32.p, s));
    g.groupBase = c.tgGroupBase.p;
    g.groupLen = c.tgGroupLen.p;
    // per-cell task counts, evaluations and cost keys, in cell order
    CK(c.tgPosCnt.ensure(nc + 1));
    CK(c.tgPosEv.ensure(nc + 1));
    CK(c.tgKeys.ensure(nc));
    CK(c.tgKeysAlt.ensure(nc));
    CK(c.tgOrder.ensure(nc));
    CK(c.tgOrderAlt.ensure(nc));
    CK(sj_tg_cells(g, nullptr, nullptr, c.tgPosCnt.p, c.tgPosEv.p,
                   byCost ? reinterpret_cast<unsigned long long *>(c.tgKeys.p) : nullptr, c.tgTotals.p, s));
    CK(sj_iota_u32(c.tgOrder.p, nc, s));
    uint32_t *order = c.tgOrder.p;
    if (byCost && nc > 1) {
        int inAlt = 0;
        CK(sj_radix_sort_u64_u32(c.tgKeys.p, c.tgOrder.p, c.tgKeysAlt.p, c.tgOrderAlt.p, nc, 64, tmp.p, &inAlt, s));
        if (inAlt) order = c.tgOrderAlt.p;
    }
    const uint8_t *workers = nullptr;
    unsigned long long *taskTotal = c.tgTotals.p;
    if (policy == 2) {
        // mode 8: the evaluations in cost order decide each cell's third of the
        // work, which sets how many tasks share each of its tiles' streams
        CK(sj_tg_cells(g, order, nullptr, c.tgPosCnt.p, c.tgPosEv.p, nullptr, c.tgTotals.p + 2, s));
        CK(c.tgEvExcl.ensure(nc + 1));
        CK(c.tgScan64.ensure(sj_scan64_temp(nc)));
        CK(sj_exclusive_scan_u64(c.tgPosEv.p, c.tgEvExcl.p, nc, c.tgScan64.p, s));
        CK(c.tgWorkers.ensure(nc));
        CK(sj_tg_thirds(c.tgEvExcl.p, nc, c.tgWorkers.p, s));
        workers = c.tgWorkers.p;
        CK(cudaMemsetAsync(c.tgTotals.p + 2, 0, sizeof(unsigned long long) * 2, s));
        CK(sj_tg_cells(g, order, workers, c.tgPosCnt.p, c.tgPosEv.p, nullptr, c.tgTotals.p + 2, s));
        taskTotal = c.tgTotals.p + 2;
    }
    // work items in order and their first tasks
    CK(c.tgItemCnt.ensure(nc + 1));
    CK(c.tgItemStart.ensure(nc + 1));
    CK(sj_tg_item_counts(g, order, c.tgItemCnt.p, s));
    CK(sj_exclusive_scan_u32(c.tgItemCnt.p, c.tgItemStart.p, nc, tmp.p, c.tgTot32.p, s));
    struct {
        uint32_t items;
        unsigned long long tasks;
    } h{};
    CK(cudaMemcpyAsync(&h.items, c.tgTot32.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&h.tasks, taskTotal, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (h.tasks > 0xffffffffULL) {
        set_error("%llu tasks exceed the 32-bit task index", h.tasks);
        return SJ_ERR_BAD_INPUT;
    }
    const uint32_t nItems = h.items;
    CK(c.tgItemTasks.ensure((size_t)nItems + 1));
    CK(c.tgItemTaskStart.ensure((size_t)nItems + 1));
    CK(tmp.ensure(sj_scan_temp_bytes((uint64_t)nItems + 1)));
    CK(sj_tg_item_tasks(g, order, workers, c.tgItemStart.p, nItems, c.tgItemTasks.p, s));
    CK(sj_exclusive_scan_u32(c.tgItemTasks.p, c.tgItemTaskStart.p, nItems, tmp.p, c.tgTot32.p + 1, s));
    uint32_t nt = 0;
    CK(cudaMemcpyAsync(&nt, c.tgTot32.p + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (nt != h.tasks) {
        set_error("internal: task builder counted %llu tasks per cell but %u per item", h.tasks, nt);
        return SJ_ERR_INTERNAL;
    }
    CK(c.dTasks.ensure(nt ? nt : 1));
    CK(c.dTaskPred.ensure(nt ? nt : 1));
    CK(sj_tg_item_write(g, order, workers, c.tgItemStart.p, nItems, c.tgItemTaskStart.p, c.dTasks.p, c.dTaskPred.p, s));
    if (shard && c.p.shard_count > 1) {
        // round-robin over the ordered list: each shard gets a similar cost mix
        const uint32_t idx = (uint32_t)c.p.shard_index, cnt = (uint32_t)c.p.shard_count;
        const uint32_t nOut = nt > idx ? (nt - idx + cnt - 1) / cnt : 0u;
        CK(c.dTasksAlt.ensure(nOut ? nOut : 1));
        CK(c.dTaskPredAlt.ensure(nOut ? nOut : 1));
        CK(sj_tg_shard(c.dTasks.p, c.dTaskPred.p, nOut, idx, cnt, c.dTasksAlt.p, c.dTaskPredAlt.p, s));
        c.dTasks.swap(c.dTasksAlt);
        c.dTaskPred.swap(c.dTaskPredAlt);
        nt = nOut;
    }
    c.nTasks = nt;
    return SJ_OK;
}

// Record offsets of c's task list (c.off[0..6], see Ctx).
sj_status task_offsets_dev(Ctx &c)
{
    const uint32_t nt = c.nTasks;
    unsigned long long *out[7];
    for (int k = 0; k < 7; k++) {
        CK(c.off[k].ensure((size_t)nt + 1));
        out[k] = c.off[k].p;
    }
    CK(c.offTemp.ensure(sj_task_offsets_temp(nt)));
    CK(sj_task_offsets(c.dTasks.p, c.dTaskPred.p, nt, c.p.alpha, c.offTemp.p, out, c.s));
    return SJ_OK;
}

// Greedy batch plan on the device: consecutive tasks whose planned pairs
// (predicted x (1 + alpha)) fit `cap` and whose hit masks fit their limit.
// Returns the batches with their predicted pairs, the largest record sizes
// of any batch (row-mask words, column-mask words, row offsets, candidate
// records) and the predicted total.
sj_status plan_dev(Ctx &c, uint64_t cap, std::vector<BatchRange> &plan, uint64_t (&maxes)[4], double &predTotal)
{
    const uint32_t nt = c.nTasks;
    plan.clear();
    for (int k = 0; k < 4; k++) maxes[k] = 1;
    unsigned long long *off[7];
    for (int k = 0; k < 7; k++) off[k] = c.off[k].p;
    CK(c.planNext.ensure(nt ? nt : 1));
    CK(c.planStart.ensure((size_t)nt + 1));
    CK(c.planCount.ensure(1));
    CK(sj_plan_batches(off, nt, cap, mask_batch_words(), c.planNext.p, c.planStart.p, c.planCount.p, c.s));
    struct {
        uint32_t nb;
        unsigned long long pred;
    } h{};
    CK(cudaMemcpyAsync(&h.nb, c.planCount.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, c.s));
    CK(cudaMemcpyAsync(&h.pred, c.off[6].p + nt, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    predTotal = (double)h.pred;
    const uint32_t nb = h.nb;
    if (nb == 0) return SJ_OK;
    CK(c.planStats.ensure((size_t)nb * 5));
    CK(sj_plan_stats(c.planStart.p, nb, off, c.planStats.p, c.s));
    std::vector<uint32_t> start(nb + 1);
    std::vector<unsigned long long> st((size_t)nb * 5);
    CK(cudaMemcpyAsync(start.data(), c.planStart.p, sizeof(uint32_t) * (nb + 1), cudaMemcpyDeviceToHost, c.s));
    CK(cudaMemcpyAsync(st.data(), c.planStats.p, sizeof(unsigned long long) * nb * 5, cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    plan.resize(nb);
    for (uint32_t b = 0; b < nb; b++) {
        plan[b] = {start[b], start[b + 1], (double)st[(size_t)b * 5], 0};
        for (int k = 0; k < 4; k++) maxes[k] = std::max<uint64_t>(maxes[k], st[(size_t)b * 5 + 1 + k]);
    }
    return SJ_OK;
}

// ------------------------------------------------------------ estimate --
// Per-cell predicted hits per evaluation (c.rate), which sizes the tasks,
// orders the queue and plans the batches.  Learned: the MLP on the cell
// features.  Sampling: the count pass over tasks for about sample_rate of
// every cell's points against the cell's whole candidate stream
// (GPU.cu:854-1065 samples every 100th point the same way); cells without a
// sampled point take the global rate.
sj_status estimate_rates(Ctx &c)
{
    Timer tm;
    tm.start(c.s);
    const uint32_t nc = c.nCells;
    CK(c.rate.ensure(2 * (size_t)(nc ? nc : 1)));
    if (c.p.scheduler == SJ_SCHED_LEARNED && !c.mlpW.empty()) {
        DevBuf<float> &out = c.sMlpOut;
        CK(out.ensure((size_t)nc * SJ_NOUT));
        CK(c.dMlpW.ensure(SJ_MLP_NPARAM));
        CK(cudaMemcpyAsync(c.dMlpW.p, c.mlpW.data(), sizeof(float) * SJ_MLP_NPARAM, cudaMemcpyHostToDevice, c.s));
        CK(sj_launch_mlp_infer(c.feat.p, nc, c.dMlpW.p, out.p, c.s));
        CK(sj_rates_mlp(out.p, c.cellStart.p, c.nbrStart.p, c.nbrCell.p, nc, c.rate.p, c.s));
        c.haveSamples = false;
        c.rateLearned = true;
    } else {
        c.rateLearned = false;
        CKS(build_tasks_dev(c, false, 0xffffffffULL, false, 1, (float)c.p.sample_rate, false));
        const uint32_t nt = c.nTasks;
        CK(c.keyCount.ensure(c.n));
        CK(c.stat.ensure(8));
        CK(c.queueHead.ensure(1));
        CK(c.taskHits.ensure(nt ? nt : 1));
        CK(c.dTaskEvals.ensure(nt ? nt : 1));
        CK(c.dTaskRefined.ensure(nt ? nt : 1));
        sj_join_args a;
        join_args_base(c, a);
        a.tasks = c.dTasks.p;
        a.queueHead = c.queueHead.p;
        a.keyCount = c.keyCount.p;   // cleared before the join's first count pass
        a.stat = c.stat.p;
        a.taskHits = c.taskHits.p;
        a.taskEvals = c.dTaskEvals.p;
        a.taskRefined = c.dTaskRefined.p;
        const FilterBounds fb = filter_bounds(c);
        a.margin = fb.margin;
        a.delta = fb.delta;
        a.taskBegin = 0;
        a.taskEnd = nt;
        CKS(run_count(c, a, true));
        CK(c.sHits.ensure(2 * (size_t)(nc ? nc : 1)));
        CK(c.sCands.ensure(2 * (size_t)(nc ? nc : 1)));
        CK(c.sScalars.ensure(2 + sj_sample_totals_len()));
        CK(sj_sample_rates(c.dTasks.p, nt, c.taskHits.p, c.dTaskEvals.p, c.cellStart.p, c.sHits.p, c.sCands.p,
                           c.sScalars.p + 2, nc, c.rate.p, c.s));
        c.haveSamples = true;
    }
    c.st.ms_estimate = tm.stop(c.s);
    return SJ_OK;
}

// ---------------------------------------------------------------- join --
sj_status prepare_join(Ctx &c, int &pattern, bool &queue)
{
    if (!c.indexed) {
        set_error("index not built: call sj_build_index first");
        return SJ_ERR_STATE;
    }
    pattern = pattern_of_mode(c.p.search_mode);
    // work queue: modes 9/10, or any mode when work is ordered by workload
    queue = (c.p.search_mode == 8 || c.p.search_mode == 9 || c.p.search_mode == 10 || c.p.sort_by_workload != 0);
    Timer tm;
    tm.start(c.s);
    CKS(build_neighbours(c, pattern));
    c.st.ms_tasks = tm.stop(c.s);
    CKS(estimate_rates(c));
    return SJ_OK;
}

uint64_t auto_capacity(Ctx &c)
{
    if (c.p.batch_capacity_pairs) return c.p.batch_capacity_pairs;
    size_t freeB = 0, totalB = 0;
    cudaMemGetInfo(&freeB, &totalB);
    uint64_t byMem = (uint64_t)(0.4 * (double)freeB / 8.0);
    return std::max<uint64_t>(1 << 20, std::min<uint64_t>(byMem, 2000000000ULL));
}

// Fills key[b, e) with k using non-temporal 32-byte stores (the destination
// is written once and read later by the consumer: streaming stores skip the
// read-for-ownership of every line, which halves the host memory traffic
// while the copy engine is writing the same memory).
__attribute__((target("avx2"))) static void fill_run_stream(int32_t *key, uint64_t b, uint64_t e, int32_t k)
{
    uint64_t i = b;
    while (i < e && (((uintptr_t)(key + i)) & 31u)) key[i++] = k;
    const __m256i v = _mm256_set1_epi32(k);
    for (; i + 8 <= e; i += 8) _mm256_stream_si256(reinterpret_cast<__m256i *>(key + i), v);
    for (; i < e; i++) key[i] = k;
}

// Keys of a delivered batch from its run offsets: key k owns slots
// [start[k], start[k+1]) (start[n] = cnt).  Parallel over keys on the host.
void expand_keys_host(const uint32_t *start, uint64_t n, uint64_t cnt, int32_t *key)
{
    if (cnt == 0) return;
    static const bool avx2 = __builtin_cpu_supports("avx2");
#pragma omp parallel
    {
#pragma omp for schedule(static)
        for (int64_t k = 0; k < (int64_t)n; k++) {
            const uint64_t b = start[k];
            const uint64_t e = (k + 1 < (int64_t)n) ? start[k + 1] : cnt;
            if (avx2 && e - b >= 64) {
                fill_run_stream(key, b, e, (int32_t)k);
            } else {
                for (uint64_t i = b; i < e; i++) key[i] = (int32_t)k;
            }
        }
        _mm_sfence();   // streaming stores are visible before the consumer reads them
    }
}

// Splits batch br into consecutive task ranges whose measured pair counts
// (taskHits, exact after a count pass over br) fit cap; appends them to `out`
// in ascending task order.
sj_status replan_exact(const BatchRange &br, const std::vector<uint32_t> &taskHits, uint64_t cap,
                       std::vector<BatchRange> &out)
{
    std::vector<BatchRange> parts;
    uint32_t t0 = br.t0;
    uint64_t acc = 0;
    for (uint32_t t = br.t0; t < br.t1; t++) {
        const uint64_t h = taskHits[t];
        if (h > cap) {
            set_error("a single task produces %llu pairs, more than the batch capacity %llu",
                      (unsigned long long)h, (unsigned long long)cap);
            return SJ_ERR_INTERNAL;
        }
        if (t > t0 && acc + h > cap) {
            parts.push_back({t0, t, -1.0, acc});
            t0 = t;
            acc = 0;
        }
        acc += h;
    }
    parts.push_back({t0, br.t1, -1.0, acc});
    out.insert(out.end(), parts.begin(), parts.end());
    return SJ_OK;
}

// Key array of the current batch (a.outKey, a.capacity) from a.keyStart and
// the batch's scan total (default: c.total).
sj_status expand_keys(Ctx &c, const sj_join_args &a, cudaStream_t st = nullptr, const uint32_t *scanTotal = nullptr)
{
    if (!st) st = c.s;
    if (!scanTotal) scanTotal = c.total.p;
    const size_t slots = sj_expand_long_slots(a.capacity);
    CK(c.longRuns.ensure(slots));
    CK(c.longCount.ensure(1));
    CK(sj_expand_keys(a.keyStart, scanTotal, c.n, a.outKey, a.batchPairs, a.capacity, c.longRuns.p,
                      (uint32_t)std::min<size_t>(c.longRuns.n, 0xffffffffu), c.longCount.p, c.numSM, st));
    return SJ_OK;
}

// Internal delivery mode of run_join: every batch is appended to the device
// CSR table set up by sj_neighbor_csr.
constexpr int SJ_DELIVER_CSR = 100;

sj_status run_join(Ctx &c, int delivery, sj_batch_cb cb, void *user)
{
    const unsigned long long launches0 = sj_launch_total();
    Timer total;
    total.start(c.s);
    int pattern;
    bool queue;
    CKS(prepare_join(c, pattern, queue));
    const uint64_t n = c.n;
    uint64_t cap = auto_capacity(c);
    if (cap > 0xffffffffULL) cap = 0xffffffffULL;
    std::vector<BatchRange> plan;
    uint64_t maxes[4];
    double predTotal = 0;
    {
        Timer tm;
        tm.start(c.s);
        const bool byCost = c.p.sort_by_workload || c.p.search_mode == 7 || c.p.search_mode == 8 ||
                            c.p.search_mode == 9 || c.p.search_mode == 10;
        // mode 8 splits each tile's stream by the third of the work its cell is in
        CKS(build_tasks_dev(c, pattern != SJ_PAT_FULL, cap, byCost, c.p.search_mode == 8 ? 2 : 0, 0.0f, true));
        CKS(task_offsets_dev(c));
        // greedy batch plan on predicted pairs (and on hit-mask words)
        CKS(plan_dev(c, cap, plan, maxes, predTotal));
        c.st.ms_tasks += tm.stop(c.s);
    }
    const uint32_t nt = c.nTasks;
    c.st.num_tasks = nt;
    c.st.estimated_pairs = predTotal;
    const uint64_t maxMaskWords = maxes[0], maxColWords = maxes[1], maxRowWords = maxes[2], maxCandRecs = maxes[3];
    CK(c.keyCount.ensure(n));
    CK(c.keyStart.ensure(n));
    CK(c.scanTemp.ensure(sj_scan_temp_bytes(n)));
    CK(c.total.ensure(1));
    CK(c.stat.ensure(8));
    CK(c.queueHead.ensure(1));
    CK(c.taskHits.ensure(nt ? nt : 1));
    CK(cudaMemsetAsync(c.taskHits.p, 0, sizeof(uint32_t) * (nt ? nt : 1), c.s));
    CK(c.dTaskEvals.ensure(nt ? nt : 1));
    CK(c.dTaskRefined.ensure(nt ? nt : 1));
    CK(cudaMemsetAsync(c.dTaskEvals.p, 0, sizeof(uint32_t) * (nt ? nt : 1), c.s));
    CK(cudaMemsetAsync(c.dTaskRefined.p, 0, sizeof(uint32_t) * (nt ? nt : 1), c.s));
    CK(c.pinTotal.ensure(64));
    CK(cudaMemsetAsync(c.stat.p, 0, sizeof(unsigned long long) * 8, c.s));

    std::reverse(plan.begin(), plan.end());   // used as a stack
    CK(c.masks.ensure(maxMaskWords));
    CK(c.colMasks.ensure(maxColWords));
    CK(c.rowRel.ensure(maxRowWords));
    CK(c.candId.ensure(maxCandRecs));
    CK(c.candRel.ensure(maxCandRecs));

    sj_join_args a;
    join_args_base(c, a);
    a.tasks = c.dTasks.p;
    a.queueHead = c.queueHead.p;
    a.keyCount = c.keyCount.p;
    a.keyStart = c.keyStart.p;
    a.outKey = c.outKey.p;
    a.outVal = c.outVal.p;
    a.capacity = cap;
    a.stat = c.stat.p;
    a.taskHits = c.taskHits.p;
    a.taskEvals = c.dTaskEvals.p;
    a.taskRefined = c.dTaskRefined.p;
    a.masks = c.masks.p;
    a.maskOff = reinterpret_cast<const uint64_t *>(c.off[0].p);
    a.colMasks = c.colMasks.p;
    a.colOff = reinterpret_cast<const uint64_t *>(c.off[1].p);
    a.rowRel = c.rowRel.p;
    a.rowOff = reinterpret_cast<const uint64_t *>(c.off[2].p);
    a.candId = c.candId.p;
    a.candRel = c.candRel.p;
    a.candOff = reinterpret_cast<const uint64_t *>(c.off[3].p);
    a.unitOff = reinterpret_cast<const uint64_t *>(c.off[4].p);
    {
        const FilterBounds fb = filter_bounds(c);
        a.margin = fb.margin;
        a.delta = fb.delta;
    }

    std::vector<uint32_t> hTaskHits(nt);
    uint64_t pairsTotal = 0, batches = 0, retries = 0, errBatches = 0;
    double relErrSum = 0;
    float msCount = 0, msScan = 0, msFill = 0, msDeliver = 0, msExpand = 0;
    int pinSel = 0;
    sj_status result = SJ_OK;
    CK(c.batchTot.ensure(plan.size() + 1));
    CK(cudaMemsetAsync(c.keyCount.p, 0, sizeof(uint32_t) * n, c.s));   // each scan clears it again
    // estimator error of a planned batch against its measured pairs
    auto noteErr = [&](const BatchRange &br, uint64_t measured) {
        if (br.pred >= 0 && measured > 0) {
            relErrSum += std::fabs(br.pred - (double)measured) / (double)measured;
            errBatches++;
        }
    };

    // ---- asynchronous phase: batches folded on the device (no host delivery).
    // Every batch runs count -> scan -> emission -> fold without a host round
    // trip; a batch whose count exceeds the output buffer skips its emission
    // and fold.  Such batches are re-planned exactly from the count pass's
    // per-task pairs and run through the same pipeline in a further round (the
    // exact parts cannot overflow again).
    std::vector<BatchRange> stack;
    std::vector<BatchRange> todo;
    if (delivery == SJ_DELIVER_NONE) todo.assign(plan.rbegin(), plan.rend());   // ascending task order
    for (int round = 0; !todo.empty(); round++) {
        double maxPairs = 0;
        for (const BatchRange &br : todo)
            maxPairs = std::max(maxPairs, br.pred >= 0 ? br.pred * (1.0 + c.p.alpha) : (double)br.exact);
        uint64_t bufCap = c.p.batch_capacity_pairs ? cap
                                                   : std::min<uint64_t>(cap, (uint64_t)(1.25 * maxPairs) + 65536);
        if (bufCap > c.outKey.n) {
            CK(c.outKey.ensure(bufCap));
            CK(c.outVal.ensure(bufCap));
        }
        bufCap = c.outKey.n;
        a.outKey = c.outKey.p;
        a.outVal = c.outVal.p;
        a.capacity = bufCap;
        CK(c.foldChunkKey.ensure(sj_fold_chunks(bufCap)));
        CK(c.batchTot.ensure(todo.size() + 1));
        CK(cudaMemsetAsync(c.batchTot.p, 0, sizeof(unsigned long long) * (todo.size() + 1), c.s));
        const size_t nplan = todo.size();
        // Two streams when the device has room for a second record set: the
        // count pass and scan of each batch on the engine's stream, its key
        // expansion, emission and fold on the second stream, so batch i + 1's
        // count pass and scan run beside batch i's emission (and the launch
        // tails of each stage fill with the other's work).  Batches alternate
        // between two sets of count-pass records and two sets of key offsets
        // and scan totals; batch i's count pass waits for batch i - 2's fold,
        // the last reader of the set it reuses (the emission reads the
        // records, the fold the key offsets and the scan total).
        // SJ_SERIAL=1 keeps every stage on the engine's stream (a diagnostic
        // knob: the per-stage CUDA-event times are then those of each stage alone)
        const char *serialEnv = getenv("SJ_SERIAL");
        bool pipe = nplan > 1 && !(serialEnv && atoi(serialEnv) != 0);
        if (pipe) {
            cudaError_t e = c.masks2.ensure(maxMaskWords);
            if (e == cudaSuccess) e = c.colMasks2.ensure(maxColWords);
            if (e == cudaSuccess) e = c.rowRel2.ensure(maxRowWords);
            if (e == cudaSuccess) e = c.candId2.ensure(maxCandRecs);
            if (e == cudaSuccess) e = c.candRel2.ensure(maxCandRecs);
            if (e == cudaSuccess) e = c.emitHead.ensure(1);
            if (e == cudaSuccess) e = c.keyStart2.ensure(n);
            if (e == cudaSuccess) e = c.total2.ensure(1);
            if (e != cudaSuccess) {
                // no room for the second set: the batches run one after another
                cudaGetLastError();
                c.masks2.release();
                c.colMasks2.release();
                c.rowRel2.release();
                c.candId2.release();
                c.candRel2.release();
                c.keyStart2.release();
                pipe = false;
            }
        }
        cudaStream_t sA = c.s, sB = pipe ? c.cs : c.s;
        int joinCtas, emitCtas;
        pipe_ctas(joinCtas, emitCtas);
        // the second stream's work is waited for on every way out
        struct Drain {
            cudaStream_t s;
            ~Drain()
            {
                if (s) cudaStreamSynchronize(s);
            }
        } drain{pipe ? sB : nullptr};
        constexpr int EV = 8;   // events per batch
        while (c.events.size() < EV * nplan) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            c.events.push_back(e);
        }
        cudaEvent_t *ev = c.events.data();
        for (size_t i = 0; i < nplan; i++) {
            const BatchRange &br = todo[i];
            cudaEvent_t *e = ev + EV * i;
            sj_join_args b = a;
            b.taskBegin = br.t0;
            b.taskEnd = br.t1;
            b.batchPairs = c.batchTot.p + i;
            const bool second = pipe && (i & 1);
            uint32_t *const scanTot = second ? c.total2.p : c.total.p;
            if (second) {
                b.masks = c.masks2.p;
                b.colMasks = c.colMasks2.p;
                b.rowRel = c.rowRel2.p;
                b.candId = c.candId2.p;
                b.candRel = c.candRel2.p;
                b.keyStart = c.keyStart2.p;
            }
            if (pipe && i > 1) CK(cudaStreamWaitEvent(sA, ev[EV * (i - 2) + 7], 0));   // set reused: fold i-2 done
            CK(cudaEventRecord(e[0], sA));
            CKS(run_count(c, b, queue, sA, pipe ? joinCtas : 0));
            CK(cudaEventRecord(e[1], sA));
            CK(cudaEventRecord(e[2], sA));
            CK(sj_exclusive_scan_u32_clear(c.keyCount.p, const_cast<uint32_t *>(b.keyStart), n, c.scanTemp.p, scanTot,
                                           sA));
            CK(cudaEventRecord(e[3], sA));
            if (pipe) CK(cudaStreamWaitEvent(sB, e[3], 0));
            // emission (values), then the consumer fold, which reads the values
            // back and writes the key array in the same pass
            CK(cudaEventRecord(e[4], sB));
            CK(cudaEventRecord(e[5], sB));
            b.queueHead = pipe ? c.emitHead.p : c.queueHead.p;
            CK(cudaMemsetAsync(b.queueHead, 0, sizeof(uint32_t), sB));
            CK(sj_launch_emit(b, c.numSM, pipe ? emitCtas : 0, sB));
            CK(cudaEventRecord(e[6], sB));
            CK(sj_fold(b.keyStart, scanTot, n, c.outVal.p, c.outKey.p, b.batchPairs, bufCap, c.foldChunkKey.p,
                       c.stat.p + 4, c.numSM, sB));
            CK(cudaEventRecord(e[7], sB));
        }
        if (pipe) CK(cudaStreamWaitEvent(sA, ev[EV * (nplan - 1) + 7], 0));
        std::vector<unsigned long long> tot(nplan);
        CK(cudaMemcpyAsync(tot.data(), c.batchTot.p, sizeof(unsigned long long) * nplan, cudaMemcpyDeviceToHost,
                           c.s));
        CK(cudaMemcpyAsync(hTaskHits.data(), c.taskHits.p, sizeof(uint32_t) * nt, cudaMemcpyDeviceToHost, c.s));
        CK(cudaStreamSynchronize(c.s));
        // stage times per batch (with two streams, each stage's time includes
        // sharing the device with the other stream's stage)
        for (size_t i = 0; i < nplan; i++) {
            const cudaEvent_t *e = ev + EV * i;
            float tc, ts, tx, tf, th;
            cudaEventElapsedTime(&tc, e[0], e[1]);
            cudaEventElapsedTime(&ts, e[2], e[3]);
            cudaEventElapsedTime(&tx, e[4], e[5]);
            cudaEventElapsedTime(&tf, e[5], e[6]);
            cudaEventElapsedTime(&th, e[6], e[7]);
            msCount += tc;
            msScan += ts;
            msExpand += tx;
            msFill += tf;
            msDeliver += th;
        }
        // SJ_BATCH_LOG=<file>: one line per batch of this round appended to the
        // file (a diagnostic knob): tasks, pairs, record sizes, stage times
        if (const char *logPath = getenv("SJ_BATCH_LOG")) {
            std::vector<unsigned long long> ho[5];
            for (int q = 0; q < 5; q++) {
                ho[q].resize((size_t)nt + 1);
                CK(cudaMemcpy(ho[q].data(), c.off[q].p, sizeof(unsigned long long) * (nt + 1),
                              cudaMemcpyDeviceToHost));
            }
            if (FILE *lf = fopen(logPath, "a")) {
                for (size_t i = 0; i < nplan; i++) {
                    const BatchRange &br = todo[i];
                    const cudaEvent_t *e = ev + EV * i;
                    float tc, tf, th;
                    cudaEventElapsedTime(&tc, e[0], e[1]);
                    cudaEventElapsedTime(&tf, e[5], e[6]);
                    cudaEventElapsedTime(&th, e[6], e[7]);
                    fprintf(lf,
                            "{\"round\": %d, \"batch\": %zu, \"t0\": %u, \"t1\": %u, \"pairs\": %llu, "
                            "\"row_words\": %llu, \"col_words\": %llu, \"query_recs\": %llu, \"cand_recs\": %llu, "
                            "\"units\": %llu, \"count_ms\": %.4f, \"emit_ms\": %.4f, \"fold_ms\": %.4f}\n",
                            round, i, br.t0, br.t1, tot[i], ho[0][br.t1] - ho[0][br.t0], ho[1][br.t1] - ho[1][br.t0],
                            ho[2][br.t1] - ho[2][br.t0], ho[3][br.t1] - ho[3][br.t0], ho[4][br.t1] - ho[4][br.t0], tc,
                            tf, th);
                }
                fclose(lf);
            }
        }
        std::vector<BatchRange> redo;
        for (size_t i = 0; i < nplan; i++) {
            const BatchRange &br = todo[i];
            noteErr(br, tot[i]);   // the count pass measured the batch exactly, overflowed or not
            if (tot[i] > bufCap) {
                // the count pass measured every task's pairs: re-plan this
                // batch's tasks exactly against the capacity (the next round
                // grows the buffers up to it; no task's worst case exceeds it)
                CKS(replan_exact(br, hTaskHits, cap, redo));
                retries++;
                continue;
            }
            pairsTotal += tot[i];
            batches++;
        }
        todo.swap(redo);
    }
    if (delivery != SJ_DELIVER_NONE) stack = plan;

    // ---- synchronous phase: host / device delivery, and batches to re-plan.
    // Host delivery does not copy the key array over PCIe: the keys of a
    // batch are ascending runs, so the copy stream brings back the values and
    // the per-key run offsets (keyStart), and the host cores expand the keys
    // into pinned memory.  A batch is handed to the callback after the next
    // batch's GPU work and copies have been queued, so the expansion and the
    // callback overlap them (double-buffered pinned sets).
    unsigned long long *slot = c.batchTot.p + plan.size();
    struct Pending {
        bool live = false;
        uint64_t cnt = 0, index = 0;
        int sel = 0;
    } pend;
    bool setUsed[2] = {false, false};
    auto finishPending = [&]() -> sj_status {
        if (!pend.live) return SJ_OK;
        pend.live = false;
        CK(cudaEventSynchronize(c.evVals[pend.sel]));
        int32_t *hk = (int32_t *)c.pinKey[pend.sel].p, *hv = (int32_t *)c.pinVal[pend.sel].p;
        expand_keys_host((const uint32_t *)c.pinStart[pend.sel].p, n, pend.cnt, hk);
        if (cb) {
            sj_batch b{pend.index, pend.cnt, hk, hv, 0};
            if (cb(&b, user)) return SJ_ERR_ABORTED;
        }
        return SJ_OK;
    };
    // stage times: six events per iteration, read after the loop
    size_t iter = 0;
    std::vector<int> iterFull;   // 1: the iteration ran all stages, 0: count + scan only (re-planned)
    auto ev = [&](size_t k) -> cudaEvent_t { return c.syncEvents[6 * iter + k]; };
    const bool hostDel = delivery == SJ_DELIVER_HOST;
    if (hostDel) CK(c.keyStartAlt.ensure(n ? n : 1));
    while (!stack.empty() && result == SJ_OK) {
        BatchRange br = stack.back();
        stack.pop_back();
        while (c.syncEvents.size() < 6 * (iter + 1)) {
            cudaEvent_t e;
            CK(cudaEventCreate(&e));
            c.syncEvents.push_back(e);
        }
        // host delivery alternates between two buffer sets (the pinned sets' index)
        const int sel = hostDel ? pinSel : 0;
        uint32_t *const ksBuf = sel ? c.keyStartAlt.p : c.keyStart.p;
        a.taskBegin = br.t0;
        a.taskEnd = br.t1;
        a.batchPairs = slot;
        a.capacity = c.outKey.n;
        a.keyStart = ksBuf;
        CK(cudaMemsetAsync(slot, 0, sizeof(unsigned long long), c.s));
        CK(cudaEventRecord(ev(0), c.s));
        CKS(run_count(c, a, queue));
        CK(cudaEventRecord(ev(1), c.s));
        // this set's run offsets must have been copied out before the scan rewrites them
        if (setUsed[sel]) CK(cudaStreamWaitEvent(c.s, c.evStart[sel], 0));
        CK(sj_exclusive_scan_u32_clear(c.keyCount.p, ksBuf, n, c.scanTemp.p, c.total.p, c.s));
        CK(cudaEventRecord(ev(2), c.s));
        unsigned long long cnt = 0;
        CK(cudaMemcpyAsync(c.pinTotal.p, slot, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c.s));
        CK(cudaMemcpyAsync(hTaskHits.data() + br.t0, c.taskHits.p + br.t0, sizeof(uint32_t) * (br.t1 - br.t0),
                           cudaMemcpyDeviceToHost, c.s));
        CK(cudaStreamSynchronize(c.s));
        memcpy(&cnt, c.pinTotal.p, sizeof(cnt));
        noteErr(br, cnt);
        if (cnt > cap) {
            // estimate too low: re-plan the batch from the measured per-task
            // pairs (the scan already cleared the counts)
            std::vector<BatchRange> parts;
            CKS(replan_exact(br, hTaskHits, cap, parts));
            for (size_t i = parts.size(); i-- > 0;) stack.push_back(parts[i]);
            retries++;
            iterFull.push_back(0);
            iter++;
            continue;
        }
        // output buffers follow the exact batch size (grow-only, 25% headroom, <= capacity)
        if (cnt > c.outKey.n) {
            CKS(finishPending());   // its copy may still read the old buffers
            CK(cudaStreamSynchronize(c.cs));
            uint64_t want = std::min<uint64_t>(cap, std::max<uint64_t>(cnt, (uint64_t)(1.25 * (double)c.outKey.n)));
            CK(c.outKey.ensure(want));
            CK(c.outVal.ensure(want));
            if (hostDel) CK(c.outValAlt.ensure(want));
        }
        if (hostDel && c.outValAlt.n < c.outVal.n) {
            CKS(finishPending());
            CK(cudaStreamSynchronize(c.cs));
            CK(c.outValAlt.ensure(c.outVal.n));
        }
        int32_t *const valBuf = sel ? c.outValAlt.p : c.outVal.p;
        a.outKey = c.outKey.p;
        a.outVal = valBuf;
        a.capacity = std::min<uint64_t>(c.outKey.n, sel ? c.outValAlt.n : c.outVal.n);
        CKS(expand_keys(c, a));
        CK(cudaEventRecord(ev(3), c.s));
        // this set's values must have been copied out before the emission rewrites them
        if (setUsed[sel]) CK(cudaStreamWaitEvent(c.s, c.evVals[sel], 0));
        CK(cudaMemsetAsync(c.queueHead.p, 0, sizeof(uint32_t), c.s));
        CK(sj_launch_emit(a, c.numSM, 0, c.s));
        CK(cudaEventRecord(ev(4), c.s));
        CK(sj_hash_pairs(c.outKey.p, valBuf, cnt, c.stat.p + 4, c.s));
        if (delivery == SJ_DELIVER_CSR) {
            CK(sj_csr_append(ksBuf, c.total.p, n, valBuf, c.csrRowPtr, c.csrFill.p, c.csrCols, c.csrCap,
                             c.stat.p + 7, c.s));
        } else if (delivery == SJ_DELIVER_DEVICE && cb) {
            CK(cudaStreamSynchronize(c.s));
            sj_batch b{batches, cnt, c.outKey.p, valBuf, 1};
            if (cb(&b, user)) result = SJ_ERR_ABORTED;
        } else if (hostDel) {
            const size_t vb = std::max<size_t>(cnt, 1) * sizeof(int32_t);
            if (vb > c.pinVal[sel].bytes) {
                size_t want = std::max<size_t>(vb, (size_t)(1.25 * (double)c.pinVal[sel].bytes));
                want = std::min<size_t>(std::max<size_t>(want, vb), cap * sizeof(int32_t));
                CK(c.pinKey[sel].ensure(want));
                CK(c.pinVal[sel].ensure(want));
            }
            CK(c.pinStart[sel].ensure(n * sizeof(uint32_t)));
            CK(cudaEventRecord(c.evEmit, c.s));
            CK(cudaStreamWaitEvent(c.cs, c.evEmit, 0));
            CK(cudaMemcpyAsync(c.pinStart[sel].p, ksBuf, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, c.cs));
            CK(cudaEventRecord(c.evStart[sel], c.cs));
            if (cnt) CK(cudaMemcpyAsync(c.pinVal[sel].p, valBuf, cnt * sizeof(int32_t), cudaMemcpyDeviceToHost, c.cs));
            CK(cudaEventRecord(c.evVals[sel], c.cs));
            setUsed[sel] = true;
            // the previous batch goes to the consumer while this one is copied
            sj_status ps = finishPending();
            if (ps != SJ_OK) {
                result = ps;
                if (ps != SJ_ERR_ABORTED) return ps;
            }
            pend.live = true;
            pend.cnt = cnt;
            pend.index = batches;
            pend.sel = sel;
            pinSel ^= 1;
        }
        CK(cudaEventRecord(ev(5), c.s));
        iterFull.push_back(1);
        iter++;
        pairsTotal += cnt;
        batches++;
    }
    if (result == SJ_OK) {
        sj_status ps = finishPending();
        if (ps != SJ_OK) {
            result = ps;
            if (ps != SJ_ERR_ABORTED) return ps;
        }
    }
    CK(cudaStreamSynchronize(c.cs));
    CK(cudaStreamSynchronize(c.s));
    for (size_t i = 0; i < iter; i++) {
        float t01 = 0, t12 = 0, t23 = 0, t34 = 0, t45 = 0;
        cudaEvent_t *e = c.syncEvents.data() + 6 * i;
        cudaEventElapsedTime(&t01, e[0], e[1]);
        cudaEventElapsedTime(&t12, e[1], e[2]);
        msCount += t01;
        msScan += t12;
        if (iterFull[i]) {
            cudaEventElapsedTime(&t23, e[2], e[3]);
            cudaEventElapsedTime(&t34, e[3], e[4]);
            cudaEventElapsedTime(&t45, e[4], e[5]);
            msExpand += t23;
            msFill += t34;
            msDeliver += t45;
        }
    }
    unsigned long long hs[8];
    CK(cudaMemcpyAsync(hs, c.stat.p, sizeof(hs), cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    if (hs[3] || hs[6] || hs[7]) {
        set_error(hs[3]   ? "internal: the emission exceeded the counted capacity"
                  : hs[6] ? "internal: the emission met a count-pass record out of range"
                          : "internal: a neighbour-table row received more values than its degree");
        return SJ_ERR_INTERNAL;
    }
    {
        // evaluations, FP32 re-evaluations, measured pairs and the predicted
        // pairs' error, summed over the tasks on the device
        CK(c.sums.ensure(3));
        CK(c.errSum.ensure(1));
        CK(sj_task_sums(c.dTaskEvals.p, c.dTaskRefined.p, c.taskHits.p, c.dTaskPred.p, nt, c.sums.p, c.errSum.p,
                        c.numSM, c.s));
        unsigned long long sm[3];
        double err = 0;
        CK(cudaMemcpyAsync(sm, c.sums.p, sizeof(sm), cudaMemcpyDeviceToHost, c.s));
        CK(cudaMemcpyAsync(&err, c.errSum.p, sizeof(double), cudaMemcpyDeviceToHost, c.s));
        CK(cudaStreamSynchronize(c.s));
        c.st.distance_calcs = sm[0];
        c.st.refined_pairs = sm[1];
        c.st.estimator_task_rel_err = sm[2] ? err / (double)sm[2] : 0.0;
    }
    if (nt) {
        // the estimator-free reference count: the same greedy plan with every
        // task's measured pairs in place of its prediction
        CK(c.exactPred.ensure(nt));
        CK(sj_u32_to_f32(c.taskHits.p, nt, c.exactPred.p, c.s));
        unsigned long long *o[7];
        for (int k = 0; k < 7; k++) o[k] = c.off[k].p;
        CK(sj_task_offsets(c.dTasks.p, c.exactPred.p, nt, c.p.alpha, c.offTemp.p, o, c.s));
        CK(sj_plan_batches(o, nt, cap, mask_batch_words(), c.planNext.p, c.planStart.p, c.planCount.p, c.s));
        uint32_t nbExact = 0;
        CK(cudaMemcpyAsync(&nbExact, c.planCount.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, c.s));
        CK(cudaStreamSynchronize(c.s));
        c.st.exact_plan_batches = nbExact;
    }
    c.st.total_pairs = pairsTotal;
    c.st.pair_hash = hs[4];
    c.st.num_batches = batches;
    c.st.overflow_retries = retries;
    c.st.estimator_mean_abs_rel_err = errBatches ? relErrSum / (double)errBatches : 0.0;
    c.st.ms_count = msCount;
    c.st.ms_scan = msScan;
    c.st.ms_fill = msFill;
    c.st.ms_deliver = msDeliver;
    c.st.ms_join_kernels = msCount + msFill;
    c.st.ms_fill_kernel = msFill;
    c.st.ms_expand = msExpand;
    c.st.ms_total = total.stop(c.s);
    c.st.kernel_launches = sj_launch_total() - launches0;
    return result;
}

// Degrees only: count pass over all tasks, no capacity limit.
sj_status run_degrees(Ctx &c, uint32_t *degHost)
{
    int pattern;
    bool queue;
    CKS(prepare_join(c, pattern, queue));
    const uint64_t n = c.n;
    CKS(build_tasks_dev(c, pattern != SJ_PAT_FULL, 0xffffffffULL, false, 0, 0.0f, true));
    const uint32_t nt = c.nTasks;
    CK(c.keyCount.ensure(n));
    CK(c.stat.ensure(8));
    CK(c.queueHead.ensure(1));
    CK(cudaMemsetAsync(c.keyCount.p, 0, sizeof(uint32_t) * n, c.s));
    CK(cudaMemsetAsync(c.stat.p, 0, sizeof(unsigned long long) * 8, c.s));
    sj_join_args a;
    join_args_base(c, a);
    a.tasks = c.dTasks.p;
    a.queueHead = c.queueHead.p;
    a.keyCount = c.keyCount.p;
    a.stat = c.stat.p;
    {
        const FilterBounds fb = filter_bounds(c);
        a.margin = fb.margin;
        a.delta = fb.delta;
    }
    CK(c.dTaskEvals.ensure(nt ? nt : 1));
    CK(c.dTaskRefined.ensure(nt ? nt : 1));
    a.taskEvals = c.dTaskEvals.p;
    a.taskRefined = c.dTaskRefined.p;
    a.taskBegin = 0;
    a.taskEnd = nt;
    CKS(run_count(c, a, true));
    // per-cell measured hits (the sum of the cell's points' degrees)
    CK(c.dCellHits.ensure(c.nCells ? c.nCells : 1));
    CK(sj_cell_hits(c.cellStart.p, c.ids.p, c.keyCount.p, c.nCells, c.dCellHits.p, c.s));
    CK(c.sums.ensure(3));
    CK(sj_task_sums(c.dTaskEvals.p, c.dTaskRefined.p, nullptr, nullptr, nt, c.sums.p, nullptr, c.numSM, c.s));
    std::vector<uint32_t> deg(n);
    CK(cudaMemcpyAsync(deg.data(), c.keyCount.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, c.s));
    unsigned long long sm[3];
    CK(cudaMemcpyAsync(sm, c.sums.p, sizeof(sm), cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    if (degHost) memcpy(degHost, deg.data(), sizeof(uint32_t) * n);
    c.haveMeas = true;
    uint64_t tot = 0;
    for (uint64_t i = 0; i < n; i++) tot += deg[i];
    c.st.total_pairs = tot;
    c.st.distance_calcs = sm[0];
    c.st.refined_pairs = sm[1];
    return SJ_OK;
}

sj_status set_points(Ctx &c, const double *pts, uint64_t n, int onDevice)
{
    if (!pts && n) {
        set_error("null points");
        return SJ_ERR_BAD_INPUT;
    }
    if (n == 0 || n > 0x7fffffffULL) {
        set_error("point count must be in 1..2^31-1 (got %llu)", (unsigned long long)n);
        return SJ_ERR_BAD_INPUT;
    }
    Timer tm;
    tm.start(c.s);
    const size_t bytes = n * (size_t)c.p.gpunumdim * sizeof(double);
    CK(c.pts.ensure(n * (size_t)c.p.gpunumdim));
    CK(cudaMemcpyAsync(c.pts.p, pts, bytes, onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c.s));
    c.n = n;
    c.havePoints = true;
    c.indexed = false;
    c.nbrPattern = -1;
    c.st = sj_stats{};
    c.st.ms_upload = tm.stop(c.s);
    return SJ_OK;
}

Ctx *as_ctx(sj_ctx *p) { return reinterpret_cast<Ctx *>(p); }

sj_status bind(Ctx &c)
{
    CK(cudaSetDevice(c.dev));
    return SJ_OK;
}

}  // namespace

void sj_set_error_message(const char *msg) { g_lastError = msg ? msg : ""; }

// =================================================================== C ABI
extern "C" {

void sj_params_default(sj_params *p)
{
    memset(p, 0, sizeof(*p));
    p->gpunumdim = 2;
    p->numindexeddim = 2;
    p->epsilon = 0.01;
    p->blocksize = 256;
    p->threadperpoint = 1;
    p->search_mode = 10;
    p->sort_by_workload = 1;
    p->precision = SJ_PREC_FP64;
    p->scheduler = SJ_SCHED_SAMPLING;
    p->batch_capacity_pairs = 0;
    p->sample_rate = 0.01;
    p->alpha = 0.05;
    p->device = 0;
    p->shard_index = 0;
    p->shard_count = 1;
    p->verbose = 0;
}

sj_status sj_create(const sj_params *p, sj_ctx **out)
{
    if (!p || !out) {
        set_error("null argument");
        return SJ_ERR_BAD_INPUT;
    }
    *out = nullptr;
    sj_status s = check_params(*p);
    if (s != SJ_OK) return s;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        set_error("no CUDA device: %s", cudaGetErrorString(e));
        return SJ_ERR_CUDA;
    }
    if (p->device < 0 || p->device >= ndev) {
        set_error("device %d out of range (have %d)", p->device, ndev);
        return SJ_ERR_BAD_INPUT;
    }
    Ctx *c = new Ctx();
    c->p = *p;
    c->dev = p->device;
    e = cudaSetDevice(c->dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->numSM, cudaDevAttrMultiProcessorCount, c->dev);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->cs, cudaStreamNonBlocking);
    for (int i = 0; i < 2 && e == cudaSuccess; i++) {
        e = cudaEventCreateWithFlags(&c->evStart[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->evVals[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->evEmit, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        set_error("device setup: %s", cudaGetErrorString(e));
        delete c;
        return SJ_ERR_CUDA;
    }
    *out = reinterpret_cast<sj_ctx *>(c);
    return SJ_OK;
}

sj_status sj_destroy(sj_ctx *ctx)
{
    if (!ctx) return SJ_OK;
    Ctx *c = as_ctx(ctx);
    cudaSetDevice(c->dev);
    cudaStreamSynchronize(c->s);
    if (c->cs) cudaStreamSynchronize(c->cs);
    cudaStream_t s = c->s, cs = c->cs;
    for (cudaEvent_t e : c->events) cudaEventDestroy(e);
    for (cudaEvent_t e : c->syncEvents) cudaEventDestroy(e);
    for (int i = 0; i < 2; i++) {
        if (c->evStart[i]) cudaEventDestroy(c->evStart[i]);
        if (c->evVals[i]) cudaEventDestroy(c->evVals[i]);
    }
    if (c->evEmit) cudaEventDestroy(c->evEmit);
    delete c;
    if (s) cudaStreamDestroy(s);
    if (cs) cudaStreamDestroy(cs);
    return SJ_OK;
}

sj_status sj_import_csv(sj_ctx *ctx, const char *path)
{
    if (!ctx || !path) {
        set_error("null argument");
        return SJ_ERR_BAD_INPUT;
    }
    Ctx &c = *as_ctx(ctx);
    CKS(bind(c));
    std::vector<double> pts;
    if (sj::import_csv(path, c.p.gpunumdim, pts) != 0) {
        set_error("cannot read %s", path);
        return SJ_ERR_IO;
    }
    if (pts.empty()) {
        set_error("%s holds no complete %d-dimensional point", path, c.p.gpunumdim);
        return SJ_ERR_BAD_INPUT;
    }
    return set_points(c, pts.data(), pts.size() / c.p.gpunumdim, 0);
}

sj_status sj_read_csv(const char *path, int gpunumdim, double *out, uint64_t cap, uint64_t *n)
{
    if (!path || !n || gpunumdim < 1 || gpunumdim > SJ_MAX_DIM) {
        set_error("bad arguments");
        return SJ_ERR_BAD_INPUT;
    }
    std::vector<double> pts;
    if (sj::import_csv(path, gpunumdim, pts) != 0) {
        set_error("cannot read %s", path);
        return SJ_ERR_IO;
    }
    uint64_t m = pts.size() / (uint64_t)gpunumdim;
    *n = m;
    if (out) memcpy(out, pts.data(), sizeof(double) * (size_t)std::min(m, cap) * gpunumdim);
    return SJ_OK;
}

sj_status sj_set_points(sj_ctx *ctx, const double *pts, uint64_t n, int on_device)
{
    if (!ctx) {
        set_error("null context");
        return SJ_ERR_BAD_INPUT;
    }
    Ctx &c = *as_ctx(ctx);
    CKS(bind(c));
    return set_points(c, pts, n, on_device);
}

sj_status sj_build_index(sj_ctx *ctx)
{
    if (!ctx) return SJ_ERR_BAD_INPUT;
    Ctx &c = *as_ctx(ctx);
    CKS(bind(c));
    return build_index(c);
}

sj_status sj_index_sizes(sj_ctx *ctx, uint32_t *n_nonempty, uint32_t *n_mask_elems, uint64_t *total_cells)
{
    if (!ctx) return SJ_ERR_BAD_INPUT;
    Ctx &c = *as_ctx(ctx);
    if (!c.indexed) {
        set_error("index not built");
        return SJ_ERR_STATE;
    }
    CKS(bind(c));
    if (n_nonempty) *n_nonempty = c.nCells;
    if (total_cells) *total_cells = c.st.total_cells;
    if (n_mask_elems) {
        std::vector<uint32_t> coord((size_t)c.nCells * c.g.k);
        CK(cudaMemcpy(coord.data(), c.cellCoord.p, coord.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        uint32_t tot = 0;
        for (int j = 0; j < c.g.k; j++) {
            std::vector<uint32_t> v(c.nCells);
            for (uint32_t i = 0; i < c.nCells; i++) v[i] = coord[(size_t)i * c.g.k + j];
            std::sort(v.begin(), v.end());
            tot += (uint32_t)(std::unique(v.begin(), v.end()) - v.begin());
        }
        *n_mask_elems = tot;
    }
    return SJ_OK;
}

sj_status sj_index_export(sj_ctx *ctx, unsigned int *indexLookupArr, sj_grid *grid, sj_grid_cell_lookup *lookup,
                          double *minArr, unsigned int *nCells, unsigned int *mask, unsigned int *maskOffsets)
{
    if (!ctx) return SJ_ERR_BAD_INPUT;
    Ctx &c = *as_ctx(ctx);
    if (!c.indexed) {
        set_error("index not built");
        return SJ_ERR_STATE;
    }
    CKS(bind(c));
    const uint32_t nc = c.nCells;
    if (indexLookupArr) CK(cudaMemcpy(indexLookupArr, c.ids.p, sizeof(uint32_t) * c.n, cudaMemcpyDeviceToHost));
    if (grid) {
        std::vector<uint32_t> cs(nc + 1);
        CK(cudaMemcpy(cs.data(), c.cellStart.p, sizeof(uint32_t) * (nc + 1), cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < nc; i++) {
            grid[i].indexmin = (int)cs[i];
            grid[i].indexmax = (int)cs[i + 1] - 1;
        }
    }
    if (lookup) {
        std::vector<uint64_t> lid(nc);
        CK(cudaMemcpy(lid.data(), c.cellLid.p, sizeof(uint64_t) * nc, cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < nc; i++) {
            lookup[i].idx = i;
            lookup[i].gridLinearID = lid[i];
        }
    }
    for (int j = 0; j < c.g.k; j++) {
        if (minArr) minArr[j] = c.g.minArr[j];
        if (nCells) nCells[j] = c.g.nCells[j];
    }
    if (mask || maskOffsets) {
        std::vector<uint32_t> coord((size_t)nc * c.g.k);
        CK(cudaMemcpy(coord.data(), c.cellCoord.p, coord.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        uint32_t off = 0;
        for (int j = 0; j < c.g.k; j++) {
            std::vector<uint32_t> v(nc);
            for (uint32_t i = 0; i < nc; i++) v[i] = coord[(size_t)i * c.g.k + j];
            std::sort(v.begin(), v.end());
            v.erase(std::unique(v.begin(), v.end()), v.end());
            if (maskOffsets) maskOffsets[2 * j] = off;
            for (uint32_t x : v) {
                if (mask) mask[off] = x;
                off++;
            }
            if (maskOffsets) maskOffsets[2 * j + 1] = off - 1;
        }
    }
    return SJ_OK;
}

sj_status sj_join(sj_ctx *ctx, int delivery, sj_batch_cb cb, void *user)
{
    if (!ctx) return SJ_ERR_BAD_INPUT;
    if (delivery < SJ_DELIVER_DEVICE || delivery > SJ_DELIVER_NONE) {
        set_error("unknown delivery mode");
        return SJ_ERR_BAD_INPUT;
    }
    Ctx &c = *as_ctx(ctx);
    CKS(bind(c));
    return run_join(c, delivery, cb, user);
}

sj_status sj_degrees(sj_ctx *ctx, uint32_t *deg)
{
    if (!ctx) return SJ_ERR_BAD_INPUT;
    Ctx &c = *as_ctx(ctx);
    CKS(bind(c));
    return run_degrees(c, deg);
}

struct TableBuild {
    std::vector<uint32_t> *deg;
    std::vector<uint64_t> *cursor;
    int *values;
};

static int table_cb(const sj_batch *b, void *user)
{
    TableBuild *t = (TableBuild *)user;
    for (uint64_t i = 0; i < b->count; i++) {
        uint32_t k = (uint32_t)b->key[i];
        t->values[(*t->cursor)[k]++] = b->val[i];
    }
    return 0;
}

sj_status sj_neighbor_table(sj_ctx *ctx, sj_neighbor_table_lookup *table, int **values, uint64_t *total)
{
    if (!ctx || !table || !values) return SJ_ERR_BAD_INPUT;
    Ctx &c = *as_ctx(ctx);
    CKS(bind(c));
    std::vector<uint32_t> deg(c.n);
    CKS(run_degrees(c, deg.data()));
    uint64_t tot = 0;
    std::vector<uint64_t> start(c.n), cursor(c.n);
    for (uint64_t i = 0; i < c.n; i++) {
        start[i] = tot;
        tot += deg[i];
    }
    if (tot > 0x7fffffffULL) {
        set_error("neighbour table of %llu values exceeds int indexing", (unsigned long long)tot);
        return SJ_ERR_BAD_INPUT;
    }
    int *vals = (int *)malloc(sizeof(int) * (tot ? tot : 1));
    if (!vals) return SJ_ERR_OOM;
    cursor = start;
    TableBuild tb{&deg, &cursor, vals};
    sj_status s = run_join(c, SJ_DELIVER_HOST, table_cb, &tb);
    if (s != SJ_OK) {
        free(vals);
        return s;
    }
    for (uint64_t i = 0; i < c.n; i++) {
        if (cursor[i] != start[i] + deg[i]) {
            free(vals);
            set_error("internal: neighbour table row %llu incomplete", (unsigned long long)i);
            return SJ_ERR_INTERNAL;
        }
        table[i].pointID = (int)i;
        table[i].indexmin = (int)start[i];
        table[i].indexmax = (int)(start[i] + deg[i]) - 1;
        table[i].dataPtr = vals;
    }
    *values = vals;
    if (total) *total = tot;
    return SJ_OK;
}

sj_status sj_neighbor_csr(sj_ctx *ctx, uint64_t *rowPtr, int32_t *cols, uint64_t cols_capacity, uint64_t *total)
{
    if (!ctx || !rowPtr) {
        set_error("null argument");
        return SJ_ERR_BAD_INPUT;
    }
    Ctx &c = *as_ctx(ctx);
    CKS(bind(c));
    // the table is written by kernels: both arrays must be memory the device can write
    for (const void *ptr : {(const void *)rowPtr, (const void *)cols}) {
        if (!ptr) continue;
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess ||
            (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)) {
            cudaGetLastError();
            set_error("rowPtr and cols must be device (or managed) memory");
            return SJ_ERR_BAD_INPUT;
        }
    }
    const uint64_t n = c.n;
    std::vector<uint32_t> deg(n);
    CKS(run_degrees(c, deg.data()));
    std::vector<uint64_t> hp(n + 1);
    hp[0] = 0;
    for (uint64_t i = 0; i < n; i++) hp[i + 1] = hp[i] + deg[i];
    if (total) *total = hp[n];
    CK(cudaMemcpyAsync(rowPtr, hp.data(), sizeof(uint64_t) * (n + 1), cudaMemcpyHostToDevice, c.s));
    CK(cudaStreamSynchronize(c.s));
    if (!cols) return SJ_OK;
    if (cols_capacity < hp[n]) {
        set_error("cols holds %llu values, the table needs %llu", (unsigned long long)cols_capacity,
                  (unsigned long long)hp[n]);
        return SJ_ERR_BAD_INPUT;
    }
    CK(c.csrFill.ensure(n ? n : 1));
    CK(cudaMemsetAsync(c.csrFill.p, 0, sizeof(uint32_t) * (n ? n : 1), c.s));
    c.csrRowPtr = rowPtr;
    c.csrCols = cols;
    c.csrCap = cols_capacity;
    const sj_status s = run_join(c, SJ_DELIVER_CSR, nullptr, nullptr);
    c.csrRowPtr = nullptr;
    c.csrCols = nullptr;
    c.csrCap = 0;
    if (s != SJ_OK) return s;
    // every row must be exactly full
    std::vector<uint32_t> fill(n);
    if (n) CK(cudaMemcpyAsync(fill.data(), c.csrFill.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    for (uint64_t i = 0; i < n; i++)
        if (fill[i] != deg[i]) {
            set_error("internal: neighbour-table row %llu holds %u of %u values", (unsigned long long)i, fill[i],
                      deg[i]);
            return SJ_ERR_INTERNAL;
        }
    return SJ_OK;
}

void sj_free(void *p) { free(p); }

sj_status sj_get_stream(sj_ctx *ctx, void **stream)
{
    if (!ctx || !stream) return SJ_ERR_BAD_INPUT;
    *stream = (void *)as_ctx(ctx)->s;
    return SJ_OK;
}

sj_status sj_get_stats(sj_ctx *ctx, sj_stats *st)
{
    if (!ctx || !st) return SJ_ERR_BAD_INPUT;
    *st = as_ctx(ctx)->st;
    return SJ_OK;
}

uint32_t sj_mlp_num_params(void) { return SJ_MLP_NPARAM; }

sj_status sj_set_estimator_weights(sj_ctx *ctx, const float *w, uint32_t count)
{
    if (!ctx || !w || count != SJ_MLP_NPARAM) {
        set_error("estimator weights: expected %d floats", SJ_MLP_NPARAM);
        return SJ_ERR_BAD_INPUT;
    }
    Ctx &c = *as_ctx(ctx);
    c.mlpW.assign(w, w + count);
    return SJ_OK;
}

sj_status sj_load_estimator(sj_ctx *ctx, const char *path)
{
    if (!ctx || !path) return SJ_ERR_BAD_INPUT;
    FILE *f = fopen(path, "rb");
    if (!f) {
        set_error("cannot open %s", path);
        return SJ_ERR_IO;
    }
    std::vector<float> w(SJ_MLP_NPARAM);
    size_t r = fread(w.data(), sizeof(float), w.size(), f);
    fclose(f);
    if (r != w.size()) {
        set_error("%s: expected %d floats", path, SJ_MLP_NPARAM);
        return SJ_ERR_BAD_INPUT;
    }
    return sj_set_estimator_weights(ctx, w.data(), (uint32_t)w.size());
}

sj_status sj_cell_features(sj_ctx *ctx, float *feat, double *hits, double *calcs)
{
    if (!ctx) return SJ_ERR_BAD_INPUT;
    Ctx &c = *as_ctx(ctx);
    if (!c.indexed) {
        set_error("index not built");
        return SJ_ERR_STATE;
    }
    CKS(bind(c));
    if (c.nbrPattern < 0) CKS(build_neighbours(c, pattern_of_mode(c.p.search_mode)));
    if (feat)
        CK(cudaMemcpy(feat, c.feat.p, sizeof(float) * (size_t)c.nCells * SJ_NFEAT, cudaMemcpyDeviceToHost));
    const uint32_t nc = c.nCells;
    if (calcs) {
        std::vector<uint64_t> v(nc);
        CK(cudaMemcpy(v.data(), c.candFull.p, sizeof(uint64_t) * nc, cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < nc; i++) calcs[i] = (double)v[i];
    }
    if (hits) {
        if (!c.haveMeas) {
            set_error("no measured counts: run sj_degrees first");
            return SJ_ERR_STATE;
        }
        std::vector<unsigned long long> v(nc);
        CK(cudaMemcpy(v.data(), c.dCellHits.p, sizeof(unsigned long long) * nc, cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < nc; i++) hits[i] = (double)v[i];
    }
    return SJ_OK;
}

sj_status sj_cell_samples(sj_ctx *ctx, double *homeHits, double *homeEvals, double *nbrHits, double *nbrEvals)
{
    if (!ctx) return SJ_ERR_BAD_INPUT;
    Ctx &c = *as_ctx(ctx);
    if (!c.indexed) {
        set_error("index not built");
        return SJ_ERR_STATE;
    }
    if (c.p.scheduler != SJ_SCHED_SAMPLING) {
        set_error("sj_cell_samples needs the sampling scheduler");
        return SJ_ERR_STATE;
    }
    CKS(bind(c));
    int pattern;
    bool queue;
    CKS(prepare_join(c, pattern, queue));   // owned-neighbour lists and the sampling estimate
    if (!c.haveSamples) {
        set_error("internal: no sampling estimate");
        return SJ_ERR_INTERNAL;
    }
    const uint32_t nc = c.nCells;
    std::vector<unsigned long long> h(2 * (size_t)nc), e(2 * (size_t)nc);
    CK(cudaMemcpyAsync(h.data(), c.sHits.p, sizeof(unsigned long long) * h.size(), cudaMemcpyDeviceToHost, c.s));
    CK(cudaMemcpyAsync(e.data(), c.sCands.p, sizeof(unsigned long long) * e.size(), cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    for (uint32_t i = 0; i < nc; i++) {
        if (homeHits) homeHits[i] = (double)h[2 * (size_t)i];
        if (homeEvals) homeEvals[i] = (double)e[2 * (size_t)i];
        if (nbrHits) nbrHits[i] = (double)h[2 * (size_t)i + 1];
        if (nbrEvals) nbrEvals[i] = (double)e[2 * (size_t)i + 1];
    }
    return SJ_OK;
}

static sj_status mlp_common(int device, uint32_t m, const float *x, const float *y, DevBuf<float> &dx,
                            DevBuf<float> &dy, cudaStream_t s)
{
    CK(cudaSetDevice(device));
    CK(dx.ensure((size_t)m * SJ_NFEAT));
    CK(cudaMemcpyAsync(dx.p, x, sizeof(float) * (size_t)m * SJ_NFEAT, cudaMemcpyHostToDevice, s));
    if (y) {
        CK(dy.ensure((size_t)m * SJ_NOUT));
        CK(cudaMemcpyAsync(dy.p, y, sizeof(float) * (size_t)m * SJ_NOUT, cudaMemcpyHostToDevice, s));
    }
    return SJ_OK;
}

sj_status sj_mlp_loss_grad(const float *x, const float *y, uint32_t m, const float *w, float *loss, float *grad,
                           int device)
{
    if (!x || !y || !w || !grad || m == 0) return SJ_ERR_BAD_INPUT;
    DevBuf<float> dx, dy, dw, dg, dl;
    cudaStream_t s = 0;
    CKS(mlp_common(device, m, x, y, dx, dy, s));
    CK(dw.ensure(SJ_MLP_NPARAM));
    CK(dg.ensure(SJ_MLP_NPARAM));
    CK(dl.ensure(1));
    CK(cudaMemcpy(dw.p, w, sizeof(float) * SJ_MLP_NPARAM, cudaMemcpyHostToDevice));
    CK(sj_launch_mlp_grad(dx.p, dy.p, m, dw.p, dg.p, dl.p, s));
    CK(cudaMemcpy(grad, dg.p, sizeof(float) * SJ_MLP_NPARAM, cudaMemcpyDeviceToHost));
    float l;
    CK(cudaMemcpy(&l, dl.p, sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) *loss = l;
    return SJ_OK;
}

sj_status sj_mlp_forward(const float *x, uint32_t m, const float *w, float *out, int device)
{
    if (!x || !w || !out || m == 0) return SJ_ERR_BAD_INPUT;
    DevBuf<float> dx, dy, dw, dout;
    cudaStream_t s = 0;
    CKS(mlp_common(device, m, x, nullptr, dx, dy, s));
    CK(dw.ensure(SJ_MLP_NPARAM));
    CK(dout.ensure((size_t)m * SJ_NOUT));
    CK(cudaMemcpy(dw.p, w, sizeof(float) * SJ_MLP_NPARAM, cudaMemcpyHostToDevice));
    CK(sj_launch_mlp_infer(dx.p, m, dw.p, dout.p, s));
    CK(cudaMemcpy(out, dout.p, sizeof(float) * (size_t)m * SJ_NOUT, cudaMemcpyDeviceToHost));
    return SJ_OK;
}

sj_status sj_mlp_train(const float *x, const float *y, uint32_t m, float *w, int steps, float lr, uint32_t batch,
                       uint64_t seed, float *final_loss, int device)
{
    if (!x || !y || !w || m == 0 || steps < 1 || batch == 0) return SJ_ERR_BAD_INPUT;
    if (batch > m) batch = m;
    DevBuf<float> dx, dy, dw, dg, dm, dv, dl, bx, by;
    cudaStream_t s = 0;
    CKS(mlp_common(device, m, x, y, dx, dy, s));
    CK(dw.ensure(SJ_MLP_NPARAM));
    CK(dg.ensure(SJ_MLP_NPARAM));
    CK(dm.ensure(SJ_MLP_NPARAM));
    CK(dv.ensure(SJ_MLP_NPARAM));
    CK(dl.ensure(1));
    CK(bx.ensure((size_t)batch * SJ_NFEAT));
    CK(by.ensure((size_t)batch * SJ_NOUT));
    CK(cudaMemcpy(dw.p, w, sizeof(float) * SJ_MLP_NPARAM, cudaMemcpyHostToDevice));
    CK(cudaMemset(dm.p, 0, sizeof(float) * SJ_MLP_NPARAM));
    CK(cudaMemset(dv.p, 0, sizeof(float) * SJ_MLP_NPARAM));
    // minibatches: contiguous windows of a host-side shuffled copy
    std::vector<uint32_t> perm(m);
    std::iota(perm.begin(), perm.end(), 0u);
    uint64_t st = seed ? seed : 0x9e3779b97f4a7c15ULL;
    auto rnd = [&st]() {
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        return st;
    };
    for (uint32_t i = m - 1; i > 0; i--) std::swap(perm[i], perm[rnd() % (i + 1)]);
    std::vector<float> sx((size_t)m * SJ_NFEAT), sy((size_t)m * SJ_NOUT);
    for (uint32_t i = 0; i < m; i++) {
        memcpy(&sx[(size_t)i * SJ_NFEAT], &x[(size_t)perm[i] * SJ_NFEAT], sizeof(float) * SJ_NFEAT);
        memcpy(&sy[(size_t)i * SJ_NOUT], &y[(size_t)perm[i] * SJ_NOUT], sizeof(float) * SJ_NOUT);
    }
    CK(cudaMemcpy(dx.p, sx.data(), sizeof(float) * sx.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dy.p, sy.data(), sizeof(float) * sy.size(), cudaMemcpyHostToDevice));
    uint32_t nbat = m / batch;
    for (int step = 1; step <= steps; step++) {
        uint32_t b = (uint32_t)((step - 1) % nbat);
        const float *px = dx.p + (size_t)b * batch * SJ_NFEAT;
        const float *py = dy.p + (size_t)b * batch * SJ_NOUT;
        CK(sj_launch_mlp_train_step(px, py, batch, dw.p, dg.p, dm.p, dv.p, step, lr, dl.p, s));
    }
    CK(sj_launch_mlp_grad(dx.p, dy.p, m, dw.p, dg.p, dl.p, s));
    float l;
    CK(cudaMemcpy(&l, dl.p, sizeof(float), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(w, dw.p, sizeof(float) * SJ_MLP_NPARAM, cudaMemcpyDeviceToHost));
    if (final_loss) *final_loss = l;
    return SJ_OK;
}

const char *sj_status_string(sj_status s)
{
    switch (s) {
    case SJ_OK: return "ok";
    case SJ_ERR_OOM: return "out of memory";
    case SJ_OVERFLOW_RETRIED: return "overflow retried";
    case SJ_ERR_BAD_INPUT: return "bad input";
    case SJ_ERR_CUDA: return "CUDA error";
    case SJ_ERR_TIMEOUT: return "timeout";
    case SJ_ERR_STATE: return "call out of order";
    case SJ_ERR_IO: return "I/O error";
    case SJ_ERR_ABORTED: return "aborted by consumer";
    case SJ_ERR_INTERNAL: return "internal error";
    }
    return "unknown";
}

const char *sj_last_error(void) { return g_lastError.c_str(); }

uint64_t sj_kernel_launch_count(void) { return sj_launch_total(); }

const char *sj_version(void) { return "sj-b200 0.1 (sm_100a)"; }

}  // extern "C"
