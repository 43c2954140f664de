// Work units of the join, built on the device: per-cell workload, its
// ordering, the task list, the record offsets and the batch plan.
//
// The reference computes per-cell candidate counts on the GPU
// (sortByWorkLoad / sortByWorkLoadLidUnicomp, kernel.cu:33-250), copies them to
// the host, sorts them there with std::sort and gathers the points in that
// order (GPU.cu:1680-1728).  Here every step stays on the device:
//
//   1. per cell (one warp): the candidate stream of each segment group (home
//      cell + owned neighbours, at most SJ_MAX_SEG segments per group), the
//      query tiles, the stream chunk of every tile from the predicted hit rate
//      (or from the mode-8 split), hence the cell's task count, evaluations
//      and predicted pairs, and a cost key (heaviest first);
//   2. the cost order: the engine's stable LSD radix sort on the keys;
//   3. work items = (cell, segment group, query tile) in that order; per item
//      its chunk count; exclusive scans give every item's first task;
//   4. one thread per item writes its tasks and their predicted pairs;
//   5. per task the sizes of its count-pass records and emission units; their
//      exclusive prefix sums are the record offsets the kernels index by;
//   6. the batch plan: from every task s the end of a batch starting at s
//      (binary searches over the prefix sums: predicted pairs within the
//      capacity, hit-mask words within their limit), then one thread follows
//      those ends from task 0 -- the greedy plan, exactly.
#include "sj_internal.h"

namespace {

constexpr uint32_t FULL = 0xffffffffu;

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

__device__ __forceinline__ double warp_sum_f64(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// Query points of a cell that get tasks: all of them, or for the sampling
// estimator floor(occ * rate) plus one more with probability equal to the
// fraction (a per-cell hash decides), so about rate * n points in all and
// every heavy cell sampled in proportion to its size.
__device__ __forceinline__ uint32_t queries_of(const sj_taskgen &g, uint32_t c, uint32_t occ)
{
    if (g.sampleRate <= 0.0f) return occ;
    const double want = (double)occ * (double)g.sampleRate;
    uint32_t q = (uint32_t)want;
    const double frac = want - (double)q;
    uint32_t h = c * 0x9e3779b1u;
    h ^= h >> 15;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    if ((double)(h >> 8) * (1.0 / 16777216.0) < frac) q++;
    return q < occ ? q : occ;
}

// Candidate evaluations of stream positions [s0, s1) of a symmetric home
// segment for query indices 0..q-1 (only candidates at or after the query).
__device__ __forceinline__ uint64_t diag_evals(uint64_t s0, uint64_t s1, uint64_t q)
{
    if (s1 <= s0) return 0;
    uint64_t e = (q < s0 ? q : s0) * (s1 - s0);
    const uint64_t a = s0, b = q < s1 ? q : s1;
    if (b > a) e += (b - a) * s1 - (a + b - 1) * (b - a) / 2;
    return e;
}

// Stream chunk (positions per task) of a tile of qc queries over a stream of
// L positions.  policy 0: cost-proportional, the tile's predicted pairs per
// task near pairsPerTask; 1: fixed 65536; 2: `workers` tasks share the
// stream (mode 8).  Never more positions than keep a task's worst case (every
// evaluation a hit, both directions when symmetric) inside one batch.
__device__ __forceinline__ uint32_t chunk_len(const sj_taskgen &g, float rate, uint32_t qc, uint32_t L, int workers)
{
    uint64_t s;
    if (g.policy == 2 && workers > 0) {
        s = ((uint64_t)L + workers - 1) / workers;
        s = (s + 31) / 32 * 32;
        if (s > 65536) s = 65536;
    } else if (g.policy == 1) {
        s = 65536;
    } else {
        const double perEval = fmax((double)rate, 1e-6) * (g.sym ? 2.0 : 1.0);
        double chunk = g.pairsPerTask / (perEval * (double)qc);
        // a sparse stretch (few pairs per evaluation) is also cut by its
        // evaluations, so that no task runs much longer than the others and
        // a batch's last tasks leave little of the device idle
        if (g.evalsPerTask > 0.0) chunk = fmin(chunk, g.evalsPerTask / (double)qc);
        s = (uint64_t)fmin(65536.0, fmax(256.0, chunk));
    }
    const uint64_t worst = g.cap / ((g.sym ? 2ULL : 1ULL) * (uint64_t)qc);
    if (s > worst) s = worst;
    s = (s / 32) * 32;
    if (s < 32) s = 32;
    return (uint32_t)s;
}

struct TileWork {
    uint32_t qBegin, qc, L, homeLen, sc, nChunks;
    uint64_t evHome, evOther;   // evaluations against the home segment / the owned neighbours
};

// Predicted hits per evaluation of cell c: [0] against its own points, [1]
// against its neighbours' (both 0 without estimates).
__device__ __forceinline__ float2 rates_of(const sj_taskgen &g, uint32_t c)
{
    return g.rate ? make_float2(g.rate[2 * c], g.rate[2 * c + 1]) : make_float2(0.0f, 0.0f);
}

// Predicted pairs of evH home and evO neighbour evaluations with `diag` of
// the home ones a query against itself: a symmetric traversal emits a hit
// in both directions, a self pair once.
__device__ __forceinline__ double pairs_of(const sj_taskgen &g, float2 r, uint64_t evH, double evO, uint64_t diag)
{
    const double hits = (double)evH * (double)r.x + evO * (double)r.y;
    return g.sym ? fmax(0.0, 2.0 * hits - (double)diag) : hits;
}

// Weighted prefix of cell c's owned-neighbour stream at position x (0 at the
// first neighbour, cellW at the end): the entries' weighted prefix plus the
// weight of the part of x's own segment before x.
__device__ __forceinline__ double weighted_prefix(const sj_taskgen &g, uint32_t c, uint32_t x)
{
    uint32_t lo = g.nbrStart[c], hi = g.nbrStart[c + 1];
    if (lo == hi) return 0.0;
    // the last entry whose prefix is <= x
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (g.nbrPre[mid] <= x) lo = mid; else hi = mid;
    }
    const uint32_t b = g.nbrCell[lo];
    const uint32_t len = g.cellStart[b + 1] - g.cellStart[b];
    const uint32_t in = min(x - g.nbrPre[lo], len);
    return g.nbrPreW[lo] + (double)in * (double)g.nbrWt[lo];
}

// Neighbour evaluations of a task, as the mean-rate equivalent: with the
// spread, qc x (its stream's weighted length) x (the cell's mean weight)^-1,
// so that the cell's tasks share its predicted neighbour hits in proportion to
// the uniform-density hits of the segments they cover; otherwise qc x length.
// [n0, n1): the task's positions in its group's neighbour stream.
__device__ __forceinline__ double neighbour_evals(const sj_taskgen &g, uint32_t c, uint32_t grp, uint32_t qc,
                                                  uint32_t n0, uint32_t n1)
{
    if (n1 <= n0) return 0.0;
    if (!g.spread || g.cellW[c] <= 0.0) return (double)qc * (double)(n1 - n0);
    const uint32_t e0 = g.nbrStart[c], e1 = g.nbrStart[c + 1];
    const uint32_t eg = e0 + (grp == 0 ? 0u : grp * SJ_MAX_SEG - 1u);   // the group's first neighbour entry
    const uint32_t base = g.nbrPre[eg];
    const uint32_t bl = g.nbrCell[e1 - 1];
    const double total = (double)g.nbrPre[e1 - 1] + (double)(g.cellStart[bl + 1] - g.cellStart[bl]);
    const double wl = weighted_prefix(g, c, base + n1) - weighted_prefix(g, c, base + n0);
    return (double)qc * wl * total / g.cellW[c];
}

// Query tile `tile` of cell c against segment group grp (non-home length S).
// Sampling tasks (policy 1) chunk the home segment and the neighbours
// separately, so that their hits are measured apart.
__device__ __forceinline__ TileWork tile_work(const sj_taskgen &g, uint32_t c, uint32_t grp, uint32_t tile, uint32_t S,
                                              int workers)
{
    TileWork w;
    const uint32_t aStart = g.cellStart[c], occ = g.cellStart[c + 1] - aStart;
    const uint32_t nq = queries_of(g, c, occ);
    const uint32_t q0 = tile * g.tile;
    w.qBegin = aStart + q0;
    w.qc = min(g.tile, nq - q0);
    w.homeLen = grp == 0 ? (g.sym ? occ - q0 : occ) : 0u;
    w.L = S + w.homeLen;
    const uint64_t qc = w.qc;
    w.evHome = g.sym ? diag_evals(0, w.homeLen, qc) : qc * (uint64_t)w.homeLen;
    w.evOther = qc * (uint64_t)S;
    const float2 r = rates_of(g, c);
    const double ev = (double)(w.evHome + w.evOther);
    const float rate = ev > 0 ? (float)(((double)w.evHome * r.x + (double)w.evOther * r.y) / ev) : 0.0f;
    w.sc = chunk_len(g, rate, w.qc, w.L, workers);
    if (g.policy == 1)
        w.nChunks = (w.homeLen + w.sc - 1) / w.sc + (S + w.sc - 1) / w.sc;
    else
        w.nChunks = (w.L + w.sc - 1) / w.sc;
    return w;
}

// Stream positions of chunk j of a tile (see tile_work).
__device__ __forceinline__ uint2 chunk_range(const sj_taskgen &g, const TileWork &w, uint32_t j)
{
    if (g.policy == 1) {
        const uint32_t nh = (w.homeLen + w.sc - 1) / w.sc;
        if (j < nh) return make_uint2(j * w.sc, min(w.homeLen, (j + 1) * w.sc));
        const uint32_t s0 = w.homeLen + (j - nh) * w.sc;
        return make_uint2(s0, min(w.L, s0 + w.sc));
    }
    return make_uint2(j * w.sc, min(w.L, (j + 1) * w.sc));
}

__device__ __forceinline__ uint32_t n_groups(const sj_taskgen &g, uint32_t c)
{
    const uint32_t nSegAll = 1 + (g.nbrStart[c + 1] - g.nbrStart[c]);
    return (nSegAll + SJ_MAX_SEG - 1) / SJ_MAX_SEG;
}

__device__ __forceinline__ uint32_t n_tiles(const sj_taskgen &g, uint32_t c)
{
    const uint32_t occ = g.cellStart[c + 1] - g.cellStart[c];
    return (queries_of(g, c, occ) + g.tile - 1) / g.tile;
}

__global__ void __launch_bounds__(256) k_tg_groups(sj_taskgen g, uint32_t *cnt)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < g.nCells) cnt[c] = n_groups(g, c);
}

// One warp per position (cell order[pos], or pos itself): task count,
// evaluations, predicted pairs and the cost key of the cell; also the
// non-home stream length of each of its segment groups.
__global__ void __launch_bounds__(256) k_tg_cells(sj_taskgen g, const uint32_t *__restrict__ order,
                                                  const uint8_t *__restrict__ workersAt, uint32_t *__restrict__ posCnt,
                                                  unsigned long long *__restrict__ posEv,
                                                  unsigned long long *__restrict__ costKey,
                                                  unsigned long long *__restrict__ totals)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t pos = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (pos >= g.nCells) return;
    const uint32_t c = order ? order[pos] : pos;
    const int workers = workersAt ? (int)workersAt[pos] : 0;
    const uint32_t nb0 = g.nbrStart[c];
    const uint32_t nSegAll = 1 + (g.nbrStart[c + 1] - nb0);
    const uint32_t G = (nSegAll + SJ_MAX_SEG - 1) / SJ_MAX_SEG;
    const uint32_t T = n_tiles(g, c);
    const float2 r = rates_of(g, c);
    uint64_t cnt = 0, ev = 0;
    double pred = 0.0;
    for (uint32_t grp = 0; grp < G; grp++) {
        const uint32_t s0 = grp * SJ_MAX_SEG, s1 = min(nSegAll, s0 + SJ_MAX_SEG);
        uint64_t S = 0;
        for (uint32_t s = s0 + lane; s < s1; s += 32) {
            if (s == 0) continue;   // the home segment's length depends on the tile
            const uint32_t b = g.nbrCell[nb0 + s - 1];
            S += g.cellStart[b + 1] - g.cellStart[b];
        }
        S = warp_sum_u64(S);
        if (lane == 0) g.groupLen[g.groupBase[c] + grp] = (uint32_t)S;
        for (uint32_t t = lane; t < T; t += 32) {
            const TileWork w = tile_work(g, c, grp, t, (uint32_t)S, workers);
            cnt += w.nChunks;
            ev += w.evHome + w.evOther;
            pred += pairs_of(g, r, w.evHome, w.evOther, w.homeLen ? w.qc : 0u);
        }
    }
    cnt = warp_sum_u64(cnt);
    ev = warp_sum_u64(ev);
    pred = warp_sum_f64(pred);
    if (lane == 0) {
        posCnt[pos] = (uint32_t)min(cnt, (uint64_t)FULL);
        if (posEv) posEv[pos] = ev;
        if (costKey) {
            // mean predicted task cost: evaluations plus a write cost per pair
            const double cost = cnt ? ((double)ev + 4.0 * pred) / (double)cnt : 0.0;
            costKey[pos] = ~(unsigned long long)__double_as_longlong(cost);   // cost >= 0: descending
        }
        atomicAdd(&totals[0], (unsigned long long)cnt);
        atomicAdd(&totals[1], (unsigned long long)ev);
    }
}

// One warp per cell: exclusive prefixes over its owned-neighbour entries of the
// occupancy and of occupancy x offset-class weight (see sj_nbr_spread).
__global__ void __launch_bounds__(256) k_nbr_spread(const uint32_t *__restrict__ cellStart,
                                                    const uint32_t *__restrict__ cellCoord,
                                                    const uint32_t *__restrict__ nbrStart,
                                                    const uint32_t *__restrict__ nbrCell, uint32_t nCells,
                                                    sj_grid_dev gd, uint32_t *__restrict__ nbrPre,
                                                    double *__restrict__ nbrPreW, float *__restrict__ nbrWt,
                                                    double *__restrict__ cellW)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= nCells) return;
    const int k = gd.k;
    const uint32_t e0 = nbrStart[c], e1 = nbrStart[c + 1];
    uint32_t carryP = 0;
    double carryW = 0.0;
    for (uint32_t base = e0; base < e1; base += 32) {
        const uint32_t e = base + lane;
        uint32_t occ = 0;
        float w = 0.0f;
        if (e < e1) {
            const uint32_t b = nbrCell[e];
            occ = cellStart[b + 1] - cellStart[b];
            int m = 0;
            for (int j = 0; j < k; j++) m += cellCoord[(uint64_t)c * k + j] != cellCoord[(uint64_t)b * k + j];
            w = gd.offW[m];
        }
        const double wv = (double)occ * (double)w;
        uint32_t ip = occ;
        double iw = wv;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t yp = __shfl_up_sync(FULL, ip, o);
            const double yw = __shfl_up_sync(FULL, iw, o);
            if (lane >= (uint32_t)o) {
                ip += yp;
                iw += yw;
            }
        }
        if (e < e1) {
            nbrPre[e] = carryP + ip - occ;
            nbrPreW[e] = carryW + iw - wv;
            nbrWt[e] = w;
        }
        carryP += __shfl_sync(FULL, ip, 31);
        carryW += __shfl_sync(FULL, iw, 31);
    }
    if (lane == 0) cellW[c] = carryW;
}

__global__ void __launch_bounds__(256) k_iota(uint32_t *v, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

// Mode 8 (the reference's dynamic threads per point, kernel.cu:2072-2188 with
// NB_THREAD_THIRD1..3 = 16, 8, 2 of params.h): the first third of the work in
// cost order splits every query tile's stream over 16 tasks, the second over
// 8, the rest over 2.  evExcl: exclusive prefix of the evaluations in order.
__global__ void __launch_bounds__(256) k_tg_thirds(const unsigned long long *__restrict__ evExcl, uint32_t n,
                                                   uint8_t *__restrict__ workers)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long total = evExcl[n];
    const double f = total ? (double)evExcl[i] / (double)total : 0.0;
    workers[i] = f < 1.0 / 3.0 ? 16 : (f < 2.0 / 3.0 ? 8 : 2);
}

// Work items of a position: segment groups x query tiles.
__global__ void __launch_bounds__(256) k_tg_item_counts(sj_taskgen g, const uint32_t *__restrict__ order,
                                                        uint32_t *__restrict__ items)
{
    const uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x;
    if (pos >= g.nCells) return;
    const uint32_t c = order[pos];
    items[pos] = n_groups(g, c) * n_tiles(g, c);
}

struct Item {
    uint32_t pos, c, grp, tile;
};

__device__ __forceinline__ Item find_item(const sj_taskgen &g, const uint32_t *__restrict__ order,
                                          const uint32_t *__restrict__ itemStart, uint32_t j)
{
    // the last position whose first item is <= j
    uint32_t lo = 0, hi = g.nCells;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (itemStart[mid] <= j) lo = mid; else hi = mid;
    }
    Item it;
    it.pos = lo;
    it.c = order[lo];
    const uint32_t T = n_tiles(g, it.c);
    const uint32_t local = j - itemStart[lo];
    it.grp = local / T;
    it.tile = local - it.grp * T;
    return it;
}

__global__ void __launch_bounds__(256) k_tg_item_tasks(sj_taskgen g, const uint32_t *__restrict__ order,
                                                       const uint8_t *__restrict__ workersAt,
                                                       const uint32_t *__restrict__ itemStart, uint32_t nItems,
                                                       uint32_t *__restrict__ itemTasks)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nItems) return;
    const Item it = find_item(g, order, itemStart, j);
    const uint32_t S = g.groupLen[g.groupBase[it.c] + it.grp];
    const TileWork w = tile_work(g, it.c, it.grp, it.tile, S, workersAt ? (int)workersAt[it.pos] : 0);
    itemTasks[j] = w.nChunks;
}

// Writes every item's tasks (in item order, chunks ascending) and their
// predicted pairs.
__global__ void __launch_bounds__(256) k_tg_item_write(sj_taskgen g, const uint32_t *__restrict__ order,
                                                       const uint8_t *__restrict__ workersAt,
                                                       const uint32_t *__restrict__ itemStart, uint32_t nItems,
                                                       const uint32_t *__restrict__ itemTaskStart,
                                                       sj_task *__restrict__ tasks, float *__restrict__ pred)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nItems) return;
    const Item it = find_item(g, order, itemStart, j);
    const uint32_t S = g.groupLen[g.groupBase[it.c] + it.grp];
    const TileWork w = tile_work(g, it.c, it.grp, it.tile, S, workersAt ? (int)workersAt[it.pos] : 0);
    const uint32_t nSegAll = 1 + (g.nbrStart[it.c + 1] - g.nbrStart[it.c]);
    const uint32_t segBase = it.grp * SJ_MAX_SEG;
    const float2 r = rates_of(g, it.c);
    uint32_t t = itemTaskStart[j];
    for (uint32_t ch = 0; ch < w.nChunks; ch++, t++) {
        const uint2 sr = chunk_range(g, w, ch);
        const uint32_t s0 = sr.x, s1 = sr.y;
        // evaluations against the home segment (positions < homeLen) and the rest
        const uint32_t h1 = min(s1, w.homeLen);
        uint64_t evH = 0, diag = 0;
        if (s0 < h1) {
            evH = g.sym ? diag_evals(s0, h1, w.qc) : (uint64_t)w.qc * (h1 - s0);
            diag = s0 < w.qc ? min(h1, w.qc) - s0 : 0u;   // queries whose own position is in the chunk
        }
        const double evO = neighbour_evals(g, it.c, it.grp, w.qc, max(s0, h1) - w.homeLen, s1 - w.homeLen);
        sj_task k;
        k.cell = it.c;
        k.qBegin = w.qBegin;
        k.qCount = w.qc;
        k.segBase = segBase;
        k.segCount = min((uint32_t)SJ_MAX_SEG, nSegAll - segBase);
        k.sBegin = s0;
        k.sEnd = s1;
        k.flags = (g.sym ? SJ_TASK_SYM : 0u) | (it.grp == 0 ? SJ_TASK_HOME : 0u);
        tasks[t] = k;
        pred[t] = (float)pairs_of(g, r, evH, evO, diag);
    }
}

// Shard `idx` of `cnt` keeps every cnt-th task of the ordered list.
__global__ void __launch_bounds__(256) k_tg_shard(const sj_task *__restrict__ in, const float *__restrict__ predIn,
                                                  uint32_t nOut, uint32_t idx, uint32_t cnt,
                                                  sj_task *__restrict__ out, float *__restrict__ predOut)
{
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nOut) return;
    const uint64_t i = (uint64_t)w * cnt + idx;
    out[w] = in[i];
    predOut[w] = predIn[i];
}

// ------------------------------------------------------ record offsets ----
constexpr int NC = 7;           // row masks, column masks, row offsets, candidate records, units,
                                // planned pairs (rounded up, x (1 + alpha)), predicted pairs (rounded)
constexpr int OT = 256;         // threads per offsets block
constexpr int OI = 8;           // tasks per thread
constexpr int OTILE = OT * OI;

__device__ __forceinline__ void task_sizes(const sj_task &t, float pred, double alpha1, uint64_t (&v)[NC])
{
    const uint32_t len = t.sEnd - t.sBegin;
    const bool sym = (t.flags & SJ_TASK_SYM) != 0;
    const uint64_t blocks = ((uint64_t)len + 31) / 32;
    const uint64_t groups = ((uint64_t)t.qCount + 31) / 32;
    v[0] = blocks * t.qCount;
    v[1] = sym ? blocks * groups * 32 : 0;
    v[2] = t.qCount;
    v[3] = len;
    v[4] = sj_task_units(t.qCount, len, sym);
    v[5] = (uint64_t)ceil((double)pred * alpha1);
    v[6] = (uint64_t)llrint((double)pred);
}

__global__ void __launch_bounds__(OT) k_off_reduce(const sj_task *__restrict__ tasks, const float *__restrict__ pred,
                                                   uint32_t nt, double alpha1, unsigned long long *__restrict__ sums)
{
    uint64_t acc[NC] = {0, 0, 0, 0, 0, 0, 0};
    const uint64_t base = (uint64_t)blockIdx.x * OTILE;
    for (int i = 0; i < OI; i++) {
        const uint64_t t = base + (uint64_t)i * OT + threadIdx.x;
        if (t < nt) {
            uint64_t v[NC];
            task_sizes(tasks[t], pred[t], alpha1, v);
#pragma unroll
            for (int k = 0; k < NC; k++) acc[k] += v[k];
        }
    }
    __shared__ unsigned long long red[OT / 32][NC];
#pragma unroll
    for (int k = 0; k < NC; k++) {
        const uint64_t s = warp_sum_u64(acc[k]);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][k] = s;
    }
    __syncthreads();
    if (threadIdx.x < NC) {
        unsigned long long s = 0;
        for (int w = 0; w < OT / 32; w++) s += red[w][threadIdx.x];
        sums[(uint64_t)blockIdx.x * NC + threadIdx.x] = s;
    }
}

// Exclusive scan of the per-block sums, one component per warp (in place).
__global__ void __launch_bounds__(32 * NC) k_off_scan_blocks(unsigned long long *sums, uint32_t nb)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t k = threadIdx.x >> 5;
    unsigned long long carry = 0;
    for (uint32_t b0 = 0; b0 < nb; b0 += 32) {
        const uint32_t b = b0 + lane;
        const unsigned long long v = b < nb ? sums[(uint64_t)b * NC + k] : 0ULL;
        unsigned long long x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(FULL, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (b < nb) sums[(uint64_t)b * NC + k] = carry + x - v;
        carry += __shfl_sync(FULL, x, 31);
    }
}

struct OffOut {
    unsigned long long *p[NC];
};

__global__ void __launch_bounds__(OT) k_off_write(const sj_task *__restrict__ tasks, const float *__restrict__ pred,
                                                  uint32_t nt, double alpha1,
                                                  const unsigned long long *__restrict__ blockBase, OffOut out)
{
    // thread th handles tasks base + th*OI .. + OI-1 (consecutive)
    const uint64_t base = (uint64_t)blockIdx.x * OTILE + (uint64_t)threadIdx.x * OI;
    uint64_t v[OI][NC];
    uint64_t tot[NC] = {0, 0, 0, 0, 0, 0, 0};
    for (int i = 0; i < OI; i++) {
        const uint64_t t = base + i;
        if (t < nt) {
            task_sizes(tasks[t], pred[t], alpha1, v[i]);
        } else {
#pragma unroll
            for (int k = 0; k < NC; k++) v[i][k] = 0;
        }
#pragma unroll
        for (int k = 0; k < NC; k++) tot[k] += v[i][k];
    }
    __shared__ unsigned long long wsum[OT / 32][NC];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint64_t excl[NC];
#pragma unroll
    for (int k = 0; k < NC; k++) {
        unsigned long long x = tot[k];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(FULL, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        excl[k] = x - tot[k];
        if (lane == 31) wsum[warp][k] = x;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NC; k++) {
        unsigned long long w = blockBase[(uint64_t)blockIdx.x * NC + k];
        for (uint32_t j = 0; j < warp; j++) w += wsum[j][k];
        excl[k] += w;
    }
    for (int i = 0; i < OI; i++) {
        const uint64_t t = base + i;
        if (t < nt) {
#pragma unroll
            for (int k = 0; k < NC; k++) {
                out.p[k][t] = excl[k];
                excl[k] += v[i][k];
            }
            if (t == nt - 1) {
#pragma unroll
                for (int k = 0; k < NC; k++) out.p[k][nt] = excl[k];
            }
        }
    }
}

// ------------------------------------------------------------ batch plan --
// Largest e in [s+1, nt] with A[e] - A[s] <= lim (s+1 when even one task exceeds).
__device__ __forceinline__ uint32_t reach(const unsigned long long *__restrict__ A, uint32_t s, uint32_t nt,
                                          unsigned long long lim)
{
    const unsigned long long top = A[s] + lim;
    uint32_t lo = s + 1, hi = nt + 1;   // first index in [s+1, nt+1) with A > top
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (A[mid] <= top) lo = mid + 1; else hi = mid;
    }
    return lo - 1 > s ? lo - 1 : s + 1;
}

__global__ void __launch_bounds__(256) k_plan_next(const unsigned long long *__restrict__ planned,
                                                   const unsigned long long *__restrict__ maskOff,
                                                   const unsigned long long *__restrict__ colOff,
                                                   const unsigned long long *__restrict__ unitOff, uint32_t nt,
                                                   unsigned long long cap, unsigned long long maskLim,
                                                   uint32_t *__restrict__ next)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nt) return;
    uint32_t e = reach(planned, s, nt, cap);
    e = min(e, reach(maskOff, s, nt, maskLim));
    e = min(e, reach(colOff, s, nt, maskLim));
    e = min(e, reach(unitOff, s, nt, 0xffffffffULL));
    next[s] = max(e, s + 1);
}

// Follows the batch ends from task 0: batch b is [start[b], start[b+1]).
__global__ void k_plan_chain(const uint32_t *__restrict__ next, uint32_t nt, uint32_t *__restrict__ start,
                             uint32_t *__restrict__ nBatches)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t s = 0, b = 0;
    while (s < nt) {
        start[b++] = s;
        s = next[s];
    }
    start[b] = nt;
    *nBatches = b;
}

// Per batch: predicted pairs and the sizes of its records.
__global__ void __launch_bounds__(256) k_plan_stats(const uint32_t *__restrict__ start, uint32_t nb, OffOut off,
                                                    unsigned long long *__restrict__ stats)
{
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const uint32_t t0 = start[b], t1 = start[b + 1];
    // [0] predicted pairs, [1] row-mask words, [2] column-mask words, [3] row offsets, [4] candidate records
    stats[(uint64_t)b * 5 + 0] = off.p[6][t1] - off.p[6][t0];
    stats[(uint64_t)b * 5 + 1] = off.p[0][t1] - off.p[0][t0];
    stats[(uint64_t)b * 5 + 2] = off.p[1][t1] - off.p[1][t0];
    stats[(uint64_t)b * 5 + 3] = off.p[2][t1] - off.p[2][t0];
    stats[(uint64_t)b * 5 + 4] = off.p[3][t1] - off.p[3][t0];
}

// ------------------------------------------------------------ estimates --
// Learned estimator: per-cell hits per evaluation from the network's two
// outputs, log2(1 + hits of the cell's points among its own points) and
// log2(1 + hits among its owned neighbours' points): divided by the cell's
// occupancy squared and by its occupancy times the owned neighbours' total.
__global__ void __launch_bounds__(256) k_rates_mlp(const float *__restrict__ out, const uint32_t *__restrict__ cellStart,
                                                   const uint32_t *__restrict__ nbrStart,
                                                   const uint32_t *__restrict__ nbrCell, uint32_t nCells,
                                                   float *__restrict__ rate)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nCells) return;
    const double occ = (double)(cellStart[c + 1] - cellStart[c]);
    double nbr = 0.0;
    for (uint32_t i = nbrStart[c]; i < nbrStart[c + 1]; i++) {
        const uint32_t b = nbrCell[i];
        nbr += (double)(cellStart[b + 1] - cellStart[b]);
    }
    const double hHome = exp2((double)out[(uint64_t)c * SJ_NOUT]) - 1.0;
    const double hNbr = exp2((double)out[(uint64_t)c * SJ_NOUT + 1]) - 1.0;
    const double rH = occ > 0 ? hHome / (occ * occ) : 0.0;
    const double rN = occ > 0 && nbr > 0 ? hNbr / (occ * nbr) : 0.0;
    rate[2 * c] = (float)fmin(1.0, fmax(rH, 0.0));
    rate[2 * c + 1] = (float)fmin(1.0, fmax(rN, 0.0));
}

// Sampling estimator: hits and evaluations of the sampled queries, per cell
// and segment kind (its own points, its neighbours'), per occupancy class of
// the cell (floor(log2(occupancy)), 32 classes) and in total.  A sampling task
// is a home task when it covers home-segment positions only (they are chunked
// apart).  totals: [4 * b + 2 * kind + 0/1] class b's hits / evaluations,
// [128 + 2 * kind + 0/1] the totals.
constexpr int SAMPLE_BINS = 32;

__device__ __forceinline__ uint32_t occ_bin(const uint32_t *__restrict__ cellStart, uint32_t c)
{
    const uint32_t occ = cellStart[c + 1] - cellStart[c];
    return occ ? 31u - __clz(occ) : 0u;
}

__global__ void __launch_bounds__(256) k_sample_sums(const sj_task *__restrict__ tasks, uint32_t nt,
                                                     const uint32_t *__restrict__ taskHits,
                                                     const uint32_t *__restrict__ taskEvals,
                                                     const uint32_t *__restrict__ cellStart,
                                                     unsigned long long *__restrict__ cellHits,
                                                     unsigned long long *__restrict__ cellEvals,
                                                     unsigned long long *__restrict__ totals)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const sj_task k = tasks[t];
    const uint32_t c = k.cell;
    const uint32_t occ = cellStart[c + 1] - cellStart[c];
    const uint32_t kind = (k.segBase == 0 && k.sEnd <= occ) ? 0u : 1u;
    const uint32_t h = taskHits[t], e = taskEvals[t];
    const uint32_t b = occ_bin(cellStart, c);
    if (h) {
        atomicAdd(&cellHits[2 * c + kind], (unsigned long long)h);
        atomicAdd(&totals[4 * b + 2 * kind], (unsigned long long)h);
        atomicAdd(&totals[4 * SAMPLE_BINS + 2 * kind], (unsigned long long)h);
    }
    if (e) {
        atomicAdd(&cellEvals[2 * c + kind], (unsigned long long)e);
        atomicAdd(&totals[4 * b + 2 * kind + 1], (unsigned long long)e);
        atomicAdd(&totals[4 * SAMPLE_BINS + 2 * kind + 1], (unsigned long long)e);
    }
}

// A cell and segment kind without a sampled evaluation take the rate of the
// sampled cells of the cell's occupancy class, or the global rate.
__global__ void __launch_bounds__(256) k_sample_rates(const unsigned long long *__restrict__ cellHits,
                                                      const unsigned long long *__restrict__ cellEvals,
                                                      const unsigned long long *__restrict__ totals,
                                                      const uint32_t *__restrict__ cellStart, uint32_t nCells,
                                                      float *__restrict__ rate)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nCells) return;
    const uint32_t b = occ_bin(cellStart, c);
    for (int kind = 0; kind < 2; kind++) {
        float v;
        if (cellEvals[2 * c + kind]) {
            v = (float)((double)cellHits[2 * c + kind] / (double)cellEvals[2 * c + kind]);
        } else {
            const unsigned long long bh = totals[4 * b + 2 * kind], be = totals[4 * b + 2 * kind + 1];
            const unsigned long long gh = totals[4 * SAMPLE_BINS + 2 * kind], ge = totals[4 * SAMPLE_BINS + 2 * kind + 1];
            v = (float)(be ? (double)bh / (double)be : (ge ? (double)gh / (double)ge : 1.0));
        }
        rate[2 * c + kind] = v;
    }
}

// ------------------------------------------------------------ statistics --
// sums[0] evaluations, [1] FP32 borderline re-evaluations, [2] measured pairs;
// errSum: sum over tasks of |predicted - measured pairs|.
__global__ void __launch_bounds__(256) k_task_sums(const uint32_t *__restrict__ taskEvals,
                                                   const uint32_t *__restrict__ taskRefined,
                                                   const uint32_t *__restrict__ taskHits,
                                                   const float *__restrict__ pred, uint32_t nt,
                                                   unsigned long long *__restrict__ sums, double *__restrict__ errSum)
{
    uint64_t e = 0, r = 0, h = 0;
    double d = 0.0;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        e += taskEvals[t];
        r += taskRefined[t];
        if (taskHits) {
            h += taskHits[t];
            if (pred) d += fabs((double)pred[t] - (double)taskHits[t]);
        }
    }
    e = warp_sum_u64(e);
    r = warp_sum_u64(r);
    h = warp_sum_u64(h);
    d = warp_sum_f64(d);
    if ((threadIdx.x & 31) == 0) {
        if (e) atomicAdd(&sums[0], (unsigned long long)e);
        if (r) atomicAdd(&sums[1], (unsigned long long)r);
        if (h) atomicAdd(&sums[2], (unsigned long long)h);
        if (d != 0.0 && errSum) atomicAdd(errSum, d);
    }
}

// Per cell: the sum of its points' degrees (measured hits, full-stencil semantics).
__global__ void __launch_bounds__(256) k_cell_hits(const uint32_t *__restrict__ cellStart,
                                                   const uint32_t *__restrict__ ids, const uint32_t *__restrict__ deg,
                                                   uint32_t nCells, unsigned long long *__restrict__ hits)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (c >= nCells) return;
    uint64_t s = 0;
    for (uint32_t p = cellStart[c] + lane; p < cellStart[c + 1]; p += 32) s += deg[ids[p]];
    s = warp_sum_u64(s);
    if (lane == 0) hits[c] = s;
}

// ------------------------------------------------------------ u64 scan --
constexpr int S64T = 256, S64I = 8, S64TILE = S64T * S64I;

__global__ void __launch_bounds__(S64T) k_s64_reduce(const unsigned long long *__restrict__ in, uint64_t n,
                                                      unsigned long long *__restrict__ sums)
{
    uint64_t acc = 0;
    const uint64_t base = (uint64_t)blockIdx.x * S64TILE;
    for (int i = 0; i < S64I; i++) {
        const uint64_t j = base + (uint64_t)i * S64T + threadIdx.x;
        if (j < n) acc += in[j];
    }
    __shared__ unsigned long long red[S64T / 32];
    acc = warp_sum_u64(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < S64T / 32; w++) t += red[w];
        sums[blockIdx.x] = t;
    }
}

__global__ void k_s64_scan_blocks(unsigned long long *sums, uint32_t nb)
{
    const uint32_t lane = threadIdx.x & 31u;
    unsigned long long carry = 0;
    for (uint32_t b0 = 0; b0 < nb; b0 += 32) {
        const uint32_t b = b0 + lane;
        const unsigned long long v = b < nb ? sums[b] : 0ULL;
        unsigned long long x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(FULL, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (b < nb) sums[b] = carry + x - v;
        carry += __shfl_sync(FULL, x, 31);
    }
}

__global__ void __launch_bounds__(S64T) k_s64_write(const unsigned long long *__restrict__ in, uint64_t n,
                                                     const unsigned long long *__restrict__ blockBase,
                                                     unsigned long long *__restrict__ out)
{
    const uint64_t base = (uint64_t)blockIdx.x * S64TILE + (uint64_t)threadIdx.x * S64I;
    unsigned long long v[S64I];
    unsigned long long tot = 0;
    for (int i = 0; i < S64I; i++) {
        v[i] = base + i < n ? in[base + i] : 0ULL;
        tot += v[i];
    }
    __shared__ unsigned long long wsum[S64T / 32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    unsigned long long x = tot;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(FULL, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    unsigned long long run = blockBase[blockIdx.x] + x - tot;
    for (uint32_t j = 0; j < warp; j++) run += wsum[j];
    for (int i = 0; i < S64I; i++) {
        const uint64_t j = base + i;
        if (j < n) {
            out[j] = run;
            run += v[i];
            if (j == n - 1) out[n] = run;
        }
    }
}

inline unsigned blocks_for(uint64_t n, unsigned per) { return (unsigned)((n + per - 1) / per); }

}  // namespace

cudaError_t sj_nbr_spread(const uint32_t *cellStart, const uint32_t *cellCoord, const uint32_t *nbrStart,
                          const uint32_t *nbrCell, uint32_t nCells, const sj_grid_dev &g, uint32_t *nbrPre,
                          double *nbrPreW, float *nbrWt, double *cellW, cudaStream_t s)
{
    if (nCells == 0) return cudaSuccess;
    k_nbr_spread<<<blocks_for((uint64_t)nCells * 32, 256), 256, 0, s>>>(cellStart, cellCoord, nbrStart, nbrCell,
                                                                          nCells, g, nbrPre, nbrPreW, nbrWt, cellW);
    sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_tg_groups(const sj_taskgen &g, uint32_t *cnt, cudaStream_t s)
{
    if (g.nCells == 0) return cudaSuccess;
    k_tg_groups<<<blocks_for(g.nCells, 256), 256, 0, s>>>(g, cnt);
    sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_tg_cells(const sj_taskgen &g, const uint32_t *order, const uint8_t *workersAt, uint32_t *posCnt,
                        unsigned long long *posEv, unsigned long long *costKey, unsigned long long *totals,
                        cudaStream_t s)
{
    if (g.nCells == 0) return cudaSuccess;
    k_tg_cells<<<blocks_for((uint64_t)g.nCells * 32, 256), 256, 0, s>>>(g, order, workersAt, posCnt, posEv, costKey,
                                                                        totals);
    sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_iota_u32(uint32_t *v, uint32_t n, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    k_iota<<<blocks_for(n, 256), 256, 0, s>>>(v, n);
    sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_tg_thirds(const unsigned long long *evExcl, uint32_t n, uint8_t *workers, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    k_tg_thirds<<<blocks_for(n, 256), 256, 0, s>>>(evExcl, n, workers);
    sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_tg_item_counts(const sj_taskgen &g, const uint32_t *order, uint32_t *items, cudaStream_t s)
{
    if (g.nCells == 0) return cudaSuccess;
    k_tg_item_counts<<<blocks_for(g.nCells, 256), 256, 0, s>>>(g, order, items);
    sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_tg_item_tasks(const sj_taskgen &g, const uint32_t *order, const uint8_t *workersAt,
                             const uint32_t *itemStart, uint32_t nItems, uint32_t *itemTasks, cudaStream_t s)
{
    if (nItems == 0) return cudaSuccess;
    k_tg_item_tasks<<<blocks_for(nItems, 256), 256, 0, s>>>(g, order, workersAt, itemStart, nItems, itemTasks);
    sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_tg_item_write(const sj_taskgen &g, const uint32_t *order, const uint8_t *workersAt,
                             const uint32_t *itemStart, uint32_t nItems, const uint32_t *itemTaskStart,
                             sj_task *tasks, float *pred, cudaStream_t s)
{
    if (nItems == 0) return cudaSuccess;
    k_tg_item_write<<<blocks_for(nItems, 256), 256, 0, s>>>(g, order, workersAt, itemStart, nItems, itemTaskStart,
                                                            tasks, pred);
    sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_tg_shard(const sj_task *in, const float *predIn, uint32_t nOut, uint32_t idx, uint32_t cnt,
                        sj_task *out, float *predOut, cudaStream_t s)
{
    if (nOut == 0) return cudaSuccess;
    k_tg_shard<<<blocks_for(nOut, 256), 256, 0, s>>>(in, predIn, nOut, idx, cnt, out, predOut);
    sj_note_launch();
    return cudaGetLastError();
}

size_t sj_task_offsets_temp(uint32_t nt) { return (size_t)(blocks_for(nt ? nt : 1, OTILE)) * NC; }

cudaError_t sj_task_offsets(const sj_task *tasks, const float *pred, uint32_t nt, double alpha,
                            unsigned long long *temp, unsigned long long *const out[7], cudaStream_t s)
{
    OffOut o;
    for (int k = 0; k < NC; k++) o.p[k] = out[k];
    if (nt == 0) {
        for (int k = 0; k < NC; k++) {
            cudaError_t e = cudaMemsetAsync(out[k], 0, sizeof(unsigned long long), s);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    const unsigned nb = blocks_for(nt, OTILE);
    const double alpha1 = 1.0 + alpha;
    k_off_reduce<<<nb, OT, 0, s>>>(tasks, pred, nt, alpha1, temp);
    sj_note_launch();
    k_off_scan_blocks<<<1, 32 * NC, 0, s>>>(temp, nb);
    sj_note_launch();
    k_off_write<<<nb, OT, 0, s>>>(tasks, pred, nt, alpha1, temp, o);
    sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_plan_batches(unsigned long long *const off[7], uint32_t nt, unsigned long long cap,
                            unsigned long long maskLim, uint32_t *next, uint32_t *start, uint32_t *nBatches,
                            cudaStream_t s)
{
    if (nt == 0) return cudaMemsetAsync(nBatches, 0, sizeof(uint32_t), s);
    k_plan_next<<<blocks_for(nt, 256), 256, 0, s>>>(off[5], off[0], off[1], off[4], nt, cap, maskLim, next);
    sj_note_launch();
    k_plan_chain<<<1, 32, 0, s>>>(next, nt, start, nBatches);
    sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_plan_stats(const uint32_t *start, uint32_t nb, unsigned long long *const off[7],
                          unsigned long long *stats, cudaStream_t s)
{
    if (nb == 0) return cudaSuccess;
    OffOut o;
    for (int k = 0; k < NC; k++) o.p[k] = off[k];
    k_plan_stats<<<blocks_for(nb, 256), 256, 0, s>>>(start, nb, o, stats);
    sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_rates_mlp(const float *out, const uint32_t *cellStart, const uint32_t *nbrStart,
                         const uint32_t *nbrCell, uint32_t nCells, float *rate, cudaStream_t s)
{
    if (nCells == 0) return cudaSuccess;
    k_rates_mlp<<<blocks_for(nCells, 256), 256, 0, s>>>(out, cellStart, nbrStart, nbrCell, nCells, rate);
    sj_note_launch();
    return cudaGetLastError();
}

size_t sj_sample_totals_len() { return 4 * SAMPLE_BINS + 4; }

cudaError_t sj_sample_rates(const sj_task *tasks, uint32_t nt, const uint32_t *taskHits, const uint32_t *taskEvals,
                            const uint32_t *cellStart, unsigned long long *cellHits, unsigned long long *cellEvals,
                            unsigned long long *totals, uint32_t nCells, float *rate, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(cellHits, 0, sizeof(unsigned long long) * 2 * nCells, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(cellEvals, 0, sizeof(unsigned long long) * 2 * nCells, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(totals, 0, sizeof(unsigned long long) * sj_sample_totals_len(), s);
    if (e != cudaSuccess) return e;
    if (nt) {
        k_sample_sums<<<blocks_for(nt, 256), 256, 0, s>>>(tasks, nt, taskHits, taskEvals, cellStart, cellHits,
                                                          cellEvals, totals);
        sj_note_launch();
    }
    if (nCells) {
        k_sample_rates<<<blocks_for(nCells, 256), 256, 0, s>>>(cellHits, cellEvals, totals, cellStart, nCells, rate);
        sj_note_launch();
    }
    return cudaGetLastError();
}

cudaError_t sj_task_sums(const uint32_t *taskEvals, const uint32_t *taskRefined, const uint32_t *taskHits,
                         const float *pred, uint32_t nt, unsigned long long *sums, double *errSum, int numSM,
                         cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(sums, 0, sizeof(unsigned long long) * 3, s);
    if (e == cudaSuccess && errSum) e = cudaMemsetAsync(errSum, 0, sizeof(double), s);
    if (e != cudaSuccess || nt == 0) return e;
    unsigned grid = blocks_for(nt, 256);
    if (grid > (unsigned)numSM * 8) grid = (unsigned)numSM * 8;
    k_task_sums<<<grid, 256, 0, s>>>(taskEvals, taskRefined, taskHits, pred, nt, sums, errSum);
    sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_cell_hits(const uint32_t *cellStart, const uint32_t *ids, const uint32_t *deg, uint32_t nCells,
                         unsigned long long *hits, cudaStream_t s)
{
    if (nCells == 0) return cudaSuccess;
    k_cell_hits<<<blocks_for((uint64_t)nCells * 32, 256), 256, 0, s>>>(cellStart, ids, deg, nCells, hits);
    sj_note_launch();
    return cudaGetLastError();
}

size_t sj_scan64_temp(uint64_t n) { return (size_t)blocks_for(n ? n : 1, S64TILE); }

cudaError_t sj_exclusive_scan_u64(const unsigned long long *in, unsigned long long *out, uint64_t n,
                                  unsigned long long *temp, cudaStream_t s)
{
    if (n == 0) return cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
    const unsigned nb = blocks_for(n, S64TILE);
    k_s64_reduce<<<nb, S64T, 0, s>>>(in, n, temp);
    sj_note_launch();
    k_s64_scan_blocks<<<1, 32, 0, s>>>(temp, nb);
    sj_note_launch();
    k_s64_write<<<nb, S64T, 0, s>>>(in, n, temp, out);
    sj_note_launch();
    return cudaGetLastError();
}
