// The distance join's count pass over cell tasks.
//
// One CTA of 128 threads takes a task: up to 128*R query points of one cell
// (R query "slots" of 128; thread t holds queries t, t+128, ... in registers)
// against a stretch of that cell's candidate stream (home cell + owned
// neighbour cells, kernel.cu:1403-1538 in the reference).  Candidates are
// staged in shared memory in steps of SJ_STAGE and read as broadcasts; each
// staged candidate is loaded once per thread and evaluated against all R of
// its queries.  Per block of 32 candidates each thread builds a 32-bit hit mask
// per slot; a 5-step butterfly transposes a warp's 32x32 mask so that lane L
// holds candidate L's hits for the mirrored direction (symmetric traversals
// emit (p,q) and (q,p) from one evaluation).
//
// The pass produces per-key pair counts (the row lengths of a batch) and
// records every hit mask, each run's offset inside its key's run (the value an
// atomicAdd on the key's count returns) and the candidates' point ids; the
// emission pass (sj_emit.cu) writes the pairs from those records at the
// exclusive offsets of the counts, so each key's values land contiguously and
// keys come out ascending -- the order thrust::sort_by_key gives the reference
// (GPU.cu:2336) -- without sorting and without evaluating any distance twice.
//
// Predicate (kernel.cu:344-349): the squared distance in the reference build's
// rounding order (ref_dist2), hit iff sqrt(acc) <= eps, evaluated as acc <= T
// with T the largest double whose rounded sqrt is <= eps (identical by
// monotonicity of the correctly rounded square root).
// FP32 filter: |b|^2 - 2 a.b against T - |a|^2 in local coordinates around the
// home cell's centre; pairs inside a proven error band of the threshold are
// re-evaluated with the exact FP64 arithmetic, so the pair set is the FP64 set.
#include "sj_internal.h"
#include "sj_device.cuh"

#include <atomic>

#ifndef SJ_EVAL_UNROLL
#define SJ_EVAL_UNROLL 2    // unrolling of the per-block candidate loop
#endif

namespace {
using namespace sjdev;
constexpr int kEvalUnroll = SJ_EVAL_UNROLL;

constexpr int NW = SJ_CTA / 32;


// Squared distance in the reference build's exact rounding order (pinned by
// its own outputs): the first addition fuses the FIRST product,
//     acc = fma(d0, d0, d1*d1),  then  acc = fma(dl, dl, acc) for l >= 2,
// with d = cand - query (kernel.cu:344-347).  Padded dimensions hold 0 in both
// points and fma(0, 0, acc) == acc, so padding never changes the result.
template <int DP>
__device__ __forceinline__ double ref_dist2(const double *c, const double *q)
{
    const double d0 = __dsub_rn(c[0], q[0]);
    if (DP == 1) return __dmul_rn(d0, d0);
    const double d1 = __dsub_rn(c[1], q[1]);
    double acc = __fma_rn(d0, d0, __dmul_rn(d1, d1));
#pragma unroll
    for (int l = 2; l < DP; l++) {
        const double d = __dsub_rn(c[l], q[l]);
        acc = __fma_rn(d, d, acc);
    }
    return acc;
}

template <int DP>
__device__ __forceinline__ bool exact_hit(const double *__restrict__ xs, uint32_t cpos, uint32_t qpos, double T)
{
    return ref_dist2<DP>(xs + (uint64_t)cpos * DP, xs + (uint64_t)qpos * DP) <= T;
}

template <int DP>
struct __align__(16) Stage64 {
    static constexpr int S = (DP <= 8) ? SJ_STAGE : ((SJ_STAGE * 8 / DP) / 32) * 32;
    double c[S][DP];
};

// FP32 stage: candidates in pairs (2p, 2p+1) so that one packed f32x2
// instruction evaluates a query against both; per pair, float2 0 holds the
// two |b|^2 and float2 1+l the two local coordinates l.
template <int DP>
struct __align__(16) Stage32 {
    static constexpr int CW2 = ((DP + 1) + 1) / 2 * 2;   // float2 per pair, even (16-byte rows)
    static constexpr int S = SJ_STAGE;
    float2 c[S / 2][CW2];
};

template <int DP, bool F32>
struct StageOf { using T = Stage64<DP>; };
template <int DP>
struct StageOf<DP, true> { using T = Stage32<DP>; };

// mask << 1 | sign bit of v: one funnel shift (the value's bits are not
// inspected as a float, so no comparison is generated)
__device__ __forceinline__ uint32_t push_sign(uint32_t mask, float v)
{
    uint32_t r;
    asm("shf.l.wrap.b32 %0, %1, %2, 1;" : "=r"(r) : "r"(__float_as_uint(v)), "r"(mask));
    return r;
}

// FP32 filter over one block of 32 staged candidates for slots 0..RR-1.
//   y = (|b|^2 - tLo) + sum_l (-2 a_l) b_l      (packed f32x2: two candidates per op)
// hit bit <- sign(y): y < 0 proves the FP64 predicate true; y >= delta proves
// it false; 0 <= y < delta is the borderline band.  Bits are shifted in from
// candidate 31 down to 0, so bit i is candidate i.  Instead of a second
// comparison per candidate, lo[r] keeps the smallest bit pattern of y over the
// block: a y in [0, delta) has a smaller pattern than delta's (non-negative
// floats order like their bits; negative ones have the sign bit and never win
// the unsigned minimum), so ymin < bits(delta) tells that the block has a
// borderline candidate, which near_bits() then finds.
template <int DP, int RR, int R>
__device__ __forceinline__ void eval_block_f32(const Stage32<DP> &st, uint32_t pb, const float2 (&qa)[R][DP],
                                               const float2 (&nt)[R], uint32_t (&hit)[R], uint32_t (&ymin)[R])
{
    constexpr int CW2 = Stage32<DP>::CW2;
#pragma unroll kEvalUnroll
    for (int p = 15; p >= 0; p--) {
        const float4 *row = reinterpret_cast<const float4 *>(&st.c[pb + p][0]);
        float2 y[RR];
        {
            const float4 v = row[0];
            const float2 nb = make_float2(v.x, v.y);
#pragma unroll
            for (int r = 0; r < RR; r++) y[r] = __fadd2_rn(nb, nt[r]);
            if (DP >= 1) {
                const float2 b = make_float2(v.z, v.w);
#pragma unroll
                for (int r = 0; r < RR; r++) y[r] = __ffma2_rn(qa[r][0], b, y[r]);
            }
        }
#pragma unroll
        for (int h = 1; h < CW2 / 2; h++) {
            const float4 v = row[h];
            if (2 * h - 1 < DP) {
                const float2 b = make_float2(v.x, v.y);
#pragma unroll
                for (int r = 0; r < RR; r++) y[r] = __ffma2_rn(qa[r][2 * h - 1], b, y[r]);
            }
            if (2 * h < DP) {
                const float2 b = make_float2(v.z, v.w);
#pragma unroll
                for (int r = 0; r < RR; r++) y[r] = __ffma2_rn(qa[r][2 * h], b, y[r]);
            }
        }
#pragma unroll
        for (int r = 0; r < RR; r++) {
            hit[r] = push_sign(hit[r], y[r].y);
            hit[r] = push_sign(hit[r], y[r].x);
            ymin[r] = min(ymin[r], min(__float_as_uint(y[r].x), __float_as_uint(y[r].y)));
        }
    }
}

// Borderline candidates of one block for the query of slot qa/nt: the same
// FP32 operations as eval_block_f32 in the same order (so y is bitwise the
// same), one candidate at a time; bit i set when 0 <= y_i < delta.  Runs only
// for blocks whose minimum says that such a candidate exists.
template <int DP>
__device__ __forceinline__ uint32_t near_bits(const Stage32<DP> &st, uint32_t pb, const float2 (&qa)[DP], float2 nt,
                                           float delta)
{
    constexpr int CW2 = Stage32<DP>::CW2;
    uint32_t m = 0;
    for (int p = 0; p < 16; p++) {
        const float *row = reinterpret_cast<const float *>(&st.c[pb + p][0]);
        for (int h = 0; h < 2; h++) {
            float y = __fadd_rn(row[h], nt.x);
#pragma unroll
            for (int l = 0; l < DP; l++) y = __fmaf_rn(qa[l].x, row[2 * (1 + l) + h], y);
            if (__float_as_uint(y) < __float_as_uint(delta)) m |= 1u << (2 * p + h);
        }
    }
    (void)CW2;
    return m;
}

// FP64 predicate over one block of 32 staged candidates for slots 0..RR-1, in
// the reference's rounding order (ref_dist2).  acc >= 0, so acc <= T is the
// sign of bits(acc) - (bits(T) + 1) as 64-bit integers.
template <int DP, int RR, int R>
__device__ __forceinline__ void eval_block_f64(const Stage64<DP> &st, uint32_t jb, const double (&q)[R][DP],
                                               long long T1, uint32_t (&hit)[R])
{
#pragma unroll kEvalUnroll
    for (int jj = 31; jj >= 0; jj--) {
        const double *cb = &st.c[jb + jj][0];
        double acc[RR];
        {
            const double c0 = cb[0];
            if (DP == 1) {
#pragma unroll
                for (int r = 0; r < RR; r++) {
                    const double d0 = __dsub_rn(c0, q[r][0]);
                    acc[r] = __dmul_rn(d0, d0);
                }
            } else {
                const double c1 = cb[DP > 1 ? 1 : 0];
#pragma unroll
                for (int r = 0; r < RR; r++) {
                    const double d0 = __dsub_rn(c0, q[r][0]);
                    const double d1 = __dsub_rn(c1, q[r][DP > 1 ? 1 : 0]);
                    acc[r] = __fma_rn(d0, d0, __dmul_rn(d1, d1));
                }
            }
        }
#pragma unroll
        for (int l = 2; l < DP; l++) {
            const double cl = cb[l];
#pragma unroll
            for (int r = 0; r < RR; r++) {
                const double d = __dsub_rn(cl, q[r][l]);
                acc[r] = __fma_rn(d, d, acc[r]);
            }
        }
#pragma unroll
        for (int r = 0; r < RR; r++) {
            const long long diff = __double_as_longlong(acc[r]) - T1;
            hit[r] = push_sign(hit[r], __int_as_float((int)((unsigned long long)diff >> 32)));
        }
    }
}

// Shared memory of one count-pass CTA.
template <int DP, bool F32, int R>
struct __align__(16) JoinSmem {
    using Stage = typename StageOf<DP, F32>::T;
    static constexpr int S = Stage::S;
    Stage st;
    uint32_t candId[S];
    uint32_t segStart[SJ_MAX_SEG];
    uint32_t segPre[SJ_MAX_SEG + 1];
    uint32_t colCnt[NW][S];
    double originS[F32 ? DP : 1];
    uint32_t scanTmp[NW];
    uint32_t curTask;
    unsigned long long taskPairs;
    unsigned long long taskEvals;
    unsigned long long taskRefined;
};

// Count pass over tasks [taskBegin, taskEnd): per-key pair counts (keyCount,
// both directions of symmetric tasks), the batch total, and -- when a.masks is
// set -- every query's hit mask per block of 32 stream positions plus its row
// count, which the emission pass turns into pairs without a second distance
// evaluation.
// Resident CTAs per SM the register allocation must allow: the FP32 filter
// gains from a fifth CTA, the FP64 predicate from keeping its registers.
#ifndef SJ_JOIN_MIN_BLOCKS_F32
#define SJ_JOIN_MIN_BLOCKS_F32 5
#endif
#ifndef SJ_JOIN_MIN_BLOCKS_F64
#define SJ_JOIN_MIN_BLOCKS_F64 1
#endif

template <int DP, bool F32, int R>
__global__ void __launch_bounds__(SJ_CTA, F32 ? SJ_JOIN_MIN_BLOCKS_F32 : SJ_JOIN_MIN_BLOCKS_F64) k_join(sj_join_args a, sj_grid_dev g, int queue)
{
    using Smem = JoinSmem<DP, F32, R>;
    constexpr int S = Smem::S;
    __shared__ Smem sm;
    auto &st = sm.st;
    auto &candId = sm.candId;
    auto &segStart = sm.segStart;
    auto &segPre = sm.segPre;
    auto &colCnt = sm.colCnt;
    auto &originS = sm.originS;

    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    const uint32_t warp = tid >> 5;
    const int D = g.D;
    const double T = g.thresh;

    for (int j = tid; j < NW * S; j += SJ_CTA) (&colCnt[0][0])[j] = 0;

    uint32_t iter = 0;
    for (;;) {
        // ---- fetch the next task
        __syncthreads();
        if (tid == 0) {
            uint32_t t = queue ? (a.taskBegin + atomicAdd(a.queueHead, 1u)) : (a.taskBegin + blockIdx.x + iter);
            sm.curTask = t;
            sm.taskPairs = 0ULL;
            sm.taskEvals = 0ULL;
            sm.taskRefined = 0ULL;
        }
        __syncthreads();
        const uint32_t t = sm.curTask;
        if (t >= a.taskEnd || (!queue && iter > 0)) break;
        iter++;
        const sj_task task = a.tasks[t];
        const bool sym = (task.flags & SJ_TASK_SYM) != 0;
        const uint32_t cellA = task.cell;
        const uint32_t aStart = a.cellStart[cellA], aEnd = a.cellStart[cellA + 1];
        const uint32_t nbrBase = a.nbrStart[cellA];
        const uint32_t nSeg = task.segCount;

        // ---- segment table (exclusive prefix of lengths over the task's segments)
        uint32_t locLen[(SJ_MAX_SEG + SJ_CTA - 1) / SJ_CTA];
        uint32_t mySum = 0;
#pragma unroll
        for (int r = 0; r < (SJ_MAX_SEG + SJ_CTA - 1) / SJ_CTA; r++) {
            uint32_t s = tid * ((SJ_MAX_SEG + SJ_CTA - 1) / SJ_CTA) + r;
            uint32_t len = 0;
            if (s < nSeg) {
                uint32_t gs = task.segBase + s;
                uint32_t st0, en;
                if (gs == 0) {
                    st0 = sym ? task.qBegin : aStart;
                    en = aEnd;
                } else {
                    uint32_t b = a.nbrCell[nbrBase + gs - 1];
                    st0 = a.cellStart[b];
                    en = a.cellStart[b + 1];
                }
                segStart[s] = st0;
                len = en - st0;
            }
            locLen[r] = len;
            mySum += len;
        }
        if (F32 && (int)tid < DP) {
            // local-coordinate origin: home cell centre (indexed dims), data centre (others)
            double o;
            if ((int)tid < g.k) o = g.minArr[tid] + ((double)a.cellCoord[(uint64_t)cellA * g.k + tid] + 0.5) * g.eps;
            else if ((int)tid < D) o = g.center[tid];
            else o = 0.0;
            originS[F32 ? tid : 0] = o;
        }
        {
            // block exclusive scan of mySum
            uint32_t x = mySum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= (uint32_t)o) x += y;
            }
            if (lane == 31) sm.scanTmp[warp] = x;
            __syncthreads();
            uint32_t wpre = 0;
            for (uint32_t w = 0; w < warp; w++) wpre += sm.scanTmp[w];
            uint32_t run = wpre + x - mySum;
#pragma unroll
            for (int r = 0; r < (SJ_MAX_SEG + SJ_CTA - 1) / SJ_CTA; r++) {
                uint32_t s = tid * ((SJ_MAX_SEG + SJ_CTA - 1) / SJ_CTA) + r;
                if (s <= nSeg) segPre[s] = run;
                run += locLen[r];
            }
            if (tid == SJ_CTA - 1) segPre[nSeg] = run;   // grand total (also covers nSeg == SJ_MAX_SEG)
        }
        __syncthreads();
        const uint32_t homeEnd = (task.segBase == 0 && (task.flags & SJ_TASK_HOME)) ? segPre[1] : 0u;

        // ---- query points of this thread: slot r holds query r*128 + tid
        // nAct: slots with at least one valid query in this warp (warp-uniform)
        const uint32_t nAct = task.qCount > warp * 32
                                  ? min((uint32_t)R, (task.qCount - warp * 32 + SJ_CTA - 1) / SJ_CTA)
                                  : 0u;
        uint32_t qid[R];
        double q64[F32 ? 1 : R][F32 ? 1 : DP];
        float2 qa[F32 ? R : 1][F32 ? DP : 1];   // (-2 a_l, -2 a_l)
        float2 nt[R];                           // (-tLo, -tLo)
#pragma unroll
        for (int r = 0; r < R; r++) {
            const uint32_t qi = (uint32_t)r * SJ_CTA + tid;
            const bool v = qi < task.qCount;
            const uint32_t qpos = task.qBegin + (v ? qi : 0u);
            qid[r] = a.ids[qpos];
            const double *src = a.xs + (uint64_t)qpos * DP;
            if (F32) {
                double na = 0.0;
#pragma unroll
                for (int l = 0; l < DP; l++) {
                    const float ql = (l < D) ? __double2float_rn(src[l] - originS[F32 ? l : 0]) : 0.0f;
                    qa[F32 ? r : 0][F32 ? l : 0] = make_float2(-2.0f * ql, -2.0f * ql);
                    na += (double)ql * (double)ql;
                }
                const float tLo = __double2float_rd(T - na - a.margin);
                nt[r] = make_float2(-tLo, -tLo);
            } else {
#pragma unroll
                for (int l = 0; l < DP; l++) q64[F32 ? 0 : r][F32 ? 0 : l] = src[l];
                nt[r] = make_float2(0.f, 0.f);
            }
        }
        const long long T1 = __double_as_longlong(T) + 1;
        uint32_t *const maskBase = a.masks ? a.masks + (a.maskOff[t] - a.maskOff[a.taskBegin]) : nullptr;
        uint32_t *const colBase = (a.colMasks && sym) ? a.colMasks + (a.colOff[t] - a.colOff[a.taskBegin]) : nullptr;
        const uint64_t candRecOff = a.candOff ? a.candOff[t] - a.candOff[a.taskBegin] : 0;
        uint32_t *const candIdRec = a.candId ? a.candId + candRecOff : nullptr;
        uint32_t *const candRelRec = (a.candRel && sym) ? a.candRel + candRecOff : nullptr;

        uint32_t rowCount[R];   // pairs keyed by each query
        uint32_t evals = 0;     // candidate evaluations
        uint32_t refined = 0;   // FP32 borderline re-evaluations
#pragma unroll
        for (int r = 0; r < R; r++) rowCount[r] = 0;

        // the stream can never extend past the segments actually present
        const uint32_t sEnd = min(task.sEnd, segPre[nSeg]);
        const uint32_t nBlk = (sEnd - task.sBegin + 31) / 32;
        const uint32_t nG = (task.qCount + 31) / 32;
        for (uint32_t sBase = task.sBegin; sBase < sEnd; sBase += S) {
            const uint32_t nIn = min((uint32_t)S, sEnd - sBase);
            __syncthreads();
            // ---- stage candidates
            for (uint32_t j = tid; j < nIn; j += SJ_CTA) {
                uint32_t s = sBase + j;
                uint32_t lo = 0, hi = nSeg;   // largest seg with segPre[seg] <= s
                while (hi - lo > 1) {
                    uint32_t mid = (lo + hi) >> 1;
                    if (segPre[mid] <= s) lo = mid; else hi = mid;
                }
                uint32_t pos = segStart[lo] + (s - segPre[lo]);
                const uint32_t cid = a.ids[pos];
                candId[j] = cid;
                if (candIdRec) candIdRec[s - task.sBegin] = cid;   // the emission's candidate record
                const double *src = a.xs + (uint64_t)pos * DP;
                if constexpr (F32) {
                    float *dst = reinterpret_cast<float *>(&st.c[j >> 1][0]) + (j & 1);
                    double nb = 0.0;
#pragma unroll
                    for (int l = 0; l < DP; l++) {
                        float b = (l < D) ? __double2float_rn(src[l] - originS[F32 ? l : 0]) : 0.0f;
                        dst[2 * (1 + l)] = b;
                        nb += (double)b * (double)b;
                    }
                    dst[0] = __double2float_rn(nb);
                } else {
                    double *dst = reinterpret_cast<double *>(&st.c[j][0]);
#pragma unroll
                    for (int l = 0; l < DP; l++) dst[l] = src[l];
                }
            }
            __syncthreads();
            // ---- hit masks of every block of the stage.  A warp without
            // queries skips the evaluation (but not the barriers).
#pragma unroll 1
            for (uint32_t jb = 0; nAct != 0 && jb < nIn; jb += 32) {
                const uint32_t nb = min(32u, nIn - jb);
                const uint32_t inRange = (nb == 32) ? 0xffffffffu : ((1u << nb) - 1u);
                uint32_t hits[R], ymin[R];
#pragma unroll
                for (int r = 0; r < R; r++) { hits[r] = 0; ymin[r] = 0xffffffffu; }
                // branch-free evaluation of the warp's active slots (a partly
                // active slot set rounds up; the extra slots are ignored below)
                if constexpr (F32) {
                    if (nAct == 1) eval_block_f32<DP, 1, R>(st, jb >> 1, qa, nt, hits, ymin);
                    else eval_block_f32<DP, R, R>(st, jb >> 1, qa, nt, hits, ymin);
                } else {
                    if (nAct == 1) eval_block_f64<DP, 1, R>(st, jb, q64, T1, hits);
                    else eval_block_f64<DP, R, R>(st, jb, q64, T1, hits);
                }
                const uint32_t blk = sBase + jb;
                const uint32_t hb = home_bits(blk, homeEnd, sym);
                const uint32_t bInTask = (blk - task.sBegin) >> 5;
                // record addresses of this block: row masks [chunk][query][block in
                // chunk], column masks [block][query group][candidate]
                uint32_t *const rowRec = maskBase ? maskBase + sj_row_mask_index(bInTask, 0, task.qCount, nBlk) : nullptr;
                const uint32_t rowStride = min(64u, nBlk - (bInTask & ~63u));
                uint32_t *const colRec = colBase ? colBase + ((uint64_t)bInTask * nG + warp) * 32 + lane : nullptr;
                uint32_t colHits = 0;   // this lane's candidate: hits over the warp's slots
#pragma unroll
                for (int r = 0; r < R; r++) {
                    if ((uint32_t)r >= nAct) continue;   // warp-uniform
                    const uint32_t qi = (uint32_t)r * SJ_CTA + tid;
                    const bool qValid = qi < task.qCount;
                    const uint32_t rowValid = qValid ? (hb ? (inRange & row_keep(qi, blk, hb)) : inRange) : 0u;
                    uint32_t h = hits[r];
                    if constexpr (F32) {
                        if (ymin[r] < __float_as_uint(a.delta)) {
                            uint32_t bm = near_bits<DP>(st, jb >> 1, qa[r], nt[r], a.delta) & ~h & rowValid;
                            while (bm) {
                                const int jj = __ffs(bm) - 1;
                                bm &= bm - 1;
                                const uint32_t s = blk + jj;
                                uint32_t lo = 0, hi = nSeg;
                                while (hi - lo > 1) {
                                    const uint32_t mid = (lo + hi) >> 1;
                                    if (segPre[mid] <= s) lo = mid; else hi = mid;
                                }
                                const uint32_t cpos = segStart[lo] + (s - segPre[lo]);
                                refined++;
                                if (exact_hit<DP>(a.xs, cpos, task.qBegin + qi, T)) h |= 1u << jj;
                            }
                        }
                    }
                    const uint32_t rowMask = h & rowValid;   // lane = query, bit = candidate
                    if (rowRec && qValid) rowRec[(uint64_t)qi * rowStride] = rowMask;
                    rowCount[r] += __popc(rowMask);
                    if (sym) {
                        // the mirrored direction: lane L gets candidate L's hits (none
                        // to transpose when the warp's block has no hit at all)
                        const uint32_t mir = hb ? (rowMask & mir_keep(qi, blk, hb)) : rowMask;
                        const uint32_t colW = __any_sync(0xffffffffu, mir) ? transpose32(mir, lane) : 0u;
                        colHits += __popc(colW);
                        if (colRec) colRec[(uint32_t)r * NW * 32] = colW;
                    }
                }
                if (sym && colHits) colCnt[warp][jb + lane] += colHits;
            }
            if (sym) {
                __syncthreads();
                uint32_t local = 0;
                for (uint32_t j = tid; j < nIn; j += SJ_CTA) {
                    uint32_t tot = 0;
#pragma unroll
                    for (int w = 0; w < NW; w++) { tot += colCnt[w][j]; colCnt[w][j] = 0; }
                    // the count before this stage's addition is the offset of
                    // these column pairs inside the candidate's key run
                    const uint32_t rel = tot ? atomicAdd(&a.keyCount[candId[j]], tot) : 0u;
                    if (candRelRec) candRelRec[sBase + j - task.sBegin] = rel;
                    local += tot;
                }
                if (local) atomicAdd(&sm.taskPairs, (unsigned long long)local);
            }
        }
        {
            uint32_t mine = 0;
            uint32_t *const rowBase = a.rowRel ? a.rowRel + (a.rowOff[t] - a.rowOff[a.taskBegin]) : nullptr;
#pragma unroll
            for (int r = 0; r < R; r++) {
                const uint32_t qi = (uint32_t)r * SJ_CTA + tid;
                // evaluations of this query: stream positions [sBegin, sEnd), in the
                // symmetric home segment only those at or after the query itself
                if (qi < task.qCount) {
                    const uint32_t from = max(task.sBegin, min(qi, sym ? homeEnd : 0u));
                    evals += sEnd > from ? sEnd - from : 0u;
                }
                // the key's count before this addition: where this task's row
                // run starts inside the query's key run
                const uint32_t rel = rowCount[r] ? atomicAdd(&a.keyCount[qid[r]], rowCount[r]) : 0u;
                if (rowBase && qi < task.qCount) rowBase[qi] = rel;
                mine += rowCount[r];
            }
            if (mine) atomicAdd(&sm.taskPairs, (unsigned long long)mine);
        }
        // ---- statistics (per task: a re-run of the task overwrites them)
        unsigned long long e = evals, rf = refined;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            e += __shfl_xor_sync(0xffffffffu, e, o);
            rf += __shfl_xor_sync(0xffffffffu, rf, o);
        }
        if (lane == 0) {
            if (e) atomicAdd(&sm.taskEvals, e);
            if (rf) atomicAdd(&sm.taskRefined, rf);
        }
        __syncthreads();
        if (tid == 0) {
            const unsigned long long tp = sm.taskPairs;
            if (tp) {
                atomicAdd(&a.stat[2], tp);
                if (a.batchPairs) atomicAdd(a.batchPairs, tp);
            }
            if (a.taskHits) a.taskHits[t] = (uint32_t)min(tp, 0xffffffffULL);
            if (a.taskEvals) a.taskEvals[t] = (uint32_t)min(sm.taskEvals, 0xffffffffULL);
            if (a.taskRefined) a.taskRefined[t] = (uint32_t)min(sm.taskRefined, 0xffffffffULL);
        }
    }
}

template <int DP, bool F32>
int occupancy_of()
{
    constexpr int MAXDEV = 64;
    static std::atomic<int> occ[MAXDEV];   // per device ordinal, 0 = not measured yet
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= MAXDEV) dev = 0;
    int o = occ[dev].load();
    if (o == 0) {
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_join<DP, F32, sj_query_slots(DP, F32)>, SJ_CTA, 0);
        o = b > 0 ? b : 1;
        occ[dev].store(o);
    }
    return o;
}

template <int DP, bool F32>
cudaError_t launch_one(const sj_join_args &a, const sj_grid_dev &g, int queue, int numSM, int maxCtasPerSM,
                       cudaStream_t s)
{
    const uint32_t nt = a.taskEnd - a.taskBegin;
    if (nt == 0) return cudaSuccess;
    // persistent queue: one full wave of resident CTAs (or fewer per SM, to
    // leave room for a kernel of the other stream)
    int perSM = occupancy_of<DP, F32>();
    if (maxCtasPerSM > 0 && maxCtasPerSM < perSM) perSM = maxCtasPerSM;
    unsigned grid = queue ? (unsigned)(numSM * perSM) : nt;
    if (queue && grid > nt) grid = nt;
    k_join<DP, F32, sj_query_slots(DP, F32)><<<grid, SJ_CTA, 0, s>>>(a, g, queue);
    sj_note_launch();
    return cudaGetLastError();
}

template <int DP>
cudaError_t launch_dp(const sj_join_args &a, const sj_grid_dev &g, int fp32, int queue, int numSM, int maxCtas,
                      cudaStream_t s)
{
    return fp32 ? launch_one<DP, true>(a, g, queue, numSM, maxCtas, s)
                : launch_one<DP, false>(a, g, queue, numSM, maxCtas, s);
}

}  // namespace

cudaError_t sj_launch_join(const sj_join_args &a, const sj_grid_dev &g, int fp32, int queue, int numSM,
                           int maxCtasPerSM, cudaStream_t s)
{
    switch (g.Dp) {
    case 1: return launch_dp<1>(a, g, fp32, queue, numSM, maxCtasPerSM, s);
    case 2: return launch_dp<2>(a, g, fp32, queue, numSM, maxCtasPerSM, s);
    case 3: return launch_dp<3>(a, g, fp32, queue, numSM, maxCtasPerSM, s);
    case 4: return launch_dp<4>(a, g, fp32, queue, numSM, maxCtasPerSM, s);
    case 6: return launch_dp<6>(a, g, fp32, queue, numSM, maxCtasPerSM, s);
    case 8: return launch_dp<8>(a, g, fp32, queue, numSM, maxCtasPerSM, s);
    case 12: return launch_dp<12>(a, g, fp32, queue, numSM, maxCtasPerSM, s);
    case 16: return launch_dp<16>(a, g, fp32, queue, numSM, maxCtasPerSM, s);
    }
    return cudaErrorInvalidValue;
}
