// The distance join: count pass and fill pass over cell tasks.
//
// One CTA of 128 threads takes a task: up to 128 query points of one cell
// (one per thread, coordinates in registers) against a stretch of that cell's
// candidate stream (home cell + owned neighbour cells, kernel.cu:1403-1538 in
// the reference).  Candidates are staged in shared memory in steps of
// SJ_STAGE and read by every thread as broadcasts.  Each thread builds a
// 32-bit hit mask per block of 32 candidates; a 5-step butterfly transposes the
// warp's 32x32 mask so that lane L holds candidate L's hits for the mirrored
// direction (symmetric traversals emit (p,q) and (q,p) from one evaluation).
//
// count pass: per-key pair counts (the row lengths of this batch).
// fill pass : keys are placed at exclusive offsets of those counts, so every
//             key's values land contiguously and keys come out ascending --
//             the order thrust::sort_by_key gives the reference (GPU.cu:2336)
//             without sorting.  Each key's share of a 32x32 block is written as
//             one run by the whole warp (ballot rank -> consecutive addresses).
//
// Predicate (kernel.cu:344-349): the squared distance in the reference build's
// rounding order (ref_dist2), hit iff sqrt(acc) <= eps, evaluated as acc <= T
// with T the largest double whose rounded sqrt is <= eps (identical by
// monotonicity of the correctly rounded square root).
// FP32 filter: acc32 = |b|^2 + sum(-2 a_l b_l) in local coordinates around the
// home cell's centre; pairs inside a proven error band of the threshold are
// re-evaluated with the exact FP64 chain above, so the pair set is the FP64 set.
#include "sj_internal.h"

namespace {

constexpr int NW = SJ_CTA / 32;
constexpr int EMIT_STAGE = 256;   // staged emissions per warp and direction (sparse blocks)

__device__ __forceinline__ uint32_t transpose32(uint32_t x, uint32_t lane)
{
    // Lane i holds row i of a 32x32 bit matrix; afterwards lane j holds column j.
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        const uint32_t lo = (s == 16) ? 0x0000ffffu
                          : (s == 8)  ? 0x00ff00ffu
                          : (s == 4)  ? 0x0f0f0f0fu
                          : (s == 2)  ? 0x33333333u
                                      : 0x55555555u;
        uint32_t y = __shfl_xor_sync(0xffffffffu, x, s);
        if (lane & s) x = (x & ~lo) | ((y & ~lo) >> s);
        else x = (x & lo) | ((y & lo) << s);
    }
    return x;
}

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
struct Stage64 {
    static constexpr int S = (DP <= 8) ? SJ_STAGE : ((SJ_STAGE * 8 / DP) / 32) * 32;
    double c[S][DP];
};

template <int DP>
struct Stage32 {
    static constexpr int CW = ((DP + 1 + 3) / 4) * 4;
    static constexpr int S = SJ_STAGE;
    float c[S][CW];   // local coordinates, then |b|^2 at [DP]
};

template <int DP, bool F32>
struct StageOf { using T = Stage64<DP>; };
template <int DP>
struct StageOf<DP, true> { using T = Stage32<DP>; };

template <int DP, bool F32, bool FILL>
__global__ void __launch_bounds__(SJ_CTA) k_join(sj_join_args a, sj_grid_dev g, int queue)
{
    using Stage = typename StageOf<DP, F32>::T;
    constexpr int S = Stage::S;
    __shared__ Stage st;
    __shared__ uint32_t candId[S];
    __shared__ uint32_t segStart[SJ_MAX_SEG];
    __shared__ uint32_t segPre[SJ_MAX_SEG + 1];
    __shared__ uint32_t colCnt[FILL ? 1 : NW][FILL ? 1 : S];
    // fill pass, sparse blocks: per-warp staging of (slot, key, value)
    __shared__ uint32_t stSlot[FILL ? NW : 1][FILL ? EMIT_STAGE : 1];
    __shared__ uint32_t stKey[FILL ? NW : 1][FILL ? EMIT_STAGE : 1];
    __shared__ uint32_t stVal[FILL ? NW : 1][FILL ? EMIT_STAGE : 1];
    __shared__ uint32_t qIdS[FILL ? SJ_CTA : 1];
    __shared__ uint32_t scanTmp[NW];
    __shared__ uint32_t curTask;
    __shared__ unsigned long long taskPairs;

    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    const uint32_t warp = tid >> 5;
    const uint32_t ltmask = (1u << lane) - 1u;
    const int D = g.D;
    // fill pass of a batch whose count exceeded the output buffer: skip it
    // (the host re-plans it); the count pass always runs
    if (FILL && a.batchPairs && *a.batchPairs > a.capacity) {
        if (tid == 0 && blockIdx.x == 0) atomicMax(&a.stat[5], 1ULL);
        return;
    }
    const double T = g.thresh;

    if (!FILL) {
        for (int j = tid; j < NW * S; j += SJ_CTA) (&colCnt[0][0])[j] = 0;
    }

    uint32_t iter = 0;
    for (;;) {
        // ---- fetch the next task
        __syncthreads();
        if (tid == 0) {
            uint32_t t = queue ? (a.taskBegin + atomicAdd(a.queueHead, 1u)) : (a.taskBegin + blockIdx.x + iter);
            curTask = t;
            taskPairs = 0ULL;
        }
        __syncthreads();
        const uint32_t t = curTask;
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
        {
            // block exclusive scan of mySum
            uint32_t x = mySum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= (uint32_t)o) x += y;
            }
            if (lane == 31) scanTmp[warp] = x;
            __syncthreads();
            uint32_t wpre = 0;
            for (uint32_t w = 0; w < warp; w++) wpre += scanTmp[w];
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

        // ---- query point of this thread
        const uint32_t qi = tid;
        const bool qValid = qi < task.qCount;
        const uint32_t qpos = task.qBegin + (qValid ? qi : 0u);
        const uint32_t qid = a.ids[qpos];
        if (FILL) qIdS[tid] = qid;
        double q64[F32 ? 1 : DP];
        float q2[F32 ? DP : 1];
        float thrLo = 0.f, thrHi = 0.f;
        double origin[F32 ? DP : 1];
        if (F32) {
            double na = 0.0;
#pragma unroll
            for (int l = 0; l < DP; l++) {
                double o;
                if (l < g.k) o = g.minArr[l] + ((double)a.cellCoord[(uint64_t)cellA * g.k + l] + 0.5) * g.eps;
                else if (l < D) o = g.center[l];
                else o = 0.0;
                origin[l] = o;
                float qa = (l < D) ? __double2float_rn(a.xs[(uint64_t)qpos * DP + l] - o) : 0.0f;
                q2[l] = -2.0f * qa;
                na += (double)qa * (double)qa;
            }
            thrLo = __double2float_rd(T - na - a.margin);
            thrHi = __double2float_ru(T - na + a.margin);
        } else {
#pragma unroll
            for (int l = 0; l < DP; l++) q64[l] = a.xs[(uint64_t)qpos * DP + l];
        }

        uint32_t rowCount = 0;       // count pass: pairs keyed by this query
        uint32_t evals = 0;          // candidate evaluations
        uint32_t refined = 0;        // FP32 borderline re-evaluations

        // the stream can never extend past the segments actually present
        const uint32_t sEnd = min(task.sEnd, segPre[nSeg]);
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
                candId[j] = a.ids[pos];
                const double *src = a.xs + (uint64_t)pos * DP;
                if (F32) {
                    float *dst = reinterpret_cast<float *>(&st.c[j][0]);
                    double nb = 0.0;
#pragma unroll
                    for (int l = 0; l < DP; l++) {
                        float b = (l < D) ? __double2float_rn(src[l] - origin[l]) : 0.0f;
                        dst[l] = b;
                        nb += (double)b * (double)b;
                    }
                    dst[DP] = __double2float_rn(nb);
                } else {
                    double *dst = reinterpret_cast<double *>(&st.c[j][0]);
#pragma unroll
                    for (int l = 0; l < DP; l++) dst[l] = src[l];
                }
            }
            __syncthreads();

            for (uint32_t jb = 0; jb < nIn; jb += 32) {
                const uint32_t nb = min(32u, nIn - jb);
                const uint32_t inRange = (nb == 32) ? 0xffffffffu : ((1u << nb) - 1u);
                uint32_t hits = 0, border = 0;
                if (qValid) {
#pragma unroll
                    for (int jj = 0; jj < 32; jj++) {
                        if (jj < (int)nb) {
                            const int j = jb + jj;
                            if (F32) {
                                const float *cb = reinterpret_cast<const float *>(&st.c[j][0]);
                                float acc = cb[DP];
#pragma unroll
                                for (int l = 0; l < DP; l++) acc = fmaf(q2[l], cb[l], acc);
                                if (acc <= thrLo) hits |= 1u << jj;
                                else if (acc <= thrHi) border |= 1u << jj;
                            } else {
                                const double *cb = reinterpret_cast<const double *>(&st.c[j][0]);
                                if (ref_dist2<DP>(cb, q64) <= T) hits |= 1u << jj;
                            }
                        }
                    }
                }
                // validity: the symmetric home segment keeps only cand >= query
                uint32_t rowValid = inRange, mirValid = sym ? inRange : 0u;
                const uint32_t blk = sBase + jb;
                if (blk < homeEnd) {
                    uint32_t hn = homeEnd - blk;
                    uint32_t homeBits = hn >= 32 ? 0xffffffffu : ((1u << hn) - 1u);
                    if (sym) {
                        int lo = (int)qi - (int)blk;     // home cand index >= query index
                        uint32_t ge = lo <= 0 ? 0xffffffffu : (lo >= 32 ? 0u : (0xffffffffu << lo));
                        uint32_t gt = (lo + 1) <= 0 ? 0xffffffffu : ((lo + 1) >= 32 ? 0u : (0xffffffffu << (lo + 1)));
                        rowValid &= (~homeBits) | (homeBits & ge);
                        mirValid &= (~homeBits) | (homeBits & gt);
                    }
                }
                if (!qValid) { rowValid = 0; mirValid = 0; }
                if (F32) {
                    uint32_t bm = border & rowValid;
                    while (bm) {
                        int jj = __ffs(bm) - 1;
                        bm &= bm - 1;
                        uint32_t s = blk + jj;
                        uint32_t lo = 0, hi = nSeg;
                        while (hi - lo > 1) {
                            uint32_t mid = (lo + hi) >> 1;
                            if (segPre[mid] <= s) lo = mid; else hi = mid;
                        }
                        uint32_t cpos = segStart[lo] + (s - segPre[lo]);
                        refined++;
                        if (exact_hit<DP>(a.xs, cpos, qpos, T)) hits |= 1u << jj;
                    }
                }
                evals += __popc(rowValid);
                const uint32_t rowMask = hits & rowValid;   // lane = query, bit = candidate
                const uint32_t mirRow = hits & mirValid;    // pairs also emitted with the candidate as key
                if (FILL) {
                    // rowT / mirT: lane j holds, for candidate jb+j, the bit mask of
                    // this warp's queries it pairs with (one transpose suffices
                    // outside the home diagonal, where both masks agree)
                    const bool diag = sym && (blk < homeEnd);
                    const uint32_t rowT = transpose32(rowMask, lane);
                    const uint32_t mirT = sym ? (diag ? transpose32(mirRow, lane) : rowT) : 0u;
                    const uint32_t cidL = candId[jb + lane];
                    const uint32_t nRow = __popc(rowMask), nCol = __popc(mirT);
                    uint32_t pRow = 0, pCol = 0;
                    if (nRow) pRow = atomicAdd(&a.keyCursor[qid], nRow);
                    if (nCol) pCol = atomicAdd(&a.keyCursor[cidL], nCol);
                    // positions come from the counted offsets; a run past the end
                    // would mean the two passes disagree
                    const bool okRow = (uint64_t)pRow + nRow <= a.capacity;
                    const bool okCol = (uint64_t)pCol + nCol <= a.capacity;
                    if (!okRow || !okCol) atomicMax(&a.stat[3], 1ULL);
                    // Two ways to write a block's pairs, chosen per direction:
                    // dense blocks: one warp iteration per non-empty run (the
                    // run is written coalesced by the lanes holding its members);
                    // sparse blocks: every lane stages its own short run in shared
                    // memory, then the warp copies the staged pairs out in order.
                    const uint32_t nr = okRow ? nRow : 0u, nc = okCol ? nCol : 0u;
                    uint32_t incR = nr, incC = nc;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const uint32_t yr = __shfl_up_sync(0xffffffffu, incR, o);
                        const uint32_t yc = __shfl_up_sync(0xffffffffu, incC, o);
                        if (lane >= (uint32_t)o) { incR += yr; incC += yc; }
                    }
                    const uint32_t totR = __shfl_sync(0xffffffffu, incR, 31);
                    const uint32_t totC = __shfl_sync(0xffffffffu, incC, 31);
                    uint32_t* const sS = stSlot[FILL ? warp : 0];
                    uint32_t* const sK = stKey[FILL ? warp : 0];
                    uint32_t* const sV = stVal[FILL ? warp : 0];
                    // row direction: key = this lane's query, values = candidates
                    if (totR <= EMIT_STAGE) {
                        uint32_t m = okRow ? rowMask : 0u, at = incR - nr, slot = pRow;
                        while (m) {
                            const int b = __ffs(m) - 1;
                            m &= m - 1;
                            sS[at] = slot++;
                            sK[at] = qid;
                            sV[at] = candId[jb + b];
                            at++;
                        }
                        __syncwarp();
                        for (uint32_t e = lane; e < totR; e += 32) {
                            a.outKey[sS[e]] = (int32_t)sK[e];
                            a.outVal[sS[e]] = (int32_t)sV[e];
                        }
                        __syncwarp();
                    } else {
                        uint32_t live = __ballot_sync(0xffffffffu, nr != 0);
                        while (live) {
                            const int L = __ffs(live) - 1;
                            live &= live - 1;
                            const uint32_t base = __shfl_sync(0xffffffffu, pRow, L);
                            const uint32_t key = __shfl_sync(0xffffffffu, qid, L);
                            const bool h = (rowT >> L) & 1u;
                            const uint32_t b = __ballot_sync(0xffffffffu, h);
                            if (h) {
                                const uint32_t at = base + __popc(b & ltmask);
                                a.outKey[at] = (int32_t)key;
                                a.outVal[at] = (int32_t)cidL;
                            }
                        }
                    }
                    // column direction: key = this lane's candidate, values = queries
                    if (totC <= EMIT_STAGE) {
                        uint32_t m = okCol ? mirT : 0u, at = incC - nc, slot = pCol;
                        while (m) {
                            const int b = __ffs(m) - 1;
                            m &= m - 1;
                            sS[at] = slot++;
                            sK[at] = cidL;
                            sV[at] = qIdS[warp * 32 + b];
                            at++;
                        }
                        __syncwarp();
                        for (uint32_t e = lane; e < totC; e += 32) {
                            a.outKey[sS[e]] = (int32_t)sK[e];
                            a.outVal[sS[e]] = (int32_t)sV[e];
                        }
                        __syncwarp();
                    } else {
                        uint32_t live = __ballot_sync(0xffffffffu, nc != 0);
                        while (live) {
                            const int j = __ffs(live) - 1;
                            live &= live - 1;
                            const uint32_t base = __shfl_sync(0xffffffffu, pCol, j);
                            const uint32_t key = __shfl_sync(0xffffffffu, cidL, j);
                            const bool h = (mirRow >> j) & 1u;
                            const uint32_t b = __ballot_sync(0xffffffffu, h);
                            if (h) {
                                const uint32_t at = base + __popc(b & ltmask);
                                a.outKey[at] = (int32_t)key;
                                a.outVal[at] = (int32_t)qid;
                            }
                        }
                    }
                } else {
                    rowCount += __popc(rowMask);
                    if (sym) colCnt[warp][jb + lane] += __popc(transpose32(mirRow, lane));
                }
            }
            if (!FILL && sym) {
                __syncthreads();
                uint32_t local = 0;
                for (uint32_t j = tid; j < nIn; j += SJ_CTA) {
                    uint32_t tot = 0;
#pragma unroll
                    for (int w = 0; w < NW; w++) { tot += colCnt[w][j]; colCnt[w][j] = 0; }
                    if (tot) { atomicAdd(&a.keyCount[candId[j]], tot); local += tot; }
                }
                if (local) atomicAdd(&taskPairs, (unsigned long long)local);
            }
        }
        if (!FILL) {
            if (rowCount) {
                atomicAdd(&a.keyCount[qid], rowCount);
                atomicAdd(&taskPairs, (unsigned long long)rowCount);
            }
        }
        // ---- statistics
        unsigned long long e = evals, r = refined;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            e += __shfl_xor_sync(0xffffffffu, e, o);
            r += __shfl_xor_sync(0xffffffffu, r, o);
        }
        if (FILL && lane == 0) {   // each task is filled exactly once
            if (e) atomicAdd(&a.stat[0], e);
            if (r) atomicAdd(&a.stat[1], r);
        }
        if (!FILL) {
            __syncthreads();
            if (tid == 0) {
                if (taskPairs) {
                    atomicAdd(&a.stat[2], taskPairs);
                    if (a.batchPairs) atomicAdd(a.batchPairs, taskPairs);
                }
                if (a.taskHits) a.taskHits[t] = (uint32_t)min(taskPairs, 0xffffffffULL);
            }
        }
    }
}

template <int DP>
cudaError_t launch_dp(const sj_join_args &a, const sj_grid_dev &g, int fill, int fp32, int queue, int numSM,
                      cudaStream_t s)
{
    uint32_t nt = a.taskEnd - a.taskBegin;
    if (nt == 0) return cudaSuccess;
    // persistent queue: one full wave of resident CTAs
    static int perSM[2][2] = {{0, 0}, {0, 0}};
    int &occ = perSM[fp32 ? 1 : 0][fill ? 1 : 0];
    if (queue && occ == 0) {
        int b = 0;
        if (fp32) {
            if (fill) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_join<DP, true, true>, SJ_CTA, 0);
            else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_join<DP, true, false>, SJ_CTA, 0);
        } else {
            if (fill) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_join<DP, false, true>, SJ_CTA, 0);
            else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_join<DP, false, false>, SJ_CTA, 0);
        }
        occ = b > 0 ? b : 4;
    }
    unsigned grid = queue ? (unsigned)(numSM * occ) : nt;
    if (queue && grid > nt) grid = nt;
    if (fp32) {
        if (fill) k_join<DP, true, true><<<grid, SJ_CTA, 0, s>>>(a, g, queue);
        else k_join<DP, true, false><<<grid, SJ_CTA, 0, s>>>(a, g, queue);
    } else {
        if (fill) k_join<DP, false, true><<<grid, SJ_CTA, 0, s>>>(a, g, queue);
        else k_join<DP, false, false><<<grid, SJ_CTA, 0, s>>>(a, g, queue);
    }
    sj_note_launch();
    return cudaGetLastError();
}

}  // namespace

cudaError_t sj_launch_join(const sj_join_args &a, const sj_grid_dev &g, int fill, int fp32, int queue, int numSM,
                           cudaStream_t s)
{
    switch (g.Dp) {
    case 1: return launch_dp<1>(a, g, fill, fp32, queue, numSM, s);
    case 2: return launch_dp<2>(a, g, fill, fp32, queue, numSM, s);
    case 3: return launch_dp<3>(a, g, fill, fp32, queue, numSM, s);
    case 4: return launch_dp<4>(a, g, fill, fp32, queue, numSM, s);
    case 6: return launch_dp<6>(a, g, fill, fp32, queue, numSM, s);
    case 8: return launch_dp<8>(a, g, fill, fp32, queue, numSM, s);
    case 12: return launch_dp<12>(a, g, fill, fp32, queue, numSM, s);
    case 16: return launch_dp<16>(a, g, fill, fp32, queue, numSM, s);
    }
    return cudaErrorInvalidValue;
}
