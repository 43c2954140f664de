// The emission pass: pairs from the count pass's hit masks.
//
// The count pass (sj_join.cu) leaves, per task, every query's hit mask per
// block of 32 stream positions (row masks), the transposed masks of symmetric
// tasks (column masks: per block and group of 32 queries, candidate j's query
// bits) and every query's row count; the exclusive scan of the per-key counts
// gives each key's slot range in the batch buffer.  This pass writes the
// values (the keys come from sj_expand_keys):
//
//   rows    : key = query, values = candidates.  One warp per query and chunk
//             of 64 blocks (2048 stream positions): the query's 64 words (two
//             per lane, contiguous), a warp scan of their popcounts, the set
//             bits decoded into chunk positions in shared memory, then the
//             candidate ids copied out as one contiguous run.  One reservation
//             (atomicAdd on the key's cursor) per query and task.
//   columns : key = candidate, values = queries (symmetric tasks).  One warp
//             per block: lane j reads candidate j's words of eight query
//             groups, one reservation per candidate and group batch, decode,
//             copy-out through shared memory.
//
// Decoding (a per-lane loop over set bits, whose trip count is the busiest
// lane's) only writes small indices; the loads and global stores run in the
// balanced copy-out.  Runs wider than the shared buffer are written directly
// by the whole warp.  No distance is evaluated here, so the pass is identical
// for both precisions.
#include "sj_internal.h"

#include <atomic>

namespace {

constexpr int EW = 128;                    // threads per emission CTA
constexpr int ENW = EW / 32;
constexpr int CHUNK = 2048;                // stream positions (64 blocks) whose candidate ids are held at once
constexpr int EM_CAP = 1024;               // staged entries per warp
constexpr int GB = 8;                      // query groups (of 32) per column batch
constexpr int MAXQ = SJ_CTA * 4;           // largest query tile
static_assert(SJ_SLOTS_F32 <= 4 && SJ_SLOTS_F64 <= 4, "query tiles are at most 4 * SJ_CTA points");
constexpr uint32_t NO_SLOT = 0xffffffffu;  // reservation refused (past capacity)

struct EmitSmem {
    uint32_t segStart[SJ_MAX_SEG];
    uint32_t segPre[SJ_MAX_SEG + 1];
    uint32_t candS[CHUNK];
    uint32_t qIdS[MAXQ];
    uint32_t rowPos[MAXQ];
    uint32_t colRun[ENW][2][32]; // column batch: per lane, run start and first staged entry
    uint16_t stQ[ENW][EM_CAP];   // row entries: chunk position; column entries: lane << 9 | query index
    uint32_t scanTmp[ENW];
    uint32_t curTask;
};

// Appends base + (index of each set bit of m) to buf[k...]; returns the new k.
__device__ __forceinline__ uint32_t decode_bits(uint32_t m, uint32_t base, uint16_t *buf, uint32_t k)
{
    while (m) {
        const uint32_t b = 31u - __clz(m);
        m ^= 1u << b;
        buf[k++] = (uint16_t)(base + b);
    }
    return k;
}

__device__ __forceinline__ uint32_t warp_excl_scan(uint32_t n, uint32_t lane, uint32_t &total)
{
    uint32_t x = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    total = __shfl_sync(0xffffffffu, x, 31);
    return x - n;
}

__global__ void __launch_bounds__(EW) k_emit(sj_join_args a, int queue)
{
    __shared__ EmitSmem sm;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    const uint32_t warp = tid >> 5;
    const uint32_t ltmask = (1u << lane) - 1u;
    // a batch whose count exceeded the output buffer is re-planned by the host
    if (a.batchPairs && *a.batchPairs > a.capacity) {
        if (tid == 0 && blockIdx.x == 0) atomicMax(&a.stat[5], 1ULL);
        return;
    }
    uint32_t iter = 0;
    for (;;) {
        __syncthreads();
        if (tid == 0)
            sm.curTask = queue ? (a.taskBegin + atomicAdd(a.queueHead, 1u)) : (a.taskBegin + blockIdx.x + iter);
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
        const uint32_t qc = task.qCount;

        // ---- segment table (as the count pass builds it)
        constexpr int PER = (SJ_MAX_SEG + EW - 1) / EW;
        uint32_t locLen[PER];
        uint32_t mySum = 0;
#pragma unroll
        for (int r = 0; r < PER; r++) {
            const uint32_t s = tid * PER + r;
            uint32_t len = 0;
            if (s < nSeg) {
                const uint32_t gs = task.segBase + s;
                uint32_t st0, en;
                if (gs == 0) {
                    st0 = sym ? task.qBegin : aStart;
                    en = aEnd;
                } else {
                    const uint32_t b = a.nbrCell[nbrBase + gs - 1];
                    st0 = a.cellStart[b];
                    en = a.cellStart[b + 1];
                }
                sm.segStart[s] = st0;
                len = en - st0;
            }
            locLen[r] = len;
            mySum += len;
        }
        {
            uint32_t dummy;
            const uint32_t ex = warp_excl_scan(mySum, lane, dummy);
            if (lane == 31) sm.scanTmp[warp] = ex + mySum;
            __syncthreads();
            uint32_t run = ex;
            for (uint32_t w = 0; w < warp; w++) run += sm.scanTmp[w];
#pragma unroll
            for (int r = 0; r < PER; r++) {
                const uint32_t s = tid * PER + r;
                if (s <= nSeg) sm.segPre[s] = run;
                run += locLen[r];
            }
            if (tid == EW - 1) sm.segPre[nSeg] = run;
        }
        for (uint32_t qi = tid; qi < qc; qi += EW) sm.qIdS[qi] = a.ids[task.qBegin + qi];
        __syncthreads();
        const uint32_t L = min(task.sEnd, sm.segPre[nSeg]) - task.sBegin;
        const uint32_t nBlk = (L + 31) / 32;
        const uint32_t *const masks = a.masks + (a.maskOff[t] - a.maskOff[a.taskBegin]);
        const uint32_t *const colMasks = a.colMasks + (a.colOff[t] - a.colOff[a.taskBegin]);
        const uint32_t *const rows = a.rowCnt + (a.rowOff[t] - a.rowOff[a.taskBegin]);

        // ---- one row reservation per query and task
        for (uint32_t qi = tid; qi < qc; qi += EW) {
            const uint32_t c = rows[qi];
            uint32_t pos = 0;
            if (c) {
                pos = atomicAdd(&a.keyCursor[sm.qIdS[qi]], c);
                if ((uint64_t)pos + c > a.capacity) {
                    atomicMax(&a.stat[3], 1ULL);
                    pos = NO_SLOT;
                }
            }
            sm.rowPos[qi] = pos;
        }

        const uint32_t nG = (qc + 31) / 32;
        uint16_t *const stQ = sm.stQ[warp];
        for (uint32_t c0 = 0; c0 < L; c0 += CHUNK) {
            const uint32_t nC = min((uint32_t)CHUNK, L - c0);
            __syncthreads();
            for (uint32_t j = tid; j < nC; j += EW) {
                const uint32_t s = task.sBegin + c0 + j;
                uint32_t lo = 0, hi = nSeg;   // largest seg with segPre[seg] <= s
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (sm.segPre[mid] <= s) lo = mid; else hi = mid;
                }
                sm.candS[j] = a.ids[sm.segStart[lo] + (s - sm.segPre[lo])];
            }
            __syncthreads();
            const uint32_t nb = (nC + 31) / 32;
            const uint32_t b0 = c0 / 32;   // first block of the chunk (a multiple of 64)

            // ---- rows: one query per warp, its words of the chunk contiguous
            // (the next query's words are loaded while this one is written)
            const uint64_t chunkBase = sj_row_mask_index(b0, 0, qc, nBlk);
            uint32_t n0 = 0, n1 = 0;
            if (warp < qc) {
                const uint32_t *wq = masks + chunkBase + (uint64_t)warp * nb;
                n0 = lane < nb ? wq[lane] : 0u;
                n1 = lane + 32 < nb ? wq[lane + 32] : 0u;
            }
            for (uint32_t qi = warp; qi < qc; qi += ENW) {
                const uint32_t w0 = n0, w1 = n1;
                if (qi + ENW < qc) {
                    const uint32_t *wq = masks + chunkBase + (uint64_t)(qi + ENW) * nb;
                    n0 = lane < nb ? wq[lane] : 0u;
                    n1 = lane + 32 < nb ? wq[lane + 32] : 0u;
                }
                uint32_t T;
                const uint32_t ex = warp_excl_scan(__popc(w0) + __popc(w1), lane, T);
                if (T == 0) continue;
                const uint32_t pos0 = sm.rowPos[qi];
                __syncwarp();
                if (lane == 0) sm.rowPos[qi] = (pos0 == NO_SLOT) ? NO_SLOT : pos0 + T;
                if (pos0 == NO_SLOT) continue;
                if (T <= (uint32_t)EM_CAP) {
                    uint32_t k = decode_bits(w0, lane * 32, stQ, ex);
                    decode_bits(w1, (lane + 32) * 32, stQ, k);
                    __syncwarp();
                    for (uint32_t e = lane; e < T; e += 32) a.outVal[pos0 + e] = (int32_t)sm.candS[stQ[e]];
                    __syncwarp();
                } else {
                    uint32_t off = 0;
                    for (uint32_t bb = 0; bb < nb; bb++) {
                        const uint32_t word = __shfl_sync(0xffffffffu, bb < 32 ? w0 : w1, bb & 31);
                        const bool h = (word >> lane) & 1u;
                        const uint32_t bal = __ballot_sync(0xffffffffu, h);
                        if (h) a.outVal[pos0 + off + __popc(bal & ltmask)] = (int32_t)sm.candS[bb * 32 + lane];
                        off += __popc(bal);
                    }
                }
            }
            if (!sym) continue;

            // ---- columns: one block of 32 candidates per warp, lane j = candidate j;
            // one reservation per candidate and task over all query groups, the
            // groups then written GB at a time
            for (uint32_t bb = warp; bb < nb; bb += ENW) {
                const uint32_t key = sm.candS[bb * 32 + lane];
                const uint32_t *const wb = colMasks + (uint64_t)(b0 + bb) * nG * 32 + lane;
                uint32_t n = 0;
                for (uint32_t g = 0; g < nG; g++) n += __popc(wb[g * 32]);
                // the reservation's result is first needed by the copy-out below,
                // so its latency overlaps the first batch's loads and decode
                const uint32_t base0 = n ? atomicAdd(&a.keyCursor[key], n) : 0u;
                uint32_t base = base0;
                bool checked = false;
                for (uint32_t g0 = 0; g0 < nG; g0 += GB) {
                    const uint32_t gn = min((uint32_t)GB, nG - g0);
                    uint32_t cw[GB];
                    uint32_t m = 0;
#pragma unroll
                    for (int gg = 0; gg < GB; gg++) {
                        cw[gg] = (uint32_t)gg < gn ? wb[(g0 + gg) * 32] : 0u;
                        m += __popc(cw[gg]);
                    }
                    uint32_t T;
                    const uint32_t ex = warp_excl_scan(m, lane, T);
                    if (T == 0) continue;
                    const bool staged = T <= (uint32_t)EM_CAP;
                    if (staged) {
                        uint32_t k = ex;
#pragma unroll
                        for (int gg = 0; gg < GB; gg++) k = decode_bits(cw[gg], (lane << 9) | ((g0 + gg) * 32), stQ, k);
                    }
                    if (!checked) {   // first use of the reservation
                        checked = true;
                        const bool bad = n && (uint64_t)base0 + n > a.capacity;
                        if (__any_sync(0xffffffffu, bad)) {
                            if (bad) atomicMax(&a.stat[3], 1ULL);
                            break;
                        }
                    }
                    if (staged) {
                        // staged entries [ex, ex + m) of lane L go to its run from base
                        sm.colRun[warp][0][lane] = base;
                        sm.colRun[warp][1][lane] = ex;
                        __syncwarp();
                        for (uint32_t e = lane; e < T; e += 32) {
                            const uint32_t ent = stQ[e];
                            const uint32_t owner = ent >> 9;
                            a.outVal[sm.colRun[warp][0][owner] + (e - sm.colRun[warp][1][owner])] =
                                (int32_t)sm.qIdS[ent & 511u];
                        }
                        __syncwarp();
                    } else {
                        uint32_t off = 0;
#pragma unroll
                        for (int gg = 0; gg < GB; gg++) {
                            uint32_t live = __ballot_sync(0xffffffffu, cw[gg] != 0);
                            while (live) {
                                const int Lk = __ffs(live) - 1;
                                live &= live - 1;
                                const uint32_t word = __shfl_sync(0xffffffffu, cw[gg], Lk);
                                const uint32_t pL = __shfl_sync(0xffffffffu, base + off, Lk);
                                const bool h = (word >> lane) & 1u;
                                const uint32_t bal = __ballot_sync(0xffffffffu, h);
                                if (h) a.outVal[pL + __popc(bal & ltmask)] = (int32_t)sm.qIdS[(g0 + gg) * 32 + lane];
                            }
                            off += __popc(cw[gg]);
                        }
                    }
                    base += m;
                }
            }
        }
    }
}

int emit_occupancy()
{
    constexpr int MAXDEV = 64;
    static std::atomic<int> occ[MAXDEV];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= MAXDEV) dev = 0;
    int o = occ[dev].load();
    if (o == 0) {
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_emit, EW, 0);
        o = b > 0 ? b : 1;
        occ[dev].store(o);
    }
    return o;
}

}  // namespace

cudaError_t sj_launch_emit(const sj_join_args &a, int queue, int numSM, cudaStream_t s)
{
    const uint32_t nt = a.taskEnd - a.taskBegin;
    if (nt == 0) return cudaSuccess;
    unsigned grid = queue ? (unsigned)(numSM * emit_occupancy()) : nt;
    if (queue && grid > nt) grid = nt;
    k_emit<<<grid, EW, 0, s>>>(a, queue);
    sj_note_launch();
    return cudaGetLastError();
}
