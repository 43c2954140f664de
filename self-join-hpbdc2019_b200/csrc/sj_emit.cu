// The emission pass: (key, value) pairs from the count pass's hit masks.
//
// The count pass (sj_join.cu) leaves, per task of the batch:
//   * every query's row hit mask per block of 32 stream positions, laid out
//     [chunk of 64 blocks][query][block in chunk];
//   * for a symmetric task the transposed (column) masks: per block and group
//     of 32 queries, candidate j's query bits, laid out [block][group][j];
//   * per query the offset of the task's row run inside the query's key run,
//     and per stream position the candidate's point id and the offset of its
//     column run inside the candidate's key run.  Both offsets are the key's
//     count just before the count pass added that run, so the runs of one key
//     tile the key's range exactly.
// With keyStart (the exclusive scan of the per-key counts) every pair's slot
// is keyStart[key] + run offset + rank inside the run: no atomics, and keys
// come out ascending with each key's values contiguous -- the order
// thrust::sort_by_key gives the reference (GPU.cu:2336) -- without a sort.
//
// Work is cut into warp units that any warp of any CTA takes from a counter:
//   row unit    (task, group of 32 queries): the group's words of a chunk are
//               contiguous; a window of 64 words (lane L holds words L and
//               32 + L; one window spans several queries when the task has
//               few blocks) is popcounted and scanned (both halves' counts
//               packed in one 32-bit scan), its set bits are decoded into
//               shared memory as 16-bit (query, stream position) entries in
//               slot order, and the warp copies the entries out: consecutive
//               entries of one query go to consecutive slots, so the stores
//               are coalesced.
//   column unit (symmetric task, block of 32 stream positions): lane j is
//               candidate j; per query group its word is decoded lane-major
//               and copied out the same way, each lane's run continuing across
//               groups.
// A window without any set bit costs one ballot.  Measured on one B200 and
// not kept: two query groups per column window (c3 emission +5 %), and row
// windows aligned to one query's words when a chunk has >= 32 blocks (c3
// +13 %, no gain elsewhere).
// Only the values are written here: the keys of a batch are its key runs in
// key order, which sj_expand_keys writes sequentially (the emission's writes
// land at scattered run positions, which HBM absorbs at a fraction of its
// sequential rate, so writing the keys there too would cost more than the
// separate sequential pass).  Every mask word is checked against its task's
// sizes before it is decoded (bits past the stream end or for queries past the
// tile, which a consistent count pass never sets, are dropped and raise an
// error flag that the host reports), so the decoded entries need no checks.  No distance is evaluated, so the pass is the same for both
// precisions.
#include "sj_internal.h"

#include <atomic>

namespace {

constexpr int EW = 256;             // threads per emission CTA (independent warps)
constexpr int ENW = EW / 32;
constexpr int EM_CAP = 2048;        // staged entries per warp: one window of 64 words x 32 bits
constexpr uint32_t FULL = 0xffffffffu;
#ifndef SJ_EMIT_UNROLL
#define SJ_EMIT_UNROLL 4
#endif
constexpr int CO = SJ_EMIT_UNROLL;  // copy-out entries per lane whose loads are in flight together
// Mask windows (rows) / query groups (columns) whose words are loaded ahead of
// the one being decoded: the emission reads the hit masks once, in order, so
// its loads can run this far ahead of the decode.
#ifndef SJ_EMIT_PF
#define SJ_EMIT_PF 4
#endif
constexpr int PF = SJ_EMIT_PF;
#ifndef SJ_EMIT_MINB
#define SJ_EMIT_MINB 4
#endif
// 1: a CTA takes EW/32 consecutive units per round (one atomic), 0: each warp
// takes units on its own
#ifndef SJ_EMIT_COOP
#define SJ_EMIT_COOP 0
#endif

struct WarpSmem {
    uint16_t ent[EM_CAP];   // staged entries in slot order: rows (query << 11) | chunk position,
                            // columns (lane << 5) | query bit
    uint32_t base[32];      // slot of entry 0 of the window for each query (rows) / lane (columns)
    uint32_t start[32];     // rows: slot of each query's first pair of the chunk
};

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t x, uint32_t lane)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    return x;
}

// Index of the highest set bit of m (m != 0).
__device__ __forceinline__ uint32_t top_bit(uint32_t m)
{
    uint32_t b;
    asm("bfind.u32 %0, %1;" : "=r"(b) : "r"(m));
    return b;
}

// Writes tag | (index of each set bit of m) to buf[k .. k + n), lowest bit
// first, where n = popc(m).  The bits are taken highest first and the entries
// filled from the end, two per round (a lone last bit on its own).
__device__ __forceinline__ void decode_bits(uint32_t m, uint32_t n, uint32_t tag, uint16_t *buf, uint32_t k)
{
    uint16_t *p = buf + k + n;
    for (; n >= 2; n -= 2) {
        const uint32_t b0 = top_bit(m);
        m ^= 1u << b0;
        const uint32_t b1 = top_bit(m);
        m ^= 1u << b1;
        p[-1] = (uint16_t)(tag | b0);
        p[-2] = (uint16_t)(tag | b1);
        p -= 2;
    }
    if (n) p[-1] = (uint16_t)(tag | top_bit(m));
}

// decode_bits for two words at once (two independent chains of bit scans):
// word a's n_a entries go to buf[ka ..), word b's to buf[kb ..).
__device__ __forceinline__ void decode_bits2(uint32_t ma, uint32_t na, uint32_t tagA, uint32_t ka, uint32_t mb,
                                             uint32_t nb, uint32_t tagB, uint32_t kb, uint16_t *buf)
{
    uint16_t *pa = buf + ka + na, *pb = buf + kb + nb;
    while (na >= 2 || nb >= 2) {
        if (na >= 2) {
            const uint32_t b0 = top_bit(ma);
            ma ^= 1u << b0;
            const uint32_t b1 = top_bit(ma);
            ma ^= 1u << b1;
            pa[-1] = (uint16_t)(tagA | b0);
            pa[-2] = (uint16_t)(tagA | b1);
            pa -= 2;
            na -= 2;
        }
        if (nb >= 2) {
            const uint32_t b0 = top_bit(mb);
            mb ^= 1u << b0;
            const uint32_t b1 = top_bit(mb);
            mb ^= 1u << b1;
            pb[-1] = (uint16_t)(tagB | b0);
            pb[-2] = (uint16_t)(tagB | b1);
            pb -= 2;
            nb -= 2;
        }
    }
    if (na) pa[-1] = (uint16_t)(tagA | top_bit(ma));
    if (nb) pb[-1] = (uint16_t)(tagB | top_bit(mb));
}

// Stores one value.  FITS: the caller has shown that every slot of the window
// is below the capacity; otherwise each slot is checked.
template <bool FITS>
__device__ __forceinline__ void put(const sj_join_args &a, uint32_t slot, int32_t val)
{
    if (FITS || slot < a.capacity) {
        a.outVal[slot] = val;
    } else {
        atomicMax(&a.stat[3], 1ULL);
    }
}

// Copies the window's T staged entries out: entry e goes to slot
// slotOf(ent[e], e) with value src[srcOf(ent[e])].  Whole rounds of 32 * CO
// entries issue all their loads before any store; the rest goes 32 at a time,
// so a window never pays for more than 31 idle lane slots.
template <bool FITS, class SlotOf, class SrcOf>
__device__ __forceinline__ void copy_out(const sj_join_args &a, const uint16_t *ent, uint32_t T,
                                         const uint32_t *__restrict__ src, uint32_t lane, SlotOf slotOf,
                                         SrcOf srcOf)
{
    uint32_t e0 = 0;
    for (; e0 + 32 * CO <= T; e0 += 32 * CO) {
        uint32_t slot[CO], pos[CO], val[CO];
#pragma unroll
        for (int i = 0; i < CO; i++) {
            const uint32_t e = e0 + 32 * i + lane;
            const uint32_t en = ent[e];
            pos[i] = srcOf(en);
            slot[i] = slotOf(en, e);
        }
#pragma unroll
        for (int i = 0; i < CO; i++) val[i] = __ldg(src + pos[i]);
#pragma unroll
        for (int i = 0; i < CO; i++) put<FITS>(a, slot[i], (int32_t)val[i]);
    }
    for (; e0 < T; e0 += 32) {
        const uint32_t e = e0 + lane;
        if (e < T) {
            const uint32_t en = ent[e];
            put<FITS>(a, slotOf(en, e), (int32_t)__ldg(src + srcOf(en)));
        }
    }
}

// Fields of the task an emission unit belongs to.
struct UnitTask {
    uint32_t t, qBegin, qc, L;
};

// Bits of a row word whose block starts at stream position p0 (< L) past the
// stream end are never set by a consistent count pass: drop them and flag it.
__device__ __forceinline__ uint32_t stream_checked(const sj_join_args &a, uint32_t word, uint32_t p0, uint32_t L)
{
    const uint32_t rem = L - p0;
    if (rem < 32u && (word >> rem) != 0u) {
        atomicMax(&a.stat[6], 1ULL);
        word &= (1u << rem) - 1u;
    }
    return word;
}

// Row unit: queries 32g .. 32g+nq-1 of task u.t (key = query, value = candidate).
__device__ __forceinline__ void emit_rows(const sj_join_args &a, const UnitTask &u, uint32_t g, WarpSmem &w,
                                          uint32_t lane)
{
    const uint32_t qc = u.qc;
    const uint32_t q0 = g * 32;
    const uint32_t nq = min(32u, qc - q0);
    const uint32_t nBlk = (u.L + 31) / 32;
    const uint32_t *const masks = a.masks + (a.maskOff[u.t] - a.maskOff[a.taskBegin]);
    const uint32_t *const cid = a.candId + (a.candOff[u.t] - a.candOff[a.taskBegin]);
    const uint32_t *const rel = a.rowRel + (a.rowOff[u.t] - a.rowOff[a.taskBegin]);
    uint32_t next = 0;   // lane q: slot of query q's next pair
    __syncwarp();        // the previous unit is done with the warp's shared memory
    if (lane < nq) {
        const uint32_t qid = a.ids[u.qBegin + q0 + lane];
        next = a.keyStart[qid] + rel[q0 + lane];
    }
    for (uint32_t c0 = 0; c0 < nBlk; c0 += 64) {
        const uint32_t cb = min(64u, nBlk - c0);          // blocks of this chunk
        const uint32_t nw = nq * cb;                      // the group's words of this chunk
        const uint32_t *const wq = masks + (uint64_t)c0 * qc + (uint64_t)q0 * cb;
        const uint32_t *const pcid = cid + c0 * 32;
        const auto srcOf = [](uint32_t en) { return en & 0x7ffu; };
        // floor(f / cb) = (f * magic) >> 32 for f < 2^26 (error < 2^-6 <= 1/cb)
        const uint64_t magic = ((1ULL << 32) + cb - 1) / cb;
        __syncwarp();
        w.start[lane] = next;
        uint32_t carry = 0;   // entries of earlier windows of this chunk
        // a window is 64 words: lane L holds words L and 32 + L; the words of
        // the next PF windows are in flight while this one is written
        uint32_t pw[PF][2];
#pragma unroll
        for (int k = 0; k < PF; k++) {
            const uint32_t f = 64u * k + lane;
            pw[k][0] = f < nw ? __ldg(wq + f) : 0u;
            pw[k][1] = f + 32 < nw ? __ldg(wq + f + 32) : 0u;
        }
        for (uint32_t ws = 0; ws < nw; ws += 64) {
            const uint32_t fa = ws + lane, fb = fa + 32;
            uint32_t wa = pw[0][0], wb = pw[0][1];
#pragma unroll
            for (int k = 0; k + 1 < PF; k++) {
                pw[k][0] = pw[k + 1][0];
                pw[k][1] = pw[k + 1][1];
            }
            {
                const uint32_t f = fa + 64u * PF;
                pw[PF - 1][0] = f < nw ? __ldg(wq + f) : 0u;
                pw[PF - 1][1] = f + 32 < nw ? __ldg(wq + f + 32) : 0u;
            }
            const uint32_t qa = (uint32_t)(((uint64_t)fa * magic) >> 32);
            const uint32_t qb = (uint32_t)(((uint64_t)fb * magic) >> 32);
            const uint32_t ra = fa - qa * cb, rb = fb - qb * cb;   // block of each word in the chunk
            // words past the group's end are zero; a word's block is inside the stream
            if (wa) wa = stream_checked(a, wa, (c0 + ra) * 32u, u.L);
            if (wb) wb = stream_checked(a, wb, (c0 + rb) * 32u, u.L);
            const uint32_t ca = __popc(wa), cbt = __popc(wb);
            if (__ballot_sync(FULL, ca | cbt) == 0) {
                // no pair in the window: only the bases of queries that start in it
                __syncwarp();
                if (fa < nw && ra == 0) w.base[qa] = w.start[qa] - carry;
                if (fb < nw && rb == 0) w.base[qb] = w.start[qb] - carry;
                continue;
            }
            // one scan of both halves' counts (each total <= 1024 fits 16 bits):
            // word fa's entries start at exA, word fb's at TA + exB
            const uint32_t incl = warp_incl_scan(ca | (cbt << 16), lane);
            const uint32_t tot = __shfl_sync(FULL, incl, 31);
            const uint32_t TA = tot & 0xffffu, T = TA + (tot >> 16);
            const uint32_t exA = (incl & 0xffffu) - ca, exB = TA + (incl >> 16) - cbt;
            __syncwarp();   // the previous window's copy-out is done with ent / base
            // a query's first word: base = its chunk start slot minus its flat prefix
            if (fa < nw && ra == 0) w.base[qa] = w.start[qa] - (carry + exA);
            if (fb < nw && rb == 0) w.base[qb] = w.start[qb] - (carry + exB);
            decode_bits2(wa, ca, (qa << 11) | (ra << 5), exA, wb, cbt, (qb << 11) | (rb << 5), exB, w.ent);
            __syncwarp();
            // copy-out.  Every entry is valid by construction (words of queries
            // < nq, bits inside the stream).
            const uint32_t qf = __shfl_sync(FULL, qa, 0);
            if (ws - qf * cb + min(64u, nw - ws) <= cb) {
                // the whole window is one query's: one base for every entry
                const uint32_t B = w.base[qf] + carry;
                const auto slotOf = [B](uint32_t, uint32_t e) { return B + e; };
                if ((uint64_t)B + T <= a.capacity) copy_out<true>(a, w.ent, T, pcid, lane, slotOf, srcOf);
                else copy_out<false>(a, w.ent, T, pcid, lane, slotOf, srcOf);
            } else {
                const uint32_t *const base = w.base;
                const uint32_t cy = carry;
                // each word's last entry has the largest slot of its run
                const bool fits = (ca == 0 || (uint64_t)base[qa] + cy + exA + ca <= a.capacity) &&
                                  (cbt == 0 || (uint64_t)base[qb] + cy + exB + cbt <= a.capacity);
                const auto slotOf = [base, cy](uint32_t en, uint32_t e) { return base[en >> 11] + cy + e; };
                if (__all_sync(FULL, fits)) copy_out<true>(a, w.ent, T, pcid, lane, slotOf, srcOf);
                else copy_out<false>(a, w.ent, T, pcid, lane, slotOf, srcOf);
            }
            carry += T;
        }
        __syncwarp();
        // query q's slot after this chunk: its base plus the flat prefix at its
        // last word's end (the next query's start prefix, or the chunk total)
        if (lane < nq) next = w.base[lane] + ((lane + 1 < nq) ? (w.start[lane + 1] - w.base[lane + 1]) : carry);
    }
}

// Column unit: stream positions 32b .. 32b+31 of symmetric task u.t (key =
// candidate, value = query).  A window is one query group: lane j's word of it.
__device__ __forceinline__ void emit_cols(const sj_join_args &a, const UnitTask &u, uint32_t b, WarpSmem &w,
                                          uint32_t lane)
{
    const uint32_t nG = (u.qc + 31) / 32;
    const uint32_t s = b * 32 + lane;
    const uint64_t rec = a.candOff[u.t] - a.candOff[a.taskBegin];
    // words of positions past the stream end are zero (the count pass masks them)
    const uint32_t *const cw = a.colMasks + (a.colOff[u.t] - a.colOff[a.taskBegin]) + (uint64_t)b * nG * 32 + lane;
    const uint32_t *const qids = a.ids + u.qBegin;
    uint32_t slot = 0;
    __syncwarp();        // the previous unit is done with the warp's shared memory
    if (s < u.L) {
        slot = a.keyStart[a.candId[rec + s]] + a.candRel[rec + s];
    }
    // the words of the next PF query groups are in flight while one is written
    uint32_t pw[PF];
#pragma unroll
    for (int k = 0; k < PF; k++) pw[k] = (uint32_t)k < nG ? __ldg(cw + k * 32) : 0u;
    for (uint32_t g = 0; g < nG; g++) {
        uint32_t cur = pw[0];
#pragma unroll
        for (int k = 0; k + 1 < PF; k++) pw[k] = pw[k + 1];
        pw[PF - 1] = g + PF < nG ? __ldg(cw + (uint64_t)(g + PF) * 32) : 0u;
        {
            // positions past the stream end and queries past the tile have no
            // bits in a consistent count pass
            const uint32_t nq = u.qc - g * 32;
            const uint32_t valid = s >= u.L ? 0u : (nq >= 32u ? FULL : (1u << nq) - 1u);
            if (cur & ~valid) {
                atomicMax(&a.stat[6], 1ULL);
                cur &= valid;
            }
        }
        const uint32_t cnt = __popc(cur);
        if (__ballot_sync(FULL, cnt) == 0) continue;   // warp-uniform
        const uint32_t incl = warp_incl_scan(cnt, lane);
        const uint32_t T = __shfl_sync(FULL, incl, 31);
        const uint32_t ex = incl - cnt;
        __syncwarp();
        w.base[lane] = slot - ex;   // lane L's entries [ex_L, ex_L + cnt_L) go to slot_L onwards
        decode_bits(cur, cnt, lane << 5, w.ent, ex);
        __syncwarp();
        const uint32_t *const base = w.base;
        const auto slotOf = [base](uint32_t en, uint32_t e) { return base[en >> 5] + e; };
        const auto srcOf = [](uint32_t en) { return en & 31u; };
        if (__all_sync(FULL, (uint64_t)slot + cnt <= a.capacity))
            copy_out<true>(a, w.ent, T, qids + g * 32, lane, slotOf, srcOf);
        else
            copy_out<false>(a, w.ent, T, qids + g * 32, lane, slotOf, srcOf);
        slot += cnt;
    }
}

__global__ void __launch_bounds__(EW, SJ_EMIT_MINB) k_emit(sj_join_args a)
{
    __shared__ WarpSmem smem[ENW];
    const uint32_t lane = threadIdx.x & 31u;
    WarpSmem &w = smem[threadIdx.x >> 5];
    // a batch whose count exceeded the output buffer is re-planned by the host
    if (a.batchPairs && *a.batchPairs > a.capacity) {
        if (threadIdx.x == 0 && blockIdx.x == 0) atomicMax(&a.stat[5], 1ULL);
        return;
    }
    const uint64_t u0 = a.unitOff[a.taskBegin];
    const uint32_t nUnits = (uint32_t)(a.unitOff[a.taskEnd] - u0);
#if SJ_EMIT_COOP
    // the CTA's warps take consecutive units (mostly of one task), so the
    // task's candidate ids and query ids are shared through L1
    __shared__ uint32_t ctaBase;
#endif
    for (;;) {
#if SJ_EMIT_COOP
        __syncthreads();   // every warp is done with the previous round's units
        if (threadIdx.x == 0) ctaBase = atomicAdd(a.queueHead, (uint32_t)ENW);
        __syncthreads();
        if (ctaBase >= nUnits) break;   // uniform over the CTA
        const uint32_t un = ctaBase + (threadIdx.x >> 5);
        if (un >= nUnits) continue;
#else
        uint32_t un = 0;
        if (lane == 0) un = atomicAdd(a.queueHead, 1u);
        un = __shfl_sync(FULL, un, 0);
        if (un >= nUnits) break;
#endif
        // the unit's task: the last t with unitOff[t] - u0 <= un
        uint32_t lo = a.taskBegin, hi = a.taskEnd;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (a.unitOff[mid] - u0 <= un) lo = mid; else hi = mid;
        }
        if (a.taskHits && a.taskHits[lo] == 0) continue;   // the count pass found no pair in this task
        const sj_task *const tp = a.tasks + lo;
        UnitTask u;
        u.t = lo;
        u.qBegin = tp->qBegin;
        u.qc = tp->qCount;
        u.L = tp->sEnd - tp->sBegin;
        const bool sym = (tp->flags & SJ_TASK_SYM) != 0;
        const uint32_t k = un - (uint32_t)(a.unitOff[lo] - u0);
        const uint32_t nG = (u.qc + 31) / 32;
        if (k < nG) emit_rows(a, u, k, w, lane);
        else if (sym) emit_cols(a, u, k - nG, w, lane);
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

cudaError_t sj_launch_emit(const sj_join_args &a, int numSM, int maxCtasPerSM, cudaStream_t s)
{
    if (a.taskEnd == a.taskBegin) return cudaSuccess;
    int perSM = emit_occupancy();
    if (maxCtasPerSM > 0 && maxCtasPerSM < perSM) perSM = maxCtasPerSM;
    k_emit<<<(unsigned)(numSM * perSM), EW, 0, s>>>(a);
    sj_note_launch();
    return cudaGetLastError();
}
