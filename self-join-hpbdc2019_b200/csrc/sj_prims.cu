// Device primitives: exclusive scan (u32), stable LSD radix sort, pair-set hash.
#include <atomic>

#include "sj_internal.h"

namespace {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;   // 2048 elements per block

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Block-wide exclusive scan of one value per thread; returns the exclusive
// prefix and writes the block total to *total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *total)
{
    __shared__ uint32_t warpSums[SCAN_THREADS / 32];
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane_id() >= (uint32_t)o) x += y;
    }
    const int w = threadIdx.x >> 5;
    if (lane_id() == 31) warpSums[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = (lane_id() < SCAN_THREADS / 32) ? warpSums[lane_id()] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane_id() >= (uint32_t)o) s += y;
        }
        if (lane_id() < SCAN_THREADS / 32) warpSums[lane_id()] = s;   // inclusive warp prefixes
    }
    __syncthreads();
    uint32_t warpPrefix = (w > 0) ? warpSums[w - 1] : 0u;
    *total = warpSums[SCAN_THREADS / 32 - 1];
    __syncthreads();
    return warpPrefix + x - v;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const uint32_t *__restrict__ in, uint64_t n,
                                                              uint32_t *__restrict__ sums)
{
    uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE;
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        uint64_t idx = base + (uint64_t)i * SCAN_THREADS + threadIdx.x;
        if (idx < n) s += in[idx];
    }
    uint32_t tot;
    block_exclusive_scan(s, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Scans one tile per block; adds the block's offset from `blockOffsets`
// (nullptr for a single-block scan, which also writes the grand total).
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tile(const uint32_t *in, uint32_t *out, uint64_t n,
                                                            const uint32_t *__restrict__ blockOffsets,
                                                            uint32_t *total_dev, uint32_t *zeroIn)
{
    uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        uint64_t idx = base + i;
        v[i] = (idx < n) ? in[idx] : 0u;
        s += v[i];
    }
    if (zeroIn) {
#pragma unroll
        for (int i = 0; i < SCAN_ITEMS; i++)
            if (base + i < n) zeroIn[base + i] = 0u;
    }
    uint32_t tot;
    uint32_t pre = block_exclusive_scan(s, &tot);
    uint32_t off = (blockOffsets ? blockOffsets[blockIdx.x] : 0u) + pre;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        uint64_t idx = base + i;
        if (idx < n) out[idx] = off;
        off += v[i];
    }
    if (!blockOffsets && total_dev && threadIdx.x == 0) *total_dev = tot;
}

// Second pass of the two-launch scan: each block finds its offset by summing
// the tile sums of all blocks before it (read from L2; used while the tile
// count is small), then scans its tile; the last block writes the total.
constexpr uint64_t SCAN_LOOKUP_MAX_TILES = 4096;

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tile_lookup(const uint32_t *in, uint32_t *out, uint64_t n,
                                                                   const uint32_t *__restrict__ sums,
                                                                   uint32_t *total_dev, uint32_t *zeroIn)
{
    uint32_t part = 0;
    for (uint32_t b = threadIdx.x; b < blockIdx.x; b += SCAN_THREADS) part += sums[b];
    uint32_t blockOff;   // sum of all earlier tiles (the block total of the parts)
    block_exclusive_scan(part, &blockOff);
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        const uint64_t idx = base + i;
        v[i] = (idx < n) ? in[idx] : 0u;
        sum += v[i];
    }
    if (zeroIn) {
#pragma unroll
        for (int i = 0; i < SCAN_ITEMS; i++)
            if (base + i < n) zeroIn[base + i] = 0u;
    }
    uint32_t tot;
    uint32_t off = blockOff + block_exclusive_scan(sum, &tot);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        const uint64_t idx = base + i;
        if (idx < n) out[idx] = off;
        off += v[i];
    }
    if (total_dev && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *total_dev = blockOff + tot;
}

__global__ void k_scan_total(const uint32_t *scannedSums, const uint32_t *sums, uint64_t nb, uint32_t *total_dev)
{
    if (threadIdx.x == 0 && blockIdx.x == 0 && total_dev) *total_dev = scannedSums[nb - 1] + sums[nb - 1];
}

uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

size_t scan_temp_elems(uint64_t n)
{
    size_t e = 0;
    while (n > (uint64_t)SCAN_TILE) {
        uint64_t nb = ceil_div(n, SCAN_TILE);
        e += 2 * nb;
        n = nb;
    }
    return e + 1;
}

cudaError_t scan_rec(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *temp, uint32_t *total_dev,
                     cudaStream_t s, uint32_t *zeroIn = nullptr)
{
    if (n == 0) {
        if (total_dev) return cudaMemsetAsync(total_dev, 0, sizeof(uint32_t), s);
        return cudaSuccess;
    }
    if (n <= (uint64_t)SCAN_TILE) {
        k_scan_tile<<<1, SCAN_THREADS, 0, s>>>(in, out, n, nullptr, total_dev, zeroIn); sj_note_launch();
        return cudaGetLastError();
    }
    uint64_t nb = ceil_div(n, SCAN_TILE);
    uint32_t *sums = temp, *scanned = temp + nb;
    k_scan_reduce<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, sums); sj_note_launch();
    if (nb <= SCAN_LOOKUP_MAX_TILES) {
        k_scan_tile_lookup<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, out, n, sums, total_dev, zeroIn);
        sj_note_launch();
        return cudaGetLastError();
    }
    cudaError_t e = scan_rec(sums, scanned, nb, temp + 2 * nb, nullptr, s);
    if (e != cudaSuccess) return e;
    if (total_dev) {
        k_scan_total<<<1, 32, 0, s>>>(scanned, sums, nb, total_dev);
        sj_note_launch();
    }
    k_scan_tile<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, out, n, scanned, nullptr, zeroIn); sj_note_launch();
    return cudaGetLastError();
}

// ------------------------------------------------------------- radix sort --

constexpr int RS_THREADS = 256;
constexpr int RS_CHUNKS = 8;                       // chunks of RS_THREADS keys per tile
constexpr int RS_TILE = RS_THREADS * RS_CHUNKS;    // 2048 keys per block
constexpr int RS_WARPS = RS_THREADS / 32;

template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_radix_hist(const K *__restrict__ keys, uint64_t n, int shift,
                                                           uint32_t *__restrict__ blockHist, uint32_t nb)
{
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
#pragma unroll
    for (int c = 0; c < RS_CHUNKS; c++) {
        uint64_t idx = base + (uint64_t)c * RS_THREADS + threadIdx.x;
        if (idx < n) atomicAdd(&h[(uint32_t)(keys[idx] >> shift) & 255u], 1u);
    }
    __syncthreads();
    blockHist[(uint64_t)threadIdx.x * nb + blockIdx.x] = h[threadIdx.x];   // digit-major
}

// Stable scatter: keys keep their input order within a digit.
template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_radix_scatter(const K *__restrict__ keysIn,
                                                              const uint32_t *__restrict__ valsIn,
                                                              K *__restrict__ keysOut, uint32_t *__restrict__ valsOut,
                                                              uint64_t n, int shift,
                                                              const uint32_t *__restrict__ digitOffsets, uint32_t nb)
{
    __shared__ uint32_t base[256];
    __shared__ uint32_t warpCnt[RS_WARPS][256];
    base[threadIdx.x] = digitOffsets[(uint64_t)threadIdx.x * nb + blockIdx.x];
#pragma unroll
    for (int w = 0; w < RS_WARPS; w++) warpCnt[w][threadIdx.x] = 0;
    __syncthreads();
    const int w = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t ltmask = (1u << lane) - 1u;
    uint64_t tileBase = (uint64_t)blockIdx.x * RS_TILE;
    for (int c = 0; c < RS_CHUNKS; c++) {
        uint64_t idx = tileBase + (uint64_t)c * RS_THREADS + threadIdx.x;
        bool valid = idx < n;
        K key = valid ? keysIn[idx] : (K)0;
        uint32_t val = valid ? valsIn[idx] : 0u;
        uint32_t d = valid ? ((uint32_t)(key >> shift) & 255u) : 256u;
        uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t rank = __popc(peers & ltmask);
        if (valid && rank == 0) warpCnt[w][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            uint32_t pre = 0;
            for (int v = 0; v < w; v++) pre += warpCnt[v][d];
            uint32_t pos = base[d] + pre + rank;
            keysOut[pos] = key;
            valsOut[pos] = val;
        }
        __syncthreads();
        uint32_t add = 0;
#pragma unroll
        for (int v = 0; v < RS_WARPS; v++) { add += warpCnt[v][threadIdx.x]; warpCnt[v][threadIdx.x] = 0; }
        base[threadIdx.x] += add;
        __syncthreads();
    }
}

template <typename K>
cudaError_t radix_sort(K *keys, uint32_t *vals, K *keysAlt, uint32_t *valsAlt, uint64_t n, int bits, void *temp,
                       int *resultInAlt, cudaStream_t s)
{
    *resultInAlt = 0;
    if (n <= 1 || bits <= 0) return cudaSuccess;
    uint32_t nb = (uint32_t)ceil_div(n, RS_TILE);
    uint32_t *hist = (uint32_t *)temp;
    uint32_t *scanTemp = hist + (size_t)256 * nb;
    K *kin = keys, *kout = keysAlt;
    uint32_t *vin = vals, *vout = valsAlt;
    int alt = 0;
    for (int shift = 0; shift < bits; shift += 8) {
        k_radix_hist<K><<<nb, RS_THREADS, 0, s>>>(kin, n, shift, hist, nb); sj_note_launch();
        cudaError_t e = scan_rec(hist, hist, (uint64_t)256 * nb, scanTemp, nullptr, s);
        if (e != cudaSuccess) return e;
        k_radix_scatter<K><<<nb, RS_THREADS, 0, s>>>(kin, vin, kout, vout, n, shift, hist, nb); sj_note_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        K *tk = kin; kin = kout; kout = tk;
        uint32_t *tv = vin; vin = vout; vout = tv;
        alt ^= 1;
    }
    *resultInAlt = alt;
    return cudaSuccess;
}

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z)
{
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

__global__ void __launch_bounds__(256) k_hash_pairs(const int32_t *__restrict__ key, const int32_t *__restrict__ val,
                                                    uint64_t m, unsigned long long *out)
{
    unsigned long long h = 0;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        unsigned long long z = ((unsigned long long)(uint32_t)key[i] << 32) | (uint32_t)val[i];
        h += splitmix64(z);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
    __shared__ unsigned long long ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = h;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += ws[w];
        atomicAdd(out, t);
    }
}

// Keys of a batch: key k owns slots [excl[k], excl[k+1]) (excl[n] = *total).
// A warp takes 32 consecutive keys and writes each key's run with all lanes,
// 128 contiguous bytes per store.  Runs longer than EXP_LONG slots (a dense
// key can own a million slots of one batch) are queued instead and written by
// whole CTAs in k_expand_long, so one warp never holds up the launch.
constexpr uint32_t EXP_LONG = 16384;

__device__ __forceinline__ void write_run(int32_t *__restrict__ outKey, uint32_t s0, uint32_t e0, int32_t key,
                                          uint32_t t, uint32_t nt)
{
    // up to 3 single slots to a 16-byte boundary, 16-byte stores, the rest
    const uint32_t a = min((s0 + 3u) & ~3u, e0);
    const uint32_t b = a + ((e0 - a) & ~3u);
    if (t < a - s0) outKey[s0 + t] = key;
    const int4 kv = make_int4(key, key, key, key);
    for (uint32_t pos = a + 4 * t; pos < b; pos += 4 * nt) *reinterpret_cast<int4 *>(outKey + pos) = kv;
    if (t < e0 - b) outKey[b + t] = key;
}

__global__ void __launch_bounds__(256) k_expand_keys(const uint32_t *__restrict__ excl,
                                                     const uint32_t *__restrict__ total, uint64_t n,
                                                     int32_t *__restrict__ outKey,
                                                     const unsigned long long *__restrict__ batchPairs, uint64_t cap,
                                                     uint4 *__restrict__ longRuns, uint32_t longCap,
                                                     uint32_t *__restrict__ longCount)
{
    if (*batchPairs > cap) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t k0 = ((uint64_t)blockIdx.x * 256 + (threadIdx.x & ~31u));
    if (k0 >= n) return;
    const uint64_t k = k0 + lane;
    const uint32_t tot = *total;
    const uint32_t st = k < n ? excl[k] : tot;
    const uint32_t en = k + 1 < n ? excl[k + 1] : tot;
    uint32_t live = __ballot_sync(0xffffffffu, en > st);
    while (live) {
        const int i = __ffs(live) - 1;
        live &= live - 1;
        const uint32_t s0 = __shfl_sync(0xffffffffu, st, i);
        const uint32_t e0 = __shfl_sync(0xffffffffu, en, i);
        const int32_t key = (int32_t)(k0 + i);
        if (e0 - s0 > EXP_LONG) {
            uint32_t j = 0;
            if (lane == 0) j = atomicAdd(longCount, 1u);
            j = __shfl_sync(0xffffffffu, j, 0);
            if (j < longCap) {
                if (lane == 0) longRuns[j] = make_uint4((uint32_t)key, s0, e0, 0u);
                continue;
            }
        }
        write_run(outKey, s0, e0, key, lane, 32);
    }
}

// The queued long runs, one CTA per run at a time.
__global__ void __launch_bounds__(256) k_expand_long(int32_t *__restrict__ outKey,
                                                     const unsigned long long *__restrict__ batchPairs, uint64_t cap,
                                                     const uint4 *__restrict__ longRuns, uint32_t longCap,
                                                     const uint32_t *__restrict__ longCount)
{
    if (*batchPairs > cap) return;
    const uint32_t cnt = min(*longCount, longCap);
    for (uint32_t j = blockIdx.x; j < cnt; j += gridDim.x) {
        const uint4 r = longRuns[j];
        write_run(outKey, r.y, r.z, (int32_t)r.x, threadIdx.x, blockDim.x);
    }
}

// The consumer fold of a device-resident batch, with the key array written in
// the same pass.  Key k owns slots [excl[k], excl[k+1]) (excl[n] = *total).
// The slots are cut into chunks of FOLD_CHUNK; k_fold_chunk_keys records the
// key at each chunk's first slot (one thread per key writes the chunks its run
// starts), and in k_fold a warp takes a chunk in rounds of 128 slots, lane L
// holding slots 4L .. 4L+3 of the round.  The warp keeps a window of 32
// consecutive keys, one per lane (its run start and end); each lane whose
// non-empty run starts inside the round marks key + 1 at that slot in a
// per-warp shared array, and an inclusive max-scan over the round (4 slots per
// lane, then across the lanes, seeded with the key carried from the previous
// round) gives every slot its key, since keys ascend with the slots.  When the
// window's runs end inside the round, the window jumps to the key whose run
// holds the first slot past it (a 32-ary search over the run starts, which
// steps over stretches of empty runs: keys are point ids).  The values are
// read back in 16-byte streaming loads, the keys stored in 16-byte streaming
// stores, and splitmix64(key << 32 | value) is added to the set hash.  Every
// chunk is the same size, so the work is balanced whatever the run lengths.
// 8 bytes per pair move, against 12 for a key expansion followed by a fold
// that reads both arrays.  Skipped when the batch's count exceeds cap.
constexpr uint32_t FOLD_CHUNK = 4096;
constexpr int FOLD_THREADS = 256;
constexpr int FOLD_CTAS_PER_SM = 6;   // resident k_fold CTAs per SM (the register budget allows 6)

__global__ void __launch_bounds__(256) k_fold_chunk_keys(const uint32_t *__restrict__ excl,
                                                         const uint32_t *__restrict__ total, uint64_t n,
                                                         const unsigned long long *__restrict__ batchPairs,
                                                         uint64_t cap, uint32_t *__restrict__ chunkKey)
{
    if (*batchPairs > cap) return;
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t tot = *total;
    const uint32_t st = excl[k];
    const uint32_t en = k + 1 < n ? excl[k + 1] : tot;
    for (uint32_t c = (st + FOLD_CHUNK - 1) / FOLD_CHUNK; (uint64_t)c * FOLD_CHUNK < en; c++) chunkKey[c] = (uint32_t)k;
}

__global__ void __launch_bounds__(FOLD_THREADS, FOLD_CTAS_PER_SM) k_fold(const uint32_t *__restrict__ excl,
                                                       const uint32_t *__restrict__ total, uint64_t n,
                                                       const int32_t *__restrict__ val, int32_t *__restrict__ outKey,
                                                       const unsigned long long *__restrict__ batchPairs,
                                                       uint64_t cap, const uint32_t *__restrict__ chunkKey,
                                                       unsigned long long *__restrict__ hashOut)
{
    __shared__ __align__(16) uint32_t marks[FOLD_THREADS / 32][128];   // per warp: key + 1 at each run start
    if (*batchPairs > cap) return;
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t *const mk = marks[threadIdx.x >> 5];
    const uint32_t tot = *total;
    const uint32_t nChunks = (tot + FOLD_CHUNK - 1) / FOLD_CHUNK;
    const uint32_t warpsAll = (gridDim.x * blockDim.x) >> 5;
    unsigned long long h = 0;
    *reinterpret_cast<uint4 *>(mk + 4 * lane) = make_uint4(0u, 0u, 0u, 0u);
    // run start and end of key kk (both the total for kk >= n)
    auto runStart = [&](uint64_t kk) -> uint32_t { return kk < n ? excl[kk] : tot; };
    auto runEnd = [&](uint64_t kk) -> uint32_t { return kk + 1 < n ? excl[kk + 1] : tot; };
    for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < nChunks; c += warpsAll) {
        const uint32_t p0 = c * FOLD_CHUNK, p1 = min(p0 + FOLD_CHUNK, tot);
        uint64_t k = chunkKey[c];         // its run holds slot p0
        uint32_t carry = (uint32_t)k;     // key of the round's slots before its first marked start
        uint32_t S = runStart(k + lane), R = runEnd(k + lane);
        for (uint32_t base = p0; base < p1; base += 128) {
            const uint32_t lim = min(base + 128u, p1);
            const uint32_t p = base + 4 * lane;
            const uint32_t cnt = p < lim ? min(4u, lim - p) : 0u;   // this lane's slots: p .. p + cnt - 1
            int4 v = make_int4(0, 0, 0, 0);   // the values, loaded while the keys are found
            if (cnt == 4) {
                v = __ldcs(reinterpret_cast<const int4 *>(val + p));
            } else {
                if (cnt > 0) v.x = __ldcs(val + p);
                if (cnt > 1) v.y = __ldcs(val + p + 1);
                if (cnt > 2) v.z = __ldcs(val + p + 2);
            }
            __syncwarp();   // every lane has cleared its slots of the previous round
            for (;;) {
                if (R > S && S >= base && S < lim) mk[S - base] = (uint32_t)(k + lane) + 1u;
                const uint32_t Rlast = __shfl_sync(0xffffffffu, R, 31);
                if (Rlast >= lim || k + 32 >= n) break;   // warp-uniform
                // the window's runs end inside the round: jump to the largest
                // key k' with excl[k'] <= Rlast (the keys in between have empty
                // runs).  Invariant: excl[lo] <= Rlast, and hi == n or
                // excl[hi] > Rlast.
                uint64_t lo = k + 32, hi = n;
                while (hi - lo > 1) {
                    const uint64_t step = (hi - lo + 31) / 32;
                    const uint64_t probe = lo + (uint64_t)(lane + 1) * step;
                    const bool ok = probe < hi && excl[probe] <= Rlast;
                    const uint32_t cntOk = __popc(__ballot_sync(0xffffffffu, ok));   // a prefix of the lanes
                    lo += (uint64_t)cntOk * step;
                    hi = min(hi, lo + step);
                }
                k = lo;
                S = runStart(k + lane);
                R = runEnd(k + lane);
            }
            __syncwarp();
            const uint4 m = *reinterpret_cast<const uint4 *>(mk + 4 * lane);
            *reinterpret_cast<uint4 *>(mk + 4 * lane) = make_uint4(0u, 0u, 0u, 0u);
            // keys ascend with the slots: each slot's key + 1 is the largest mark
            // at or before it (or the carried key + 1)
            const uint32_t m1 = max(m.x, m.y), m2 = max(m1, m.z), m3 = max(m2, m.w);
            uint32_t x = m3;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= (uint32_t)o) x = max(x, y);
            }
            uint32_t pre = __shfl_up_sync(0xffffffffu, x, 1);
            pre = max(lane ? pre : 0u, carry + 1u);
            const uint32_t k0 = max(pre, m.x) - 1u, k1 = max(pre, m1) - 1u, k2 = max(pre, m2) - 1u,
                           k3 = max(pre, m3) - 1u;
            carry = __shfl_sync(0xffffffffu, k3, 31);
            if (cnt == 4) {
                __stcs(reinterpret_cast<int4 *>(outKey + p), make_int4((int)k0, (int)k1, (int)k2, (int)k3));
            } else {
                if (cnt > 0) outKey[p] = (int32_t)k0;
                if (cnt > 1) outKey[p + 1] = (int32_t)k1;
                if (cnt > 2) outKey[p + 2] = (int32_t)k2;
            }
            if (cnt > 0) h += splitmix64(((unsigned long long)k0 << 32) | (uint32_t)v.x);
            if (cnt > 1) h += splitmix64(((unsigned long long)k1 << 32) | (uint32_t)v.y);
            if (cnt > 2) h += splitmix64(((unsigned long long)k2 << 32) | (uint32_t)v.z);
            if (cnt > 3) h += splitmix64(((unsigned long long)k3 << 32) | (uint32_t)v.w);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
    __shared__ unsigned long long ws[FOLD_THREADS / 32];
    if (lane == 0) ws[threadIdx.x >> 5] = h;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < FOLD_THREADS / 32; w++) t += ws[w];
        if (t) atomicAdd(hashOut, t);
    }
}

// Appends a batch to a device CSR neighbour table: key k's run
// [start[k], start[k+1]) of vals (start[n] = *total) goes to
// cols[rowPtr[k] + fill[k] ...] and fill[k] grows by its length.  A warp takes
// 32 consecutive keys and copies each run with all lanes.  A run that would
// pass its row's end or the caller's capacity is not written and sets *err.
__global__ void __launch_bounds__(256) k_csr_append(const uint32_t *__restrict__ start,
                                                    const uint32_t *__restrict__ total, uint64_t n,
                                                    const int32_t *__restrict__ vals,
                                                    const uint64_t *__restrict__ rowPtr, uint32_t *__restrict__ fill,
                                                    int32_t *__restrict__ cols, uint64_t colsCap,
                                                    unsigned long long *__restrict__ err)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t k0 = ((uint64_t)blockIdx.x * 256 + (threadIdx.x & ~31u));
    if (k0 >= n) return;
    const uint64_t k = k0 + lane;
    const uint32_t tot = *total;
    const uint32_t st = k < n ? start[k] : tot;
    const uint32_t en = k + 1 < n ? start[k + 1] : tot;
    unsigned long long dst = 0;
    bool ok = true;
    if (en > st) {
        const uint64_t rowEnd = rowPtr[k + 1];
        dst = rowPtr[k] + fill[k];
        ok = dst + (en - st) <= rowEnd && rowEnd <= colsCap;
        if (ok) fill[k] += en - st;
        else atomicMax(err, 1ULL);
    }
    uint32_t live = __ballot_sync(0xffffffffu, en > st && ok);
    while (live) {
        const int i = __ffs(live) - 1;
        live &= live - 1;
        const uint32_t s0 = __shfl_sync(0xffffffffu, st, i);
        const uint32_t e0 = __shfl_sync(0xffffffffu, en, i);
        const unsigned long long d0 = __shfl_sync(0xffffffffu, dst, i);
        for (uint32_t p = lane; p < e0 - s0; p += 32) cols[d0 + p] = vals[s0 + p];
    }
}

__global__ void __launch_bounds__(256) k_u32_to_f32(const uint32_t *__restrict__ in, uint64_t n,
                                                    float *__restrict__ out)
{
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)in[i];
}

}  // namespace

cudaError_t sj_u32_to_f32(const uint32_t *in, uint64_t n, float *out, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    k_u32_to_f32<<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(in, n, out);
    sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_expand_keys(const uint32_t *excl, const uint32_t *total, uint64_t n, int32_t *outKey,
                           const unsigned long long *batchPairs, uint64_t cap, void *longRuns, uint32_t longCap,
                           uint32_t *longCount, int numSM, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(longCount, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    k_expand_keys<<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(excl, total, n, outKey, batchPairs, cap,
                                                            (uint4 *)longRuns, longCap, longCount);
    sj_note_launch();
    k_expand_long<<<(unsigned)(numSM * 8), 256, 0, s>>>(outKey, batchPairs, cap, (const uint4 *)longRuns, longCap,
                                                       longCount);
    sj_note_launch();
    return cudaGetLastError();
}

size_t sj_fold_chunks(uint64_t cap) { return (size_t)(cap / FOLD_CHUNK) + 2; }

cudaError_t sj_fold(const uint32_t *excl, const uint32_t *total, uint64_t n, const int32_t *val, int32_t *outKey,
                    const unsigned long long *batchPairs, uint64_t cap, uint32_t *chunkKey,
                    unsigned long long *hashOut, int numSM, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    k_fold_chunk_keys<<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(excl, total, n, batchPairs, cap, chunkKey);
    sj_note_launch();
    k_fold<<<(unsigned)(numSM * FOLD_CTAS_PER_SM), FOLD_THREADS, 0, s>>>(excl, total, n, val, outKey, batchPairs, cap, chunkKey, hashOut);
    sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_csr_append(const uint32_t *start, const uint32_t *total, uint64_t n, const int32_t *vals,
                          const uint64_t *rowPtr, uint32_t *fill, int32_t *cols, uint64_t colsCap,
                          unsigned long long *err, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    k_csr_append<<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(start, total, n, vals, rowPtr, fill, cols, colsCap, err);
    sj_note_launch();
    return cudaGetLastError();
}

size_t sj_expand_long_slots(uint64_t cap) { return (size_t)(cap / EXP_LONG) + 1; }

static std::atomic<unsigned long long> g_launches{0};
void sj_note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
unsigned long long sj_launch_total() { return g_launches.load(std::memory_order_relaxed); }

size_t sj_scan_temp_bytes(uint64_t n) { return scan_temp_elems(n) * sizeof(uint32_t); }

cudaError_t sj_exclusive_scan_u32(const uint32_t *in, uint32_t *out, uint64_t n, void *temp, uint32_t *total_dev,
                                  cudaStream_t s)
{
    return scan_rec(in, out, n, (uint32_t *)temp, total_dev, s);
}

cudaError_t sj_exclusive_scan_u32_clear(uint32_t *in, uint32_t *out, uint64_t n, void *temp, uint32_t *total_dev,
                                        cudaStream_t s)
{
    return scan_rec(in, out, n, (uint32_t *)temp, total_dev, s, in);
}

size_t sj_radix_temp_bytes(uint64_t n)
{
    uint64_t nb = ceil_div(n ? n : 1, RS_TILE);
    return (size_t)256 * nb * sizeof(uint32_t) + sj_scan_temp_bytes((uint64_t)256 * nb);
}

cudaError_t sj_radix_sort_u64_u32(uint64_t *keys, uint32_t *vals, uint64_t *keysAlt, uint32_t *valsAlt, uint64_t n,
                                  int bits, void *temp, int *resultInAlt, cudaStream_t s)
{
    return radix_sort<uint64_t>(keys, vals, keysAlt, valsAlt, n, bits, temp, resultInAlt, s);
}

cudaError_t sj_radix_sort_u32_u32(uint32_t *keys, uint32_t *vals, uint32_t *keysAlt, uint32_t *valsAlt, uint64_t n,
                                  int bits, void *temp, int *resultInAlt, cudaStream_t s)
{
    return radix_sort<uint32_t>(keys, vals, keysAlt, valsAlt, n, bits, temp, resultInAlt, s);
}

cudaError_t sj_hash_pairs(const int32_t *key, const int32_t *val, uint64_t m, unsigned long long *hashOut,
                          cudaStream_t s)
{
    if (m == 0) return cudaSuccess;
    uint64_t blocks = ceil_div(m, 256 * 16);
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_hash_pairs<<<(unsigned)blocks, 256, 0, s>>>(key, val, m, hashOut); sj_note_launch();
    return cudaGetLastError();
}
