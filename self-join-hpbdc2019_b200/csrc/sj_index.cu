// Grid-index construction on the device.
//
// Restates the reference's host build (main.cu:240-503) as data-parallel
// kernels: per-dimension min/max, FP64 cell coordinates and linear ids, a
// stable radix sort by linear id (point ids stay ascending inside a cell, as
// the reference's push_back order leaves them), run-length cell boundaries, and
// a cell-sorted copy of the coordinates for coalesced staging in the join.
#include "sj_internal.h"

namespace {

// Order-preserving map from double to uint64 (for atomicMin/atomicMax).
__device__ __forceinline__ unsigned long long ord_encode(double x)
{
    unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ULL);
}

__global__ void __launch_bounds__(256) k_minmax(const double *__restrict__ pts, uint64_t n, int D,
                                                unsigned long long *__restrict__ mm)
{
    // mm[2*j] = encoded min of dim j, mm[2*j+1] = encoded max, mm[2*D] = non-finite flag
    __shared__ unsigned long long smin[SJ_MAX_DIM], smax[SJ_MAX_DIM];
    __shared__ int sbad;
    if (threadIdx.x < SJ_MAX_DIM) { smin[threadIdx.x] = ~0ULL; smax[threadIdx.x] = 0ULL; }
    if (threadIdx.x == 0) sbad = 0;
    __syncthreads();
    unsigned long long lmin[SJ_MAX_DIM], lmax[SJ_MAX_DIM];
    for (int j = 0; j < D; j++) { lmin[j] = ~0ULL; lmax[j] = 0ULL; }
    int bad = 0;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        for (int j = 0; j < D; j++) {
            double x = pts[i * D + j];
            if (!isfinite(x)) bad = 1;
            unsigned long long e = ord_encode(x);
            lmin[j] = e < lmin[j] ? e : lmin[j];
            lmax[j] = e > lmax[j] ? e : lmax[j];
        }
    }
    for (int j = 0; j < D; j++) {
        unsigned long long a = lmin[j], b = lmax[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long x = __shfl_xor_sync(0xffffffffu, a, o);
            unsigned long long y = __shfl_xor_sync(0xffffffffu, b, o);
            a = x < a ? x : a;
            b = y > b ? y : b;
        }
        if ((threadIdx.x & 31) == 0) { atomicMin(&smin[j], a); atomicMax(&smax[j], b); }
    }
    if (bad) sbad = 1;
    __syncthreads();
    if (threadIdx.x < (unsigned)D) {
        atomicMin(&mm[2 * threadIdx.x], smin[threadIdx.x]);
        atomicMax(&mm[2 * threadIdx.x + 1], smax[threadIdx.x]);
    }
    if (threadIdx.x == 0 && sbad) atomicMax(&mm[2 * D], 1ULL);
}

__global__ void k_minmax_init(unsigned long long *mm, int D)
{
    int j = threadIdx.x;
    if (j < D) { mm[2 * j] = ~0ULL; mm[2 * j + 1] = 0ULL; }
    if (j == 0) mm[2 * D] = 0ULL;
}

__global__ void k_minmax_decode(unsigned long long *mm, int D)
{
    int j = threadIdx.x;
    if (j < 2 * D) {
        unsigned long long u = mm[j];
        u = (u >> 63) ? (u & 0x7fffffffffffffffULL) : ~u;
        mm[j] = u;  // now the raw bits of the double
    }
}

// Cell coordinate (main.cu:294, kernel.cu:1457) and linear id (main.cu:423-439).
// A coordinate at or past its dimension's cell count (which the grid's eps
// margins rule out up to rounding) would alias another cell's linear id: it
// sets *outOfGrid, and the host refuses the index.
__global__ void __launch_bounds__(256) k_cell_keys(const double *__restrict__ pts, uint64_t n, sj_grid_dev g,
                                                   uint64_t *__restrict__ keys, uint32_t *__restrict__ vals,
                                                   uint32_t *__restrict__ outOfGrid)
{
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned long long lid = 0, mul = 1;
    for (int j = 0; j < g.k; j++) {
        double x = pts[i * g.D + j];
        unsigned c = __double2uint_rz(__ddiv_rn(__dsub_rn(x, g.minArr[j]), g.eps));
        if (c >= g.nCells[j]) atomicOr(outOfGrid, 1u);
        lid += (unsigned long long)c * mul;
        mul *= g.nCells[j];
    }
    keys[i] = lid;
    vals[i] = (uint32_t)i;
}

__global__ void __launch_bounds__(256) k_cell_flags(const uint64_t *__restrict__ keys, uint64_t n,
                                                    uint32_t *__restrict__ flags)
{
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// flags were scanned in place: excl[i] = number of cell starts before i.
__global__ void __launch_bounds__(256) k_cell_build(const uint64_t *__restrict__ keys,
                                                    const uint32_t *__restrict__ excl, uint64_t n,
                                                    uint32_t *__restrict__ cellStart, uint64_t *__restrict__ cellLid)
{
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    bool start = (i == 0) || (keys[i] != keys[i - 1]);
    if (start) {
        uint32_t c = excl[i];
        cellStart[c] = (uint32_t)i;
        cellLid[c] = keys[i];
    }
}

__global__ void __launch_bounds__(256) k_gather(const double *__restrict__ pts, const uint32_t *__restrict__ ids,
                                                uint64_t n, int D, int Dp, double *__restrict__ xs)
{
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * (uint64_t)Dp) return;
    uint64_t pos = t / Dp;
    int l = (int)(t - pos * Dp);
    xs[t] = (l < D) ? pts[(uint64_t)ids[pos] * D + l] : 0.0;
}

__global__ void __launch_bounds__(256) k_cell_coords(const uint64_t *__restrict__ cellLid, uint32_t nCells,
                                                     sj_grid_dev g, uint32_t *__restrict__ coord)
{
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nCells) return;
    unsigned long long lid = cellLid[c];
    for (int j = 0; j < g.k; j++) {
        coord[(uint64_t)c * g.k + j] = (uint32_t)(lid % g.nCells[j]);
        lid /= g.nCells[j];
    }
}

inline unsigned blocks_for(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t sj_launch_minmax(const double *pts, uint64_t n, int D, double *minmax_dev, cudaStream_t s)
{
    unsigned long long *mm = (unsigned long long *)minmax_dev;
    k_minmax_init<<<1, 64, 0, s>>>(mm, D); sj_note_launch();
    uint64_t blocks = (n + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks == 0) blocks = 1;
    k_minmax<<<(unsigned)blocks, 256, 0, s>>>(pts, n, D, mm); sj_note_launch();
    k_minmax_decode<<<1, 64, 0, s>>>(mm, D); sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_launch_cell_keys(const double *pts, uint64_t n, sj_grid_dev g, uint64_t *keys, uint32_t *vals,
                                uint32_t *outOfGrid, cudaStream_t s)
{
    k_cell_keys<<<blocks_for(n, 256), 256, 0, s>>>(pts, n, g, keys, vals, outOfGrid); sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_launch_cell_flags(const uint64_t *keys, uint64_t n, uint32_t *flags, cudaStream_t s)
{
    k_cell_flags<<<blocks_for(n, 256), 256, 0, s>>>(keys, n, flags); sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_launch_cell_build(const uint64_t *keys, const uint32_t *cellIdxExcl, uint64_t n, uint32_t *cellStart,
                                 uint64_t *cellLid, cudaStream_t s)
{
    k_cell_build<<<blocks_for(n, 256), 256, 0, s>>>(keys, cellIdxExcl, n, cellStart, cellLid); sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_launch_gather(const double *pts, const uint32_t *ids, uint64_t n, int D, int Dp, double *xs,
                             cudaStream_t s)
{
    k_gather<<<blocks_for(n * (uint64_t)Dp, 256), 256, 0, s>>>(pts, ids, n, D, Dp, xs); sj_note_launch();
    return cudaGetLastError();
}

cudaError_t sj_launch_cell_coords(const uint64_t *cellLid, uint32_t nCells, sj_grid_dev g, uint32_t *coord,
                                  cudaStream_t s)
{
    if (nCells == 0) return cudaSuccess;
    k_cell_coords<<<blocks_for(nCells, 256), 256, 0, s>>>(cellLid, nCells, g, coord); sj_note_launch();
    return cudaGetLastError();
}
