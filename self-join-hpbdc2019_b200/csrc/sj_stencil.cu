// Owned neighbour-cell lists and per-cell estimator features.
//
// The reference enumerates the clamped 3^k stencil per query POINT with a
// binary search per neighbour (kernel.cu:1455-1534, 387-396).  Here the
// stencil is enumerated once per non-empty CELL by a depth-first walk over the
// linear-id ordering (dim k-1 most significant): each level narrows the range
// of the sorted id array to the cells sharing the chosen coordinate prefix, so
// empty sub-stencils are pruned early (sparse high-dimensional grids).
//
// Ownership rules decide which cell of an adjacent pair evaluates it:
//   FULL      every neighbour (mode 3/7/9 semantics; one direction emitted)
//   LID       neighbours with a larger linear id (kernel.cu:1529-1534)
//   UNICOMP   the highest differing dimension's coordinate of the owner is odd
//             (stamploops.h)
//   BUNICOMP  checkerboard colour rules for k = 2, 3 (kernel.cu:1346-1392)
// Each rule assigns every adjacent pair to exactly one owner.
#include "sj_internal.h"

namespace {

__device__ __forceinline__ uint32_t lower_bound_u64(const uint64_t *__restrict__ a, uint32_t lo, uint32_t hi,
                                                    unsigned long long key)
{
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ bool owns(int pattern, int k, const uint32_t *a, const int *off, unsigned long long myLid,
                                     unsigned long long nbLid)
{
    switch (pattern) {
    case SJ_PAT_FULL:
        return true;
    case SJ_PAT_LID:
        return nbLid > myLid;
    case SJ_PAT_UNICOMP: {
        int d = k - 1;
        while (d > 0 && off[d] == 0) d--;
        return (a[d] & 1u) != 0;
    }
    case SJ_PAT_BUNICOMP: {
        if (k == 2) {
            uint32_t v0 = a[0] + off[0], v1 = a[1] + off[1];
            bool odd = ((a[0] + a[1]) & 1u) != 0;
            if (odd) return (a[1] <= v1) && (a[0] != v0);
            return (a[1] < v1) || (v1 < a[1] && v0 == a[0]);
        } else {
            uint32_t v0 = a[0] + off[0], v1 = a[1] + off[1], v2 = a[2] + off[2];
            bool odd = ((a[0] + a[1] + a[2]) & 1u) != 0;
            if (odd)
                return (a[0] != v0 && a[1] <= v1 && a[2] <= v2) || (a[0] == v0 && a[1] <= v1 && a[2] < v2) ||
                       (a[1] < v1 && v2 < a[2]);
            return (a[1] < v1 && a[2] <= v2) || (a[0] == v0 && v1 < a[1] && a[2] <= v2) ||
                   (a[0] != v0 && a[1] < v1 && v2 < a[2]) || (a[1] == v1 && a[2] < v2);
        }
    }
    }
    return false;
}

// pass 0: count owned neighbours (out = counts), full-stencil candidates and
//         features; pass 1: write owned neighbour cell indices (out = list).
__global__ void __launch_bounds__(128) k_neighbours(const uint64_t *__restrict__ cellLid,
                                                    const uint32_t *__restrict__ cellCoord,
                                                    const uint32_t *__restrict__ cellStart, uint32_t nCells,
                                                    sj_grid_dev g, int pattern,
                                                    const uint32_t *__restrict__ nbrStart, uint32_t *__restrict__ out,
                                                    uint64_t *__restrict__ candFull,
                                                    unsigned long long *__restrict__ candTotal,
                                                    float *__restrict__ feat, int pass)
{
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nCells) return;
    const int k = g.k;
    uint32_t a[SJ_MAX_K];
    for (int j = 0; j < k; j++) a[j] = cellCoord[(uint64_t)c * k + j];
    const unsigned long long myLid = cellLid[c];
    const uint32_t myOcc = cellStart[c + 1] - cellStart[c];

    uint32_t lo[SJ_MAX_K + 1], hi[SJ_MAX_K + 1];
    unsigned long long base[SJ_MAX_K + 1];
    int t[SJ_MAX_K], off[SJ_MAX_K];
    lo[k] = 0; hi[k] = nCells; base[k] = 0;
    for (int j = 0; j < k; j++) off[j] = 0;

    uint32_t owned = 0, writePos = (pass == 1) ? nbrStart[c] : 0u;
    unsigned long long stencilOcc = 0;
    uint32_t hist[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    // owned neighbours' occupancy weighted by the uniform-density hit
    // probability of their offset class (all classes, classes 1 and 2)
    float ownW = 0.0f, ownW1 = 0.0f, ownW2 = 0.0f;

    int j = k - 1;
    t[j] = 0;
    while (j < k) {
        if (t[j] == 3) {
            j++;
            if (j < k) t[j]++;
            continue;
        }
        long long v = (long long)a[j] + t[j] - 1;
        if (v >= 0 && v < (long long)g.nCells[j]) {
            unsigned long long idLo = base[j + 1] + (unsigned long long)v * g.mult[j];
            unsigned long long idHi = idLo + g.mult[j];
            uint32_t l = lower_bound_u64(cellLid, lo[j + 1], hi[j + 1], idLo);
            uint32_t h = lower_bound_u64(cellLid, l, hi[j + 1], idHi);
            if (l < h) {
                off[j] = t[j] - 1;
                if (j == 0) {
                    // leaf: exactly one cell (mult[0] == 1)
                    uint32_t b = l;
                    uint32_t occ = cellStart[b + 1] - cellStart[b];
                    stencilOcc += occ;
                    bool home = (b == c);
                    if (!home) {
                        int bin = 31 - __clz(occ);
                        hist[bin > 7 ? 7 : bin]++;
                        if (owns(pattern, k, a, off, myLid, cellLid[b])) {
                            if (pass == 1) out[writePos++] = b;
                            owned++;
                            if (feat) {
                                int m = 0;
                                for (int q = 0; q < k; q++) m += off[q] != 0;
                                const float wo = (float)occ * g.offW[m];
                                ownW += wo;
                                if (m == 1) ownW1 += wo;
                                else if (m == 2) ownW2 += wo;
                            }
                        }
                    }
                    t[0]++;
                    continue;
                }
                lo[j] = l; hi[j] = h; base[j] = idLo;
                j--;
                t[j] = 0;
                continue;
            }
        }
        t[j]++;
    }
    if (pass == 0) {
        out[c] = owned;
        candFull[c] = stencilOcc * (unsigned long long)myOcc;
        if (candTotal) atomicAdd(candTotal, stencilOcc * (unsigned long long)myOcc);
        if (feat) {
            float *f = feat + (uint64_t)c * SJ_NFEAT;
            float nst = 1.0f;
            for (int q = 0; q < k; q++) nst *= 3.0f;
            nst -= 1.0f;
            // occupancy, neighbour-occupancy histogram, eps / cell width,
            // dimension; f9, f13, f14: the expected hits with the owned
            // neighbours (all offset classes, face neighbours, edge neighbours)
            // under a locally uniform density, log2(1 + occupancy x weighted sum)
            const float o = (float)myOcc;
            f[0] = log2f(1.0f + o);
            for (int b = 0; b < 8; b++) f[1 + b] = (float)hist[b] / nst;
            f[9] = log2f(1.0f + o * ownW);
            f[10] = log2f(1.0f + (float)stencilOcc);
            f[11] = 1.0f;                          // eps / cell width (cells are eps wide)
            f[12] = (float)g.D / 16.0f;
            f[13] = log2f(1.0f + o * ownW1);
            f[14] = log2f(1.0f + o * ownW2);
            f[15] = log2f((float)g.eps) / 8.0f;
        }
    }
}

}  // namespace

cudaError_t sj_launch_neighbours(const uint64_t *cellLid, const uint32_t *cellCoord, const uint32_t *cellStart,
                                 uint32_t nCells, sj_grid_dev g, int pattern, const uint32_t *nbrStart,
                                 uint32_t *nbrCountOrCell, uint64_t *candFull, unsigned long long *candTotal,
                                 float *feat, int pass, cudaStream_t s)
{
    if (nCells == 0) return cudaSuccess;
    k_neighbours<<<(nCells + 127) / 128, 128, 0, s>>>(cellLid, cellCoord, cellStart, nCells, g, pattern, nbrStart,
                                                      nbrCountOrCell, candFull, candTotal, feat, pass);
    sj_note_launch();
    return cudaGetLastError();
}
