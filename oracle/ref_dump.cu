// ref_dump: runs ONE of the reference's own join kernels (kernel.cu, modes
// 3/4/5/6, SORT_BY_WORKLOAD 0) over the whole dataset as a single batch and
// writes the raw (key, value) pairs, so parity tests can compare against the
// reference's actual device arithmetic.  Test infrastructure only.
//
// Everything the kernels see is built by the reference's own host code:
// importNDDataset + sortInNDBins (import_dataset.cpp) and
// generateNDGridDimensions + populateNDGridIndexAndLookupArray (main.cu,
// compiled with its main() renamed).  The output buffer is sized to an upper
// bound on what the kernel can write: every candidate evaluation emits at most
// two pairs, and the candidate count is computed here from the same index.
//
// usage: ref_dump <dataset.csv> <epsilon> <searchmode> <out.bin>
// out.bin: uint64 count, int32 keys[count], int32 vals[count]
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "kernel.h"
#include "params.h"
#include "structs.h"

void importNDDataset(std::vector<std::vector<DTYPE> > *dataPoints, char *fname);
void sortInNDBins(std::vector<std::vector<DTYPE> > *dataPoints);
void generateNDGridDimensions(std::vector<std::vector<DTYPE> > *NDdataPoints, DTYPE epsilon, DTYPE *minArr,
                              DTYPE *maxArr, unsigned int *nCells, uint64_t *totalCells);
void populateNDGridIndexAndLookupArray(std::vector<std::vector<DTYPE> > *NDdataPoints, DTYPE epsilon,
                                       struct gridCellLookup **gridCellLookupArr, struct grid **index,
                                       unsigned int *indexLookupArr, DTYPE *minArr, unsigned int *nCells,
                                       uint64_t totalCells, unsigned int *nNonEmptyCells,
                                       unsigned int **gridCellNDMask, unsigned int *gridCellNDMaskOffsets,
                                       unsigned int *nNDMaskElems);

#define CHECK(x)                                                                              \
    do {                                                                                      \
        cudaError_t e = (x);                                                                  \
        if (e != cudaSuccess) {                                                               \
            fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e), __FILE__, __LINE__); \
            exit(3);                                                                          \
        }                                                                                     \
    } while (0)

template <typename T>
static T *upload(const T *h, size_t n)
{
    T *d = nullptr;
    CHECK(cudaMalloc((void **)&d, sizeof(T) * (n ? n : 1)));
    if (n) CHECK(cudaMemcpy(d, h, sizeof(T) * n, cudaMemcpyHostToDevice));
    return d;
}

int main(int argc, char **argv)
{
    if (argc != 5) {
        fprintf(stderr, "usage: %s <dataset.csv> <epsilon> <searchmode> <out.bin>\n", argv[0]);
        return 2;
    }
    DTYPE epsilon = atof(argv[2]);
    int mode = atoi(argv[3]);
    if (mode < 3 || mode > 6) {
        fprintf(stderr, "modes 3..6 only\n");
        return 2;
    }
    std::vector<std::vector<DTYPE> > pts;
    importNDDataset(&pts, argv[1]);
    sortInNDBins(&pts);
    const unsigned n = (unsigned)pts.size();
    DTYPE minArr[NUMINDEXEDDIM], maxArr[NUMINDEXEDDIM];
    unsigned nCells[NUMINDEXEDDIM];
    uint64_t totalCells = 0;
    generateNDGridDimensions(&pts, epsilon, minArr, maxArr, nCells, &totalCells);
    struct grid *index;
    struct gridCellLookup *lookup;
    unsigned *mask, nMask = 0, maskOff[2 * NUMINDEXEDDIM], nNonEmpty = 0;
    std::vector<unsigned> indexLookupArr(n);
    populateNDGridIndexAndLookupArray(&pts, epsilon, &lookup, &index, indexLookupArr.data(), minArr, nCells,
                                      totalCells, &nNonEmpty, &mask, maskOff, &nMask);

    // Upper bound on pairs written: 2 x sum over cells |c| * sum over its 3^k stencil |c'|.
    unsigned long long evals = 0;
    {
        std::vector<uint64_t> lids(nNonEmpty);
        for (unsigned i = 0; i < nNonEmpty; i++) lids[i] = lookup[i].gridLinearID;
        for (unsigned c = 0; c < nNonEmpty; c++) {
            uint64_t lid = lids[c], rem = lid;
            long long coord[NUMINDEXEDDIM];
            for (int j = 0; j < NUMINDEXEDDIM; j++) { coord[j] = (long long)(rem % nCells[j]); rem /= nCells[j]; }
            int off[NUMINDEXEDDIM];
            for (int j = 0; j < NUMINDEXEDDIM; j++) off[j] = -1;
            unsigned long long sum = 0;
            for (;;) {
                bool ok = true;
                uint64_t id = 0, mul = 1;
                for (int j = 0; j < NUMINDEXEDDIM; j++) {
                    long long v = coord[j] + off[j];
                    if (v < 0 || v >= (long long)nCells[j]) { ok = false; break; }
                    id += (uint64_t)v * mul;
                    mul *= nCells[j];
                }
                if (ok) {
                    auto it = std::lower_bound(lids.begin(), lids.end(), id);
                    if (it != lids.end() && *it == id) {
                        size_t b = it - lids.begin();
                        sum += (unsigned long long)(index[b].indexmax - index[b].indexmin + 1);
                    }
                }
                int j = 0;
                while (j < NUMINDEXEDDIM && off[j] == 1) { off[j] = -1; j++; }
                if (j == NUMINDEXEDDIM) break;
                off[j]++;
            }
            evals += sum * (unsigned long long)(index[c].indexmax - index[c].indexmin + 1);
        }
    }
    unsigned long long cap = 2ULL * evals + 1024ULL;
    if (cap > 0x7fffffffULL) {
        fprintf(stderr, "candidate bound %llu too large for one batch\n", cap);
        return 4;
    }

    std::vector<DTYPE> db((size_t)n * GPUNUMDIM);
    for (unsigned i = 0; i < n; i++)
        for (int l = 0; l < GPUNUMDIM; l++) db[(size_t)i * GPUNUMDIM + l] = pts[i][l];

    unsigned zero = 0, one = 1, N = n;
    DTYPE *d_db = upload(db.data(), db.size());
    DTYPE *d_eps = upload(&epsilon, 1);
    struct grid *d_index = upload(index, nNonEmpty);
    unsigned *d_lookupArr = upload(indexLookupArr.data(), n);
    struct gridCellLookup *d_gcl = upload(lookup, nNonEmpty);
    DTYPE *d_min = upload(minArr, NUMINDEXEDDIM);
    unsigned *d_nCells = upload(nCells, NUMINDEXEDDIM);
    unsigned *d_cnt = upload(&zero, 1);
    unsigned *d_nne = upload(&nNonEmpty, 1);
    unsigned *d_mask = upload(mask, nMask);
    unsigned *d_maskOff = upload(maskOff, 2 * NUMINDEXEDDIM);
    unsigned *d_N = upload(&N, 1);
    unsigned *d_offset = upload(&one, 1);
    unsigned *d_batch = upload(&zero, 1);
    unsigned *d_dbg1 = upload(&zero, 1), *d_dbg2 = upload(&zero, 1);
    int *d_key, *d_val;
    CHECK(cudaMalloc((void **)&d_key, sizeof(int) * cap));
    CHECK(cudaMalloc((void **)&d_val, sizeof(int) * cap));
    const int blocks = (int)((N + BLOCKSIZE - 1) / BLOCKSIZE);
    switch (mode) {
    case 3:
        kernelNDGridIndexGlobal<<<blocks, BLOCKSIZE>>>(d_dbg1, d_dbg2, d_N, d_offset, d_batch, d_db, NULL, d_eps,
                                                       d_index, d_lookupArr, d_gcl, d_min, d_nCells, d_cnt, d_nne,
                                                       d_mask, d_maskOff, d_key, d_val);
        break;
    case 4:
        kernelNDGridIndexGlobalUnicomp<<<blocks, BLOCKSIZE>>>(d_dbg1, d_dbg2, d_N, d_offset, d_batch, d_db, NULL,
                                                              d_eps, d_index, d_lookupArr, d_gcl, d_min, d_nCells,
                                                              d_cnt, d_nne, d_mask, d_maskOff, d_key, d_val);
        break;
    case 5:
        kernelNDGridIndexGlobalBUnicomp<<<blocks, BLOCKSIZE>>>(d_dbg1, d_dbg2, d_N, d_offset, d_batch, d_db, NULL,
                                                               d_eps, d_index, d_lookupArr, d_gcl, d_min, d_nCells,
                                                               d_cnt, d_nne, d_mask, d_maskOff, d_key, d_val);
        break;
    case 6:
        kernelNDGridIndexGlobalLinearIDUnicomp<<<blocks, BLOCKSIZE>>>(d_dbg1, d_dbg2, d_N, d_offset, d_batch, d_db,
                                                                      NULL, d_eps, d_index, d_lookupArr, d_gcl, d_min,
                                                                      d_nCells, d_cnt, d_nne, d_mask, d_maskOff,
                                                                      d_key, d_val);
        break;
    }
    CHECK(cudaGetLastError());
    CHECK(cudaDeviceSynchronize());
    unsigned cnt = 0;
    CHECK(cudaMemcpy(&cnt, d_cnt, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if ((unsigned long long)cnt > cap) {
        fprintf(stderr, "kernel wrote %u pairs, bound %llu\n", cnt, cap);
        return 5;
    }
    std::vector<int> key(cnt), val(cnt);
    if (cnt) {
        CHECK(cudaMemcpy(key.data(), d_key, sizeof(int) * cnt, cudaMemcpyDeviceToHost));
        CHECK(cudaMemcpy(val.data(), d_val, sizeof(int) * cnt, cudaMemcpyDeviceToHost));
    }
    FILE *f = fopen(argv[4], "wb");
    if (!f) return 6;
    uint64_t c64 = cnt;
    fwrite(&c64, sizeof(c64), 1, f);
    fwrite(key.data(), sizeof(int), cnt, f);
    fwrite(val.data(), sizeof(int), cnt, f);
    fclose(f);
    printf("\nref_dump: n=%u mode=%d pairs=%u evals=%llu\n", n, mode, cnt, evals);
    return 0;
}
