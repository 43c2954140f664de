// ref_pipeline: times the reference's own batched GPU self-join
// (distanceTableNDGridBatches, GPU.cu:1297-2569) exactly as its main() does
// (main.cu:83-197): import + bin sort, CPU grid build (untimed, as in the
// reference), warm-up, then the timed call.  Test / baseline infrastructure.
//
// usage: ref_pipeline <dataset.csv> <epsilon> <searchmode>
// prints one JSON line: {"time_s", "index_s", "total_neighbors", "n", "pair_hash"}
// pair_hash (sum of splitmix64(key<<32|val)) is computed from the neighbour
// table only for mode 3 with SORT_BY_WORKLOAD 0, where every key lives in one
// batch and the reference's table is complete.
#include <omp.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "GPU.h"
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

static unsigned long long mix(unsigned long long z)
{
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

int main(int argc, char **argv)
{
    if (argc != 4) {
        fprintf(stderr, "usage: %s <dataset.csv> <epsilon> <searchmode>\n", argv[0]);
        return 2;
    }
    DTYPE epsilon = atof(argv[2]);
    int mode = atoi(argv[3]);
    std::vector<std::vector<DTYPE> > pts;
    importNDDataset(&pts, argv[1]);
    sortInNDBins(&pts);
    warmUpGPU();
    double ti0 = omp_get_wtime();
    DTYPE *minArr = new DTYPE[NUMINDEXEDDIM], *maxArr = new DTYPE[NUMINDEXEDDIM];
    unsigned *nCells = new unsigned[NUMINDEXEDDIM];
    uint64_t totalCells = 0, totalNeighbors = 0;
    unsigned nNonEmpty = 0;
    generateNDGridDimensions(&pts, epsilon, minArr, maxArr, nCells, &totalCells);
    struct grid *index;
    struct gridCellLookup *lookup;
    unsigned *mask, *nMask = new unsigned, *maskOff = new unsigned[2 * NUMINDEXEDDIM];
    unsigned *indexLookupArr = new unsigned[pts.size()];
    populateNDGridIndexAndLookupArray(&pts, epsilon, &lookup, &index, indexLookupArr, minArr, nCells, totalCells,
                                      &nNonEmpty, &mask, maskOff, nMask);
    double ti1 = omp_get_wtime();
    neighborTableLookup *table = new neighborTableLookup[pts.size()]();
    std::vector<struct neighborDataPtrs> ptrs;
    double t0 = omp_get_wtime();
    distanceTableNDGridBatches(mode, &pts, &epsilon, index, lookup, &nNonEmpty, minArr, nCells, indexLookupArr, table,
                               &ptrs, &totalNeighbors, mask, maskOff, nMask);
    double t1 = omp_get_wtime();
    unsigned long long h = 0;
    int hashed = 0, missing = 0;
    if (mode == 3 && SORT_BY_WORKLOAD == 0) {
        hashed = 1;
        for (size_t i = 0; i < pts.size(); i++) {
            if (!table[i].dataPtr) { missing++; continue; }
            for (int j = table[i].indexmin; j <= table[i].indexmax; j++)
                h += mix(((unsigned long long)(unsigned)i << 32) | (unsigned)table[i].dataPtr[j]);
        }
    }
    char hs[64];
    if (hashed && !missing) snprintf(hs, sizeof(hs), "%llu", h);
    else snprintf(hs, sizeof(hs), "null");
    printf("\n{\"time_s\": %.6f, \"index_s\": %.6f, \"total_neighbors\": %llu, \"n\": %zu, \"mode\": %d, "
           "\"pair_hash\": %s, \"missing_rows\": %d}\n",
           t1 - t0, ti1 - ti0, (unsigned long long)totalNeighbors, pts.size(), mode, hs, missing);
    return 0;
}
