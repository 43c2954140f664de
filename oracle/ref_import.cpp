// ref_import: runs the reference's own importNDDataset + sortInNDBins
// (import_dataset.cpp:34-80) and writes the resulting points, row-major, as raw
// float64 (preceded by a uint64 point count).  CPU only; test infrastructure.
//
// usage: ref_import <dataset.csv> <out.bin>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "params.h"

void importNDDataset(std::vector<std::vector<DTYPE> > *dataPoints, char *fname);
void sortInNDBins(std::vector<std::vector<DTYPE> > *dataPoints);

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s <dataset.csv> <out.bin>\n", argv[0]);
        return 2;
    }
    std::vector<std::vector<DTYPE> > pts;
    importNDDataset(&pts, argv[1]);
    sortInNDBins(&pts);
    FILE *f = fopen(argv[2], "wb");
    if (!f) return 3;
    uint64_t n = pts.size();
    fwrite(&n, sizeof(n), 1, f);
    for (auto &p : pts) fwrite(p.data(), sizeof(DTYPE), p.size(), f);
    fclose(f);
    return 0;
}
