// sj_main: command-line driver with the reference's interface (main.cu:36-222).
//
//   sj_main <dataset.csv> <epsilon> <ndim> <searchmode> [options]
//
// Positional arguments are the reference's (main.cu:46-65).  Options replace
// its compile-time params.h knobs:
//   --k K              NUMINDEXEDDIM (default: ndim)
//   --precision P      fp64 | mixed   (FP32 filter + FP64 refinement)
//   --learned FILE     learned batch estimator weights
//   --capacity N       result pairs per batch (default: automatic)
//   --sort S           SORT_BY_WORKLOAD 0/1 (default 1)
//   --print            print every point's sorted neighbour list (main.cu:212-222)
// Appends one line to gpu_<mode>_stats.txt in the format of main.cu:203-206.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "sj.h"

static const char *stats_file(int mode)
{
    switch (mode) {
    case 3: return "gpu_global_stats.txt";
    case 4: return "gpu_unicomp_stats.txt";
    case 5: return "gpu_b-unicomp_stats.txt";
    case 6: return "gpu_linID-unicomp_stats.txt";
    case 7: return "gpu_sorting-cells_stats.txt";
    case 8: return "gpu_dynamic-threads-fixed_stats.txt";
    case 9: return "gpu_working-queue_stats.txt";
    case 10: return "gpu_working-queue_lid-unicomp_stats.txt";
    }
    return "gpu_stats.txt";
}

static int fail(sj_status s)
{
    fprintf(stderr, "\nERROR: %s: %s\n", sj_status_string(s), sj_last_error());
    return 1;
}

int main(int argc, char **argv)
{
    if (argc < 5) {
        printf("\n\nIncorrect number of input parameters.  \nShould be dataset file, epsilon, number of dimensions, "
               "searchmode\n");
        return 0;
    }
    const char *fname = argv[1];
    double eps = atof(argv[2]);
    int ndim = atoi(argv[3]);
    int mode = atoi(argv[4]);
    sj_params p;
    sj_params_default(&p);
    p.gpunumdim = ndim;
    p.numindexeddim = ndim;
    p.epsilon = eps;
    p.search_mode = mode;
    bool print = false;
    const char *learned = nullptr;
    for (int i = 5; i < argc; i++) {
        std::string a = argv[i];
        auto next = [&](void) -> const char * { return (i + 1 < argc) ? argv[++i] : ""; };
        if (a == "--k") p.numindexeddim = atoi(next());
        else if (a == "--precision") p.precision = (std::string(next()) == "mixed") ? SJ_PREC_FP32_REFINE : SJ_PREC_FP64;
        else if (a == "--learned") { learned = next(); p.scheduler = SJ_SCHED_LEARNED; }
        else if (a == "--capacity") p.batch_capacity_pairs = strtoull(next(), nullptr, 10);
        else if (a == "--sort") p.sort_by_workload = atoi(next());
        else if (a == "--print") print = true;
        else { fprintf(stderr, "unknown option %s\n", a.c_str()); return 2; }
    }
    printf("\nDataset file: %s", fname);
    printf("\nEpsilon: %f", eps);
    printf("\nNumber of dimensions (NDIM): %d\n", ndim);
    sj_ctx *ctx = nullptr;
    sj_status s = sj_create(&p, &ctx);
    if (s != SJ_OK) return fail(s);
    s = sj_import_csv(ctx, fname);
    if (s != SJ_OK) return fail(s);
    if (learned && (s = sj_load_estimator(ctx, learned)) != SJ_OK) return fail(s);
    auto t0 = std::chrono::steady_clock::now();
    s = sj_build_index(ctx);
    if (s != SJ_OK) return fail(s);
    auto t1 = std::chrono::steady_clock::now();
    uint64_t totalNeighbors = 0;
    std::vector<sj_neighbor_table_lookup> table;
    int *values = nullptr;
    uint32_t n = 0;
    sj_stats st;
    sj_get_stats(ctx, &st);
    n = st.n_points;
    if (print) {
        table.resize(n);
        s = sj_neighbor_table(ctx, table.data(), &values, &totalNeighbors);
    } else {
        s = sj_join(ctx, SJ_DELIVER_NONE, nullptr, nullptr);
    }
    if (s != SJ_OK) return fail(s);
    auto t2 = std::chrono::steady_clock::now();
    sj_get_stats(ctx, &st);
    if (!print) totalNeighbors = st.total_pairs;
    double tJoin = std::chrono::duration<double>(t2 - t1).count();
    double tAll = std::chrono::duration<double>(t2 - t0).count();
    printf("\nGrid: total cells (including empty) %llu, non-empty %u", (unsigned long long)st.total_cells,
           st.n_nonempty_cells);
    printf("\nTotal result set size: %llu, batches %llu, refined pairs %llu",
           (unsigned long long)totalNeighbors, (unsigned long long)st.num_batches,
           (unsigned long long)st.refined_pairs);
    printf("\n~~~Time: %f (join), %f (index build + join)\n", tJoin, tAll);
    FILE *f = fopen(stats_file(mode), "a");
    if (f) {
        fprintf(f, "%g, %s, %g, %llu, GPUNUMDIM/NUMINDEXEDDIM/DTYPE/BLOCKSIZE/THperPOINT/SORT: %d, %d, double, %d, %d, %d\n",
                tJoin, fname, eps, (unsigned long long)totalNeighbors, p.gpunumdim, p.numindexeddim, p.blocksize,
                p.threadperpoint, p.sort_by_workload);
        fclose(f);
    }
    if (print) {
        for (uint32_t i = 0; i < n; i++) {
            int lo = table[i].indexmin, hi = table[i].indexmax;
            std::sort(values + lo, values + hi + 1);
            printf("\npoint id: %u, neighbors: ", i);
            printf("nb neighbor %d\n", hi - lo + 1);
            for (int j = lo; j <= hi; j++) printf("%d,", values[j]);
        }
        printf("\n\n\n");
        sj_free(values);
    }
    sj_destroy(ctx);
    return 0;
}
