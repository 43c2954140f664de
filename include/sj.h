/*
 * sj.h -- C ABI of the B200 epsilon self-join engine (libsj.so).
 *
 * Drop-in boundary for the reference's grid-indexed self-join path.  The
 * reference has no plugin API; its de-facto boundary is the C++ function
 *     distanceTableNDGridBatches(searchMode, NDdataPoints, epsilon, index,
 *         gridCellLookupArr, nNonEmptyCells, minArr, nCells, indexLookupArr,
 *         neighborTable, pointersToNeighbors, totalNeighbors, gridCellNDMask,
 *         gridCellNDMaskOffsets, nNDMaskElems)            (GPU.h:37-40, GPU.cu:1297-2569)
 * called from main.cu:194 after the host grid build (main.cu:164-182) and the
 * CSV import (import_dataset.cpp:34-80).  Every entry point below says which
 * part of that path it replaces.
 *
 * Conventions: plain C types only; every call returns sj_status; a context is
 * bound to one CUDA device and is not thread-safe.  Point ids are int32
 * (n < 2^31), exactly like the reference's key/value arrays.
 */
#ifndef SJ_H
#define SJ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SJ_OK = 0,
    SJ_ERR_OOM = 1,            /* device or pinned-host allocation failed */
    SJ_OVERFLOW_RETRIED = 2,   /* informational: a batch overflowed its estimate and was split */
    SJ_ERR_BAD_INPUT = 3,      /* invalid parameter, empty / non-finite / malformed input */
    SJ_ERR_CUDA = 4,           /* CUDA runtime error (message in sj_last_error) */
    SJ_ERR_TIMEOUT = 5,        /* a bounded device wait ran out */
    SJ_ERR_STATE = 6,          /* call made out of order (e.g. join before index) */
    SJ_ERR_IO = 7,             /* file could not be read */
    SJ_ERR_ABORTED = 8,        /* the batch consumer asked to stop */
    SJ_ERR_INTERNAL = 9        /* an internal consistency check failed */
} sj_status;

typedef enum { SJ_PREC_FP64 = 0, SJ_PREC_FP32_REFINE = 1 } sj_precision;
typedef enum { SJ_SCHED_SAMPLING = 0, SJ_SCHED_LEARNED = 1 } sj_scheduler;
typedef enum { SJ_DELIVER_DEVICE = 0, SJ_DELIVER_HOST = 1, SJ_DELIVER_NONE = 2 } sj_delivery;

/*
 * Run parameters.  Field names follow params.h (params.h:1-14) plus the
 * runtime arguments of main.cu:46-65 and the hidden constants of GPU.cu.
 */
typedef struct {
    int gpunumdim;            /* GPUNUMDIM: data dimensions (1..16) */
    int numindexeddim;        /* NUMINDEXEDDIM: grid dimensions, the first k dims (1..min(D,16)) */
    double epsilon;           /* search radius (main.cu:62) */
    int blocksize;            /* BLOCKSIZE: accepted and not used; the engine's CTA shapes are fixed per
                                 kernel (128-thread count pass, 256-thread emission) */
    int threadperpoint;       /* THREADPERPOINT: accepted and not used; the work per query tile is split
                                 across tasks by the scheduler instead (see search_mode 8) */
    int search_mode;          /* 3 full stencil, 4 Unicomp, 5 B-Unicomp (k=2,3), 6 linear-ID Unicomp,
                                 7 full stencil in workload order, 8 full stencil with every query tile's
                                 stream split over 16 / 8 / 2 tasks by the third of the work (in cost
                                 order) its cell falls in (the reference's dynamic threads per point,
                                 NB_THREAD_THIRD1..3), 9 work queue, 10 work queue + LID-Unicomp */
    int sort_by_workload;     /* SORT_BY_WORKLOAD: order work by estimated cost, heaviest first */
    int precision;            /* sj_precision */
    int scheduler;            /* sj_scheduler: estimator used to size result batches */
    uint64_t batch_capacity_pairs; /* max (key,value) pairs per result batch; 0 = automatic */
    double sample_rate;       /* sampling estimator rate (GPU.cu:873 uses 0.01) */
    double alpha;             /* over-estimation factor applied to predictions (GPU.cu:1037 uses 0.05) */
    int device;               /* CUDA device ordinal */
    int shard_index;          /* query-task shard served by this context (0..shard_count-1) */
    int shard_count;          /* number of shards (1 = whole join) */
    int verbose;              /* print per-phase information to stderr */
} sj_params;

/* Reference layouts (structs.h:41-100), kept member-for-member so a caller can
 * hand the arrays to code written against the reference. */
typedef struct { int indexmin; int indexmax; } sj_grid;                      /* struct grid */
typedef struct { unsigned int idx; uint64_t gridLinearID; } sj_grid_cell_lookup; /* struct gridCellLookup */
typedef struct { int pointID; int indexmin; int indexmax; int *dataPtr; } sj_neighbor_table_lookup;
                                                                             /* struct neighborTableLookup */

/* One delivered result batch.  Pairs are sorted by key (ascending point id);
 * the values of one key are contiguous.  A key may appear in several batches
 * (as in the reference); the neighbour-table helper merges them. */
typedef struct {
    uint64_t batch_index;
    uint64_t count;        /* pairs in this batch */
    const int32_t *key;    /* query point ids */
    const int32_t *val;    /* neighbour point ids */
    int on_device;         /* 1: key/val are device pointers valid during the callback */
} sj_batch;

/* Consumer callback; return 0 to continue, non-zero to stop the join. */
typedef int (*sj_batch_cb)(const sj_batch *batch, void *user);

typedef struct {
    uint64_t total_pairs;       /* totalNeighbors (main.cu:194) */
    uint64_t pair_hash;         /* order-independent set hash: wrapping sum of splitmix64(key<<32|val) */
    uint64_t distance_calcs;    /* candidate evaluations performed (both passes counted once) */
    uint64_t full_stencil_calcs;/* evaluations a full-stencil traversal would do (work unit) */
    uint64_t refined_pairs;     /* FP32-borderline candidate pairs re-evaluated in FP64 */
    uint64_t num_batches;
    uint64_t overflow_retries;  /* batches split because the estimate was too low */
    uint64_t num_tasks;
    uint64_t total_cells;       /* grid cells including empty ones */
    uint32_t n_points;
    uint32_t n_nonempty_cells;
    double estimated_pairs;     /* scheduler's prediction of the total pair count */
    double estimator_mean_abs_rel_err; /* mean |pred-meas|/meas over batches */
    double estimator_task_rel_err;     /* sum|pred-meas| / sum(meas) over tasks */
    float ms_upload, ms_index, ms_tasks, ms_estimate, ms_count, ms_scan, ms_fill, ms_deliver, ms_total;
    float ms_join_kernels;      /* count + fill kernel time */
    float ms_fill_kernel;       /* fill kernel time alone */
    uint64_t kernel_launches;   /* this library's kernel launches during the last join */
    float ms_expand;            /* key-array expansion from the batch's key runs */
    uint32_t exact_plan_batches;/* batches the same greedy plan needs with the measured per-task pairs
                                   in place of the predictions (the estimator-free reference count) */
} sj_stats;

/* Opaque engine context: one per device, created by sj_create, released by
 * sj_destroy.  Not thread-safe; calls on one context must not overlap. */
typedef struct sj_ctx sj_ctx;

/* Fill `p` with params.h defaults: D=k=2, BLOCKSIZE 256, THREADPERPOINT 1,
 * SORT_BY_WORKLOAD 1, mode 10, FP64, sampling estimator, rate 0.01, alpha 0.05. */
void sj_params_default(sj_params *p);

/* Replaces the setup half of distanceTableNDGridBatches (GPU.cu:1315-1585) and
 * warmUpGPU (GPU.cu:2572): validates parameters, binds the device. */
sj_status sj_create(const sj_params *p, sj_ctx **ctx_out);
sj_status sj_destroy(sj_ctx *ctx);

/* Replaces importNDDataset + sortInNDBins (import_dataset.cpp:34-80): parses
 * comma/whitespace separated doubles, groups them by gpunumdim, applies the
 * same integer-bin sort (so point ids equal the reference's), uploads. */
sj_status sj_import_csv(sj_ctx *ctx, const char *path);

/* The same parse and point order without a device (host memory only): writes
 * up to `cap` points (cap x gpunumdim doubles) to `out` and the number of
 * complete points in the file to *n.  Call with out = NULL to size. */
sj_status sj_read_csv(const char *path, int gpunumdim, double *out, uint64_t cap, uint64_t *n);

/* Supplies points directly: n x gpunumdim doubles, row-major (the flattened
 * NDdataPoints of GPU.cu:1333-1346).  `on_device` = 1 if `pts` is a device
 * pointer; otherwise it is copied host-to-device. */
sj_status sj_set_points(sj_ctx *ctx, const double *pts, uint64_t n, int on_device);

/* Replaces generateNDGridDimensions + populateNDGridIndexAndLookupArray
 * (main.cu:240-503), built on the device. */
sj_status sj_build_index(sj_ctx *ctx);

/* Reference-layout export of the index for parity checks: sizes first, then
 * arrays (indexLookupArr[n], grid[nNonEmpty], gridCellLookup[nNonEmpty],
 * minArr[k], nCells[k], gridCellNDMask[nMask], gridCellNDMaskOffsets[2k]). */
sj_status sj_index_sizes(sj_ctx *ctx, uint32_t *n_nonempty, uint32_t *n_mask_elems, uint64_t *total_cells);
sj_status sj_index_export(sj_ctx *ctx, unsigned int *indexLookupArr, sj_grid *grid,
                          sj_grid_cell_lookup *gridCellLookupArr, double *minArr, unsigned int *nCells,
                          unsigned int *gridCellNDMask, unsigned int *gridCellNDMaskOffsets);

/* Replaces the batch loop of distanceTableNDGridBatches (GPU.cu:2086-2377):
 * estimates, plans batches, and streams every result batch to `cb`.
 * SJ_DELIVER_NONE runs the join and only folds each batch into the pair count
 * and set hash (sj_stats). */
sj_status sj_join(sj_ctx *ctx, int delivery, sj_batch_cb cb, void *user);

/* Neighbour count of every point (row lengths of the neighbour table) without
 * materialising pairs.  deg: n uint32 on the host. */
sj_status sj_degrees(sj_ctx *ctx, uint32_t *deg);

/* Replaces constructNeighborTableKeyValueWithPtrs (GPU.cu:2595-2637) and the
 * table of main.cu:185: runs the join and fills table[n] with each point's
 * complete neighbour range inside one values array (allocated with malloc,
 * owned by the caller; free it with sj_free).  Keys that span batches are
 * merged, which the reference's table does not do. */
sj_status sj_neighbor_table(sj_ctx *ctx, sj_neighbor_table_lookup *table, int **values, uint64_t *total);
void sj_free(void *p);

/* On-device CSR neighbour table (replaces the host table of
 * constructNeighborTableKeyValueWithPtrs, GPU.cu:2595-2637, without leaving
 * the GPU): rowPtr (n+1 uint64, DEVICE memory, required) receives the row
 * offsets, cols (DEVICE memory, cols_capacity int32) point i's neighbour ids in
 * cols[rowPtr[i] .. rowPtr[i+1]), complete across batches.  With cols = NULL
 * only the degrees run: rowPtr and *total are filled so the caller can size
 * cols.  Fails with SJ_ERR_BAD_INPUT when cols_capacity < total.  Values inside
 * a row are in no particular order (the reference's rows are not sorted
 * either). */
sj_status sj_neighbor_csr(sj_ctx *ctx, uint64_t *rowPtr, int32_t *cols, uint64_t cols_capacity, uint64_t *total);

sj_status sj_get_stats(sj_ctx *ctx, sj_stats *st);

/* The CUDA stream (cudaStream_t) this context's work is ordered on, so a
 * caller can record events around sj_build_index / sj_join.  Work the join runs
 * on its internal second stream is joined back into this one before sj_join
 * returns. */
sj_status sj_get_stream(sj_ctx *ctx, void **stream);

/* Learned estimator.  Weights: SJ_MLP_NPARAM floats laid out W1[16x64], b1[64],
 * W2[64x64], b2[64], W3[64x2], b3[2] (row-major, input-major).  The network's
 * two outputs predict, per cell, log2(1 + hits among its own points) and
 * log2(1 + hits among its owned neighbours' points) (the targets
 * sj_cell_samples measures); the evaluations themselves are computed exactly. */
uint32_t sj_mlp_num_params(void);
sj_status sj_set_estimator_weights(sj_ctx *ctx, const float *w, uint32_t count);
sj_status sj_load_estimator(sj_ctx *ctx, const char *path);

/* Per-cell learned-estimator features and, after sj_degrees or sj_join, the
 * measured per-cell hits and distance calculations (full-stencil semantics).
 * feat: nNonEmpty x 16 floats; hits/calcs: nNonEmpty doubles; NULL skips. */
sj_status sj_cell_features(sj_ctx *ctx, float *feat, double *hits, double *calcs);

/* Per-cell counts of the sampling estimator (scheduler SJ_SCHED_SAMPLING):
 * runs the estimate for the built index and writes, per non-empty cell, the
 * hits and evaluations of its sampled points among its own points (home, self
 * included) and among its owned neighbours' points (one direction).  With
 * sample_rate = 1 every point is sampled and the counts are exact: they are
 * the learned estimator's training targets.  Each array: nNonEmpty doubles;
 * NULL skips it.  No counterpart in the reference (its estimator returns one
 * total, GPU.cu:854-1065). */
sj_status sj_cell_samples(sj_ctx *ctx, double *homeHits, double *homeEvals, double *nbrHits, double *nbrEvals);

/* Device training of the estimator MLP by the project's own kernels.
 * x: m x 16, y: m x 2 (host float arrays); w: in/out parameters. */
sj_status sj_mlp_train(const float *x, const float *y, uint32_t m, float *w, int steps, float lr,
                       uint32_t batch, uint64_t seed, float *final_loss, int device);
/* Loss and gradient of the mean squared error at w on (x, y): grad has
 * SJ_MLP_NPARAM floats.  Used by the gradient check against the CPU oracle. */
sj_status sj_mlp_loss_grad(const float *x, const float *y, uint32_t m, const float *w, float *loss,
                           float *grad, int device);
/* Forward pass only: out m x 2. */
sj_status sj_mlp_forward(const float *x, uint32_t m, const float *w, float *out, int device);

/* Loss and gradient of the estimator MLP, like sj_mlp_loss_grad, for callers
 * that cannot allocate device memory: code that runs while its stream is being
 * captured into a CUDA graph (where cudaMalloc and cudaFree are not allowed),
 * and services that reserve all of their GPU memory up front and must not grow
 * the device heap afterwards.  No counterpart in the reference.
 *
 * Every pointer is DEVICE memory owned by the caller: x (m x 16), y (m x 2),
 * w (SJ_MLP_NPARAM), loss (1 float, overwritten), grad (SJ_MLP_NPARAM).  The
 * per-sample activations live in a fixed array inside the library sized for
 * SJ_MLP_NOALLOC_MAX_SAMPLES samples (about 8.5 MB, held by every device that
 * loads the library until the process exits); larger m is rejected with
 * SJ_ERR_BAD_INPUT.  Work is queued on `stream` (a cudaStream_t; NULL = the
 * default stream) and the call returns without synchronising.  The first call
 * on each device looks up the array's device address; make that first call
 * before any stream capture begins.  All calls on a device share the one
 * array: calls whose work overlaps on the GPU (different streams, or
 * different threads on one device) race and corrupt each other's results, so
 * order them on one stream or serialise them.  The array's address is looked
 * up once per device and kept for the life of the process: after
 * cudaDeviceReset on a device, this entry point must not be called on it
 * again.  A CUDA error still pending from earlier work on the calling thread
 * makes the call return SJ_ERR_CUDA without launching (the error is left for
 * its owner to read). */
#define SJ_MLP_NOALLOC_MAX_SAMPLES 8192
sj_status sj_mlp_loss_grad_noalloc(const float *x, const float *y, uint32_t m, const float *w, float *loss,
                                   float *grad, void *stream);

/* Kernels this library has launched since it was loaded (all contexts). */
uint64_t sj_kernel_launch_count(void);

const char *sj_status_string(sj_status s);
const char *sj_last_error(void);
const char *sj_version(void);

#ifdef __cplusplus
}
#endif
#endif /* SJ_H */
