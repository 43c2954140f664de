// Internal declarations shared by the engine's host code and its CUDA kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "sj.h"

#define SJ_MAX_DIM 16        // data dimensions handled by the kernels (padded to a template width)
#define SJ_MAX_K 16          // indexed dimensions
#define SJ_CTA 128           // threads per join CTA (one query point per thread)
#define SJ_STAGE 256         // candidates staged in shared memory per step
#define SJ_MAX_SEG 1024      // candidate segments (home + neighbour cells) per task
#define SJ_NFEAT 16          // learned-estimator input features per cell
#define SJ_HID 64            // learned-estimator hidden width
#define SJ_NOUT 2            // learned-estimator outputs (log distance calcs, log hits)

// Query slots per join thread: a join task covers up to SJ_CTA * slots query
// points of one cell (each thread evaluates every staged candidate against
// `slots` queries held in registers).
#ifndef SJ_SLOTS_F32
#define SJ_SLOTS_F32 4       // query slots of the FP32 filter for Dp <= 8 (2 above)
#endif
#ifndef SJ_SLOTS_F64
#define SJ_SLOTS_F64 4       // query slots of the FP64 predicate for Dp <= 8 (2 above)
#endif
constexpr int sj_query_slots(int Dp, bool fp32)
{
    return Dp <= 8 ? (fp32 ? SJ_SLOTS_F32 : SJ_SLOTS_F64) : 2;
}

// Traversal (neighbour ownership) patterns, mapped from the reference's search modes.
enum sj_pattern { SJ_PAT_FULL = 0, SJ_PAT_UNICOMP = 1, SJ_PAT_BUNICOMP = 2, SJ_PAT_LID = 3 };

// Grid geometry, passed by value to kernels.
struct sj_grid_dev {
    int D;            // data dimensions
    int Dp;           // padded stride of the cell-sorted coordinate array
    int k;            // indexed dimensions
    double eps;
    double thresh;    // largest T with sqrt(T) <= eps (FP64 round-to-nearest)
    double minArr[SJ_MAX_K];
    unsigned nCells[SJ_MAX_K];
    unsigned long long mult[SJ_MAX_K];
    double center[SJ_MAX_DIM];  // origin used for non-indexed dimensions in the FP32 filter
    float offW[SJ_MAX_K + 1];   // estimator features: P(two points uniform in two cells whose coordinates
                                // differ by one in m of the k indexed dims lie within eps), m = 0..k
};

// One unit of join work: query points [qBegin, qBegin+qCount) of cell `cell`
// (cell-sorted positions) against stream positions [sBegin, sEnd) of the
// concatenation of segments segBase..segBase+segCount-1 of that cell's
// candidate list (segment 0 is the home cell, the rest are owned neighbours).
struct sj_task {
    uint32_t cell;
    uint32_t qBegin;
    uint32_t qCount;
    uint32_t segBase;
    uint32_t segCount;
    uint32_t sBegin;
    uint32_t sEnd;
    uint32_t flags;   // bit0: symmetric emission, bit1: home segment included
};

#define SJ_TASK_SYM 1u
#define SJ_TASK_HOME 2u

// Device-side state of one join (all pointers device memory).
struct sj_join_args {
    const double *xs;           // n x Dp cell-sorted coordinates (FP64)
    const uint32_t *ids;        // n point ids in cell-sorted order (indexLookupArr)
    const uint32_t *cellStart;  // nCells+1
    const uint32_t *nbrStart;   // nCells+1 (owned neighbour list, excludes home)
    const uint32_t *nbrCell;
    const uint32_t *cellCoord;  // nCells x k
    const sj_task *tasks;
    uint32_t taskBegin, taskEnd;
    uint32_t *queueHead;        // persistent-queue cursor (work-queue modes)
    uint32_t *keyCount;         // count pass: per point-id pair counts
    const uint32_t *keyStart;   // emission: first slot of each point id's key run (exclusive scan)
    int32_t *outKey, *outVal;   // batch output: keys by sj_expand_keys, values by the emission
    uint64_t capacity;          // pairs the output buffers hold
    unsigned long long *stat;   // [2] pairs (count pass), [3] run past capacity, [4] set hash,
                                // [5] batches skipped for overflow, [6] emission record out of range,
                                // [7] CSR table row overflow
    unsigned long long *batchPairs;  // this batch's pair total (count pass adds, later passes read)
    uint32_t *taskHits;         // optional per-task measured pairs (count pass)
    // count-pass records consumed by the emission pass (null: not recorded).
    // Offsets are absolute over all tasks; a batch indexes from its first task's.
    uint32_t *masks;            // per task: row hit masks, bit i = candidate 32*block+i, laid out
                                // [chunk of 64 blocks][query][block in chunk] (sj_row_mask_index)
    const uint64_t *maskOff;    // per task: first row-mask word
    uint32_t *colMasks;         // per symmetric task: column hit masks [block][query group][candidate],
                                // bit i = query 32*group+i (the query itself dropped on the home diagonal)
    const uint64_t *colOff;     // per task: first column-mask word
    uint32_t *rowRel;           // per task and query: offset of the task's row run inside the
                                // query's key run (the key's count before the task added to it)
    const uint64_t *rowOff;     // per task: first row offset
    uint32_t *candId;           // per task and stream position: the candidate's point id
    uint32_t *candRel;          // per symmetric task and stream position: offset of the position's
                                // column run inside the candidate's key run
    const uint64_t *candOff;    // per task: first candidate record (prefix of stream lengths)
    const uint64_t *unitOff;    // per task: first emission unit (query groups, then column blocks)
    uint32_t *taskEvals;        // per task: candidate evaluations
    uint32_t *taskRefined;      // per task: FP32 borderline re-evaluations
    double margin;              // FP32 filter: bound M on |FP32 estimate - (FP64 d2 - T)|
    float delta;                // FP32 filter: width of the borderline band (>= 2M plus threshold rounding)
};

// Row-mask word of query qi and block b of a task with qc queries and nBlk
// blocks: chunks of 64 blocks, each [query][block in chunk], so one query's
// words of a chunk are contiguous.
__host__ __device__ inline uint64_t sj_row_mask_index(uint32_t b, uint32_t qi, uint32_t qc, uint32_t nBlk)
{
    const uint32_t c = b >> 6;
    const uint32_t cb = (nBlk - 64 * c) < 64 ? (nBlk - 64 * c) : 64;
    return (uint64_t)64 * c * qc + (uint64_t)qi * cb + (b & 63);
}

// Parameters of the device task builder (sj_tasks.cu).
struct sj_taskgen {
    const uint32_t *cellStart;   // nCells+1
    const uint32_t *nbrStart;    // nCells+1, owned neighbour lists
    const uint32_t *nbrCell;
    const float *rate;           // per cell: predicted hits per evaluation against its own points and
                                 // against its neighbours' (2 floats; null: 0)
    const uint32_t *groupBase;   // per cell: first slot in groupLen (exclusive scan of segment groups)
    uint32_t *groupLen;          // per segment group: stream length without the home segment
    uint32_t nCells;
    uint32_t tile;               // query points per task (SJ_CTA x query slots)
    uint64_t cap;                // batch capacity: a task's worst case must fit
    double pairsPerTask;         // chunking target of policy 0
    double evalsPerTask;         // policy 0: evaluations per task at most (0: no limit)
    int sym;                     // symmetric traversal (owned neighbours, both directions emitted)
    int policy;                  // 0 cost-proportional chunks, 1 fixed 65536, 2 mode-8 split by thirds of the work
    float sampleRate;            // > 0: tasks for the sampled queries of each cell only (sampling estimator)
    // spread != 0: a task's neighbour pairs follow the offset-class model
    // (sj_nbr_spread) instead of the cell's mean rate
    int spread;
    const uint32_t *nbrPre;      // per owned-neighbour entry: exclusive prefix of occupancy within its cell
    const double *nbrPreW;       // per entry: exclusive prefix of occupancy x offset-class weight
    const float *nbrWt;          // per entry: its offset-class weight
    const double *cellW;         // per cell: sum of occupancy x weight over its owned neighbours
};

// Kernel launches made by this library since load (every launcher calls
// sj_note_launch() after each <<<...>>>; bench and tests read the total).
void sj_note_launch();
unsigned long long sj_launch_total();
// sets the text returned by sj_last_error() for this thread
void sj_set_error_message(const char *msg);

// ---------------------------------------------------------------- launchers
// primitives (sj_prims.cu)
size_t sj_scan_temp_bytes(uint64_t n);
cudaError_t sj_exclusive_scan_u32(const uint32_t *in, uint32_t *out, uint64_t n, void *temp,
                                  uint32_t *total_dev, cudaStream_t s);
// same, and sets every input element to zero after reading it
cudaError_t sj_exclusive_scan_u32_clear(uint32_t *in, uint32_t *out, uint64_t n, void *temp, uint32_t *total_dev,
                                        cudaStream_t s);
size_t sj_radix_temp_bytes(uint64_t n);
cudaError_t sj_radix_sort_u64_u32(uint64_t *keys, uint32_t *vals, uint64_t *keysAlt, uint32_t *valsAlt,
                                  uint64_t n, int bits, void *temp, int *resultInAlt, cudaStream_t s);
cudaError_t sj_radix_sort_u32_u32(uint32_t *keys, uint32_t *vals, uint32_t *keysAlt, uint32_t *valsAlt,
                                  uint64_t n, int bits, void *temp, int *resultInAlt, cudaStream_t s);
cudaError_t sj_hash_pairs(const int32_t *key, const int32_t *val, uint64_t m,
                          unsigned long long *hashOut, cudaStream_t s);

// keys of a batch from its row structure: key k owns [excl[k], excl[k+1])
// (excl[n] = *total); skipped when the batch's count exceeds cap.  longRuns
// (16-byte records, sj_expand_long_slots(cap) of them) and longCount are
// scratch for the runs too long for one warp.
cudaError_t sj_expand_keys(const uint32_t *excl, const uint32_t *total, uint64_t n, int32_t *outKey,
                           const unsigned long long *batchPairs, uint64_t cap, void *longRuns, uint32_t longCap,
                           uint32_t *longCount, int numSM, cudaStream_t s);
size_t sj_expand_long_slots(uint64_t cap);
// consumer fold of a device-resident batch with the key array written in the
// same pass: reads the values, writes the keys from the key runs (as
// sj_expand_keys), adds the pairs' set hash to *hashOut; skipped when the
// batch's count exceeds cap.  chunkKey: sj_fold_chunks(cap) entries of scratch.
size_t sj_fold_chunks(uint64_t cap);
// out[i] = (float)in[i]
cudaError_t sj_u32_to_f32(const uint32_t *in, uint64_t n, float *out, cudaStream_t s);
cudaError_t sj_fold(const uint32_t *excl, const uint32_t *total, uint64_t n, const int32_t *val, int32_t *outKey,
                    const unsigned long long *batchPairs, uint64_t cap, uint32_t *chunkKey,
                    unsigned long long *hashOut, int numSM, cudaStream_t s);
// appends a batch (values vals, key runs start[0..n], start[n] = *total) to a
// device CSR table rowPtr[n+1] / cols[colsCap]; fill[n] are the rows' cursors
cudaError_t sj_csr_append(const uint32_t *start, const uint32_t *total, uint64_t n, const int32_t *vals,
                          const uint64_t *rowPtr, uint32_t *fill, int32_t *cols, uint64_t colsCap,
                          unsigned long long *err, cudaStream_t s);

// index build (sj_index.cu)
cudaError_t sj_launch_minmax(const double *pts, uint64_t n, int D, double *minmax_dev, cudaStream_t s);
cudaError_t sj_launch_cell_keys(const double *pts, uint64_t n, sj_grid_dev g, uint64_t *keys, uint32_t *vals,
                                uint32_t *outOfGrid, cudaStream_t s);
cudaError_t sj_launch_cell_flags(const uint64_t *keys, uint64_t n, uint32_t *flags, cudaStream_t s);
cudaError_t sj_launch_cell_build(const uint64_t *keys, const uint32_t *cellIdxExcl, uint64_t n,
                                 uint32_t *cellStart, uint64_t *cellLid, cudaStream_t s);
cudaError_t sj_launch_gather(const double *pts, const uint32_t *ids, uint64_t n, int D, int Dp, double *xs,
                             cudaStream_t s);
cudaError_t sj_launch_cell_coords(const uint64_t *cellLid, uint32_t nCells, sj_grid_dev g, uint32_t *coord,
                                  cudaStream_t s);

// neighbour lists and features (sj_stencil.cu)
// pass 0: owned-neighbour counts, full-stencil candidates per cell (and their
// total, added to *candTotal) and features; pass 1: the owned lists
cudaError_t sj_launch_neighbours(const uint64_t *cellLid, const uint32_t *cellCoord, const uint32_t *cellStart,
                                 uint32_t nCells, sj_grid_dev g, int pattern, const uint32_t *nbrStart,
                                 uint32_t *nbrCountOrCell, uint64_t *candFull, unsigned long long *candTotal,
                                 float *feat, int pass, cudaStream_t s);

// join (sj_join.cu): the count pass (per-key pair counts, hit masks)
// (persistent queue: numSM x resident CTAs per SM, at most maxCtasPerSM when > 0)
cudaError_t sj_launch_join(const sj_join_args &a, const sj_grid_dev &g, int fp32, int queue, int numSM,
                           int maxCtasPerSM, cudaStream_t s);
// emission (sj_emit.cu): the values of the pairs from the recorded hit masks
// into their key runs; a.queueHead must be zero at launch
cudaError_t sj_launch_emit(const sj_join_args &a, int numSM, int maxCtasPerSM, cudaStream_t s);

// emission units of a task: one per group of 32 queries, plus one per block of
// 32 stream positions for a symmetric task
__host__ __device__ inline uint32_t sj_task_units(uint32_t qCount, uint32_t streamLen, bool sym)
{
    return (qCount + 31) / 32 + (sym ? (streamLen + 31) / 32 : 0u);
}

// device task builder (sj_tasks.cu)
cudaError_t sj_tg_groups(const sj_taskgen &g, uint32_t *cnt, cudaStream_t s);
// Per owned-neighbour entry of every cell: the exclusive prefixes of the
// neighbours' occupancy and of occupancy x offset-class weight (g.offW of the
// number of indexed coordinates in which the two cells differ), the entry's
// weight, and per cell the weighted total.
cudaError_t sj_nbr_spread(const uint32_t *cellStart, const uint32_t *cellCoord, const uint32_t *nbrStart,
                          const uint32_t *nbrCell, uint32_t nCells, const sj_grid_dev &g, uint32_t *nbrPre,
                          double *nbrPreW, float *nbrWt, double *cellW, cudaStream_t s);
cudaError_t sj_tg_cells(const sj_taskgen &g, const uint32_t *order, const uint8_t *workersAt, uint32_t *posCnt,
                        unsigned long long *posEv, unsigned long long *costKey, unsigned long long *totals,
                        cudaStream_t s);
cudaError_t sj_iota_u32(uint32_t *v, uint32_t n, cudaStream_t s);
// mode 8: workers per position from the exclusive prefix of the evaluations
// in cost order (evExcl[n] = total): 16, 8 or 2 by third of the work
cudaError_t sj_tg_thirds(const unsigned long long *evExcl, uint32_t n, uint8_t *workers, cudaStream_t s);
cudaError_t sj_tg_item_counts(const sj_taskgen &g, const uint32_t *order, uint32_t *items, cudaStream_t s);
cudaError_t sj_tg_item_tasks(const sj_taskgen &g, const uint32_t *order, const uint8_t *workersAt,
                             const uint32_t *itemStart, uint32_t nItems, uint32_t *itemTasks, cudaStream_t s);
cudaError_t sj_tg_item_write(const sj_taskgen &g, const uint32_t *order, const uint8_t *workersAt,
                             const uint32_t *itemStart, uint32_t nItems, const uint32_t *itemTaskStart,
                             sj_task *tasks, float *pred, cudaStream_t s);
cudaError_t sj_tg_shard(const sj_task *in, const float *predIn, uint32_t nOut, uint32_t idx, uint32_t cnt,
                        sj_task *out, float *predOut, cudaStream_t s);
// record offsets of a task list: out[0..6] = row-mask words, column-mask words,
// row offsets, candidate records, emission units, planned pairs
// (ceil(pred * (1 + alpha))), predicted pairs (rounded); each nt+1 entries
// (exclusive prefix, total last).  temp: sj_task_offsets_temp(nt) entries.
size_t sj_task_offsets_temp(uint32_t nt);
cudaError_t sj_task_offsets(const sj_task *tasks, const float *pred, uint32_t nt, double alpha,
                            unsigned long long *temp, unsigned long long *const out[7], cudaStream_t s);
// greedy batch plan over the offsets: start[0..nb] (start[nb] = nt), *nBatches
cudaError_t sj_plan_batches(unsigned long long *const off[7], uint32_t nt, unsigned long long cap,
                            unsigned long long maskLim, uint32_t *next, uint32_t *start, uint32_t *nBatches,
                            cudaStream_t s);
// per batch: predicted pairs, row-mask words, column-mask words, row offsets, candidate records
cudaError_t sj_plan_stats(const uint32_t *start, uint32_t nb, unsigned long long *const off[7],
                          unsigned long long *stats, cudaStream_t s);
// learned estimator: rates (2 per cell: home, owned neighbours) from the
// network's outputs (log2(1 + home hits), log2(1 + owned-neighbour hits))
cudaError_t sj_rates_mlp(const float *out, const uint32_t *cellStart, const uint32_t *nbrStart,
                         const uint32_t *nbrCell, uint32_t nCells, float *rate, cudaStream_t s);
// sampling estimator: per-cell rates (2 per cell: home, neighbours) from the
// sampled tasks' hits and evaluations; cellHits / cellEvals: 2 per cell;
// totals has sj_sample_totals_len() entries (per occupancy class and global,
// for the cells without a sample)
size_t sj_sample_totals_len();
cudaError_t sj_sample_rates(const sj_task *tasks, uint32_t nt, const uint32_t *taskHits, const uint32_t *taskEvals,
                            const uint32_t *cellStart, unsigned long long *cellHits, unsigned long long *cellEvals,
                            unsigned long long *totals, uint32_t nCells, float *rate, cudaStream_t s);
// sums[0] evaluations, [1] refined, [2] measured pairs; *errSum = sum |pred - measured|
cudaError_t sj_task_sums(const uint32_t *taskEvals, const uint32_t *taskRefined, const uint32_t *taskHits,
                         const float *pred, uint32_t nt, unsigned long long *sums, double *errSum, int numSM,
                         cudaStream_t s);
cudaError_t sj_cell_hits(const uint32_t *cellStart, const uint32_t *ids, const uint32_t *deg, uint32_t nCells,
                         unsigned long long *hits, cudaStream_t s);
// exclusive scan of n u64 values (out has n+1 entries, out[n] = total); temp: sj_scan64_temp(n) entries
size_t sj_scan64_temp(uint64_t n);
cudaError_t sj_exclusive_scan_u64(const unsigned long long *in, unsigned long long *out, uint64_t n,
                                  unsigned long long *temp, cudaStream_t s);

// estimators (sj_estimate.cu)
cudaError_t sj_launch_mlp_infer(const float *feat, uint32_t nCells, const float *weights, float *out,
                                cudaStream_t s);
cudaError_t sj_launch_mlp_train_step(const float *x, const float *y, uint32_t m, float *weights, float *grad,
                                     float *adamM, float *adamV, int step, float lr, float *lossOut,
                                     cudaStream_t s);
cudaError_t sj_launch_mlp_grad(const float *x, const float *y, uint32_t m, const float *weights, float *grad,
                               float *lossOut, cudaStream_t s);

// number of learned-estimator parameters (W1,b1,W2,b2,W3,b3)
#define SJ_MLP_NPARAM (SJ_NFEAT * SJ_HID + SJ_HID + SJ_HID * SJ_HID + SJ_HID + SJ_HID * SJ_NOUT + SJ_NOUT)
