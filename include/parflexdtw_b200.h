/*
 * parflexdtw_b200.h -- C ABI of the B200-native ParFlex alignment path.
 *
 * ParFlex ("sparse parallel FlexDTW") aligns two feature sequences through an
 * N x M cost matrix C cut into L x L tiles that overlap by one cell.
 * Stage 1 runs FlexDTW in every tile; stage 2 propagates accumulated cost and
 * path length across tile edges, scans the global top and right edges for
 * the best cost-per-length endpoint and stitches the per-tile backtraces into
 * one warping path.  Everything runs on the GPU; the host sees only the
 * result (and, on request, stage-2 intermediates).
 *
 * Conventions (all follow the reference, ishitajain21/ParFlexDTW):
 *   - C is row-major FP64, rows = frames of the first sequence, with leading
 *     dimension ldc >= M (elements).  Device pointers unless stated.
 *   - steps is n_steps (row, col) pairs, weights n_steps FP64 values.  The
 *     device kernels accept any ordered subset of {(1,1), (1,2), (2,1)}
 *     (the reference's default set, in any order); other steps return
 *     PFX_ERR_STEPS.
 *   - A warping path is K (row, col) pairs, int64, start first.
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).
 *   - Every function returns a pfx_status; pfx_last_error() describes the
 *     last failure of the calling thread.
 * One plan must not be used by two host threads at the same time.
 */
#ifndef PARFLEXDTW_B200_H
#define PARFLEXDTW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pfx_status {
    PFX_OK = 0,
    PFX_ERR_ARG = 1,          /* bad argument (the reference raises ValueError)   */
    PFX_ERR_STEPS = 2,        /* step set outside {(1,1),(1,2),(2,1)}              */
    PFX_ERR_CUDA = 3,         /* CUDA runtime error                                */
    PFX_ERR_NO_ENDPOINT = 4,  /* "Stage 2: No valid endpoint found on global
                                 top/right edges." (Parflex.py:1285-1286)          */
    PFX_ERR_TOO_LARGE = 5,    /* tile length beyond the kernel's on-chip limit     */
    PFX_ERR_NO_DEVICE = 6     /* no CUDA device                                    */
} pfx_status;

typedef struct pfx_plan pfx_plan;

/* DP precision of a plan.  PFX_FP64: the plain form, bit-exact with the
 * reference.  PFX_FP32: the chosen form -- FP32 cost (from a BF16 tensor-core
 * GEMM when built from features) and FP32 stage-1 DP; stage 2 stays FP64 on
 * the exactly widened FP32 edge values.  No reference counterpart. */
typedef enum pfx_precision { PFX_FP64 = 0, PFX_FP32 = 1 } pfx_precision;

/* Human-readable status and the calling thread's last error detail. */
const char *pfx_status_string(int status);
const char *pfx_last_error(void);

/* Library version as major*10000 + minor*100 + patch. */
int pfx_version(void);

/* Number of CUDA kernels this library has launched in this process (all
 * devices, all threads).  No reference counterpart: launch accounting for
 * benchmarks. */
int64_t pfx_kernel_launches(void);

/* ---------------------------------------------------------------------------
 * Plans.  A plan fixes (N, M, L, steps, weights) and owns the device
 * workspace of one alignment: stage-1 edge tensors and packed backpointers
 * (0.25 B per cell), the stage-2 slot arrays (n1*n2*2*L each), edge-scan and
 * stitch buffers.  Created on the current CUDA device.
 *
 * Replaces the per-call state of run_flexdtw_on_tiles / propagate_tile_edge_costs
 * / stage2_scan_and_stitch (Parflex.py:376-469, 862-912, 1229-1356;
 * Parflex_gpu.py:342-607, 247-339).
 * ------------------------------------------------------------------------- */
int pfx_plan_create(int64_t N, int64_t M, int32_t L, const int64_t *steps,
                    const double *weights, int32_t n_steps, pfx_plan **out);
/* pfx_plan_create with a precision (pfx_precision). */
int pfx_plan_create_ex(int64_t N, int64_t M, int32_t L, const int64_t *steps,
                       const double *weights, int32_t n_steps, int32_t precision,
                       pfx_plan **out);
void pfx_plan_destroy(pfx_plan *plan);

/* Stage-1 warps per tile CTA (4, 8 or 16; the plan picks one from its tile
 * count).  A masked run with few tiles is faster with 16.  No reference
 * counterpart. */
int pfx_plan_set_warps(pfx_plan *plan, int32_t nw);

/* info[0..7] = n1, n2, L, hop, n_steps, b_words_per_tile, device_bytes,
 * stage-1 warps per CTA. */
int pfx_plan_info(const pfx_plan *plan, int64_t *info);

/* Device buffers of a plan, for zero-copy views.  which: see pfx_buffer_id. */
typedef enum pfx_buffer_id {
    PFX_BUF_EDGE_D = 0,   /* f64 [n1][n2][2][L] stage-1 D on tile edges (+inf past the edge) */
    PFX_BUF_EDGE_P = 1,   /* i32 [n1][n2][2][L] stage-1 start encoding S on tile edges       */
    PFX_BUF_BACKPTR = 2,  /* u32 [n1*n2][b_words] packed 2-bit backpointers                   */
    PFX_BUF_EDGE_CF = 3,  /* f64 [n1][n2][2][L] C at each slot's start cell (edge_Cf_olap)    */
    PFX_BUF_VALID = 4,    /* u8  [n1][n2][2][L] sparse valid mask                             */
    PFX_BUF_D_ARR = 5,    /* f64 [n1][n2][2][L] accumulated cost after overlap sync           */
    PFX_BUF_L_ARR = 6,    /* f64 [n1][n2][2][L] path length after overlap sync                */
    PFX_BUF_TOP_D = 7,    /* f64 [M] */
    PFX_BUF_TOP_L = 8,    /* f64 [M] */
    PFX_BUF_RIGHT_D = 9,  /* f64 [N] */
    PFX_BUF_RIGHT_L = 10, /* f64 [N] */
    PFX_BUF_SEG_NORM = 11,/* f64 [2][max_segs] per-segment best cost/length               */
    PFX_BUF_SEG_META = 12,/* i64 [2][max_segs][6] ci cj edge idx grow gcol (-1 = none)    */
    PFX_BUF_D_PROP = 13,  /* f64 [n1][n2][2][L] snapshot before overlap sync (pfx_snapshot_prop) */
    PFX_BUF_L_PROP = 14,
    PFX_BUF_COST = 15,    /* f64 (f32 in the FP32 form) [n1*n2][strips][span][64]: the
                             tile-skewed cost slabs; element (k, tau, rho) of a tile is
                             C[r0 + 64k + rho][c0 + tau - rho], 0 outside the tile;
                             span = 16 * ceil((W + 63) / 16) of that tile, slab stride
                             that of an L x L tile */
    PFX_BUF_FEAT_BF16 = 16 /* bf16 [N + M][Kp] FP32 form: the L2-normalised features
                             the tensor-core cost GEMM read (rows of F1, then F2) */
} pfx_buffer_id;
int pfx_plan_buffer(pfx_plan *plan, int which, void **ptr, int64_t *nbytes);

/* ---------------------------------------------------------------------------
 * Stages.  All asynchronous on `stream`.
 * ------------------------------------------------------------------------- */

/* Loads the cost matrix into the plan's tile-skewed copy (the layout the
 * stage-1 kernel reads: per tile, 64-row strips with each row shifted by its
 * index, so one wavefront step of a warp reads 512 contiguous bytes; about
 * 1.03x the size of C).  From a row-major C (leading dimension ldc), or
 * directly from features: F1 d x N and F2 d x M row-major by feature (the
 * (d, frames) layout), any d >= 1, giving 1 - L2norm(F1)^T L2norm(F2) with
 * the same fixed-order FP64 sum as pfx_cost_matrix_f64
 * (cost_matrix_from_features_gpu, gpu_flexdtw.py:95-109; Parflex.py:1470). */
int pfx_plan_load_cost(pfx_plan *plan, const double *C, int64_t ldc, void *stream);
int pfx_plan_load_features(pfx_plan *plan, const double *F1, const double *F2,
                           int32_t d, void *stream);
/* FP32 plans: loads an FP32 row-major C (pfx_plan_load_cost on an FP32 plan
 * takes an FP64 C and rounds it to FP32).  Stage 2 of an FP32 plan always
 * reads the overlap costs from this FP32 copy. */
int pfx_plan_load_cost_f32(pfx_plan *plan, const float *C, int64_t ldc, void *stream);
/* FP32 plans: the chosen-form cost from features (F1 d x N, F2 d x M, FP64,
 * row-major by feature, 1 <= d <= 256): each frame is L2-normalised in FP64
 * and rounded to bf16, and C = 1 - A^T B is one BF16 x BF16 -> FP32
 * tensor-core GEMM (tcgen05, TMEM accumulator) whose epilogue writes the FP32
 * tile-skewed slabs directly.  Replaces cost_matrix_from_features_gpu
 * (gpu_flexdtw.py:95-109) in the FP32 form. */
int pfx_plan_load_features_bf16(pfx_plan *plan, const double *F1, const double *F2,
                                int32_t d, void *stream);

/* Restricts cost building (load_cost / load_features*), stage 1 and the
 * stage-2 overlap gather to the tiles set in mask[n1*n2] (row-major tile
 * index; device memory when on_device, else host); tiles outside it keep
 * +inf edge costs, so no stage-2 path crosses them.  mask NULL lifts the
 * restriction.  The masked tile queue is built on the device (no host
 * round trip when on_device).  Used by the learned tile-pruning proposer;
 * no reference counterpart. */
int pfx_plan_set_tile_mask(pfx_plan *plan, const uint8_t *mask, int32_t on_device,
                           void *stream);

/* Restrict the plan for good to tiles [lo, hi) of the tile order
 * (t = i * n2 + j): it allocates cost slabs for those tiles only, packed,
 * and works as a tile mask of that range that cannot be changed or lifted
 * (pfx_plan_set_tile_mask then fails).  Must come before any cost is
 * loaded.  For a pair whose tiles are sharded across devices, so that each
 * device holds the cost of its own tiles only; no reference counterpart. */
int pfx_plan_set_tile_range(pfx_plan *plan, int32_t lo, int32_t hi, void *stream);

/* Stage 1: FlexDTW on every tile (run_flexdtw_on_tiles, Parflex.py:376-469;
 * GPU variant flexdtw_chunk_from_global_C, gpu_flexdtw.py:288-402).  Writes D
 * and S on tile edges and the packed backpointers.  C non-null: loads it
 * first (pfx_plan_load_cost); C null: uses the loaded cost. */
int pfx_stage1(pfx_plan *plan, const double *C, int64_t ldc, void *stream);

/* Stage 2a: edge tensors, valid mask and cross-tile propagation
 * (propagate_tile_edge_costs, Parflex.py:862-912 / Parflex_gpu.py:247-339).
 * Overlap costs are read from C if non-null, else from the loaded cost. */
int pfx_stage2_propagate(pfx_plan *plan, const double *C, int64_t ldc, void *stream);

/* Stage 2a in two parts, for a pair whose tiles are sharded across devices
 * (each owner runs stage 1 and pfx_stage2_edges on its tiles under a tile
 * mask; one rank gathers edge_D, edge_P, edge_Cf and the OR of the valid
 * masks, then runs pfx_stage2_prop).  pfx_stage2_edges: edge tensors and
 * valid mask (_build_edge_data, Parflex.py:509-564; _build_valid_mask,
 * Parflex.py:582-624), the only part of stage 2 that reads the cost; it
 * also resets D_arr / L_arr to +inf.  pfx_stage2_prop: the cross-tile
 * propagation (Parflex.py:632-855).  pfx_stage2_propagate = both. */
int pfx_stage2_edges(pfx_plan *plan, const double *C, int64_t ldc, void *stream);
int pfx_stage2_prop(pfx_plan *plan, void *stream);

/* Copies D_arr / L_arr into the D_PROP / L_PROP buffers (test hook: the
 * state between propagation and overlap sync). */
int pfx_snapshot_prop(pfx_plan *plan, void *stream);

/* Stage 2b: overlap sync and global edge scan (sync_tile_overlap_edges,
 * Parflex.py:920-969; _nb_scan_edges, Parflex.py:1154-1222) with
 * buffer_global = min(N,M) * (1 - (1 - beta) * min(N,M) / max(N,M))
 * (Parflex.py:1520). */
int pfx_stage2_scan(pfx_plan *plan, double beta, void *stream);

/* Stage 2c: stitched backtrace (backtrace_and_stitch, Parflex.py:1032-1103)
 * from the scan's best endpoint (from_best = 1) or from tile (i, j), edge,
 * idx (from_best = 0). */
int pfx_stage2_stitch(pfx_plan *plan, int from_best, int64_t i, int64_t j,
                      int64_t edge, int64_t idx, void *stream);

/* The tile chain of the stitched backtrace alone (backtrace_and_stitch's
 * tile-to-tile walk, Parflex.py:1032-1103): reads only the start encodings
 * on the tile edges, not the backpointers, and copies the crossed tiles'
 * (i, j) into tiles_host[2 * k], [2 * k + 1] (cap >= 101 entries), end tile
 * first; *n_tiles = their number.  Synchronises `stream`.  A sharded pair
 * uses it to fetch only the crossed tiles' backpointers before
 * pfx_stage2_stitch. */
int pfx_stage2_chain(pfx_plan *plan, int from_best, int64_t i, int64_t j,
                     int64_t edge, int64_t idx, int32_t *tiles_host, int32_t cap,
                     int32_t *n_tiles, void *stream);

/* Stage 1 + 2a + 2b + 2c in one call on a device-resident C (or, with C
 * null, on the loaded cost). */
int pfx_parflex_device(pfx_plan *plan, const double *C, int64_t ldc,
                       double beta, void *stream);

/* Synchronises `stream` and reads the scan/stitch results: best normalised
 * cost, best_end[7] = (grow, gcol, ci, cj, edge, idx, found), path length. */
int pfx_result(pfx_plan *plan, void *stream, double *best_cost,
               int64_t *best_end7, int64_t *wp_len);

/* Copies the last stitched path (K x 2 int64, start first) into host memory
 * wp_host of capacity `cap` points (synchronises `stream`). */
int pfx_copy_path(pfx_plan *plan, void *stream, int64_t *wp_host, int64_t cap);

/* ---------------------------------------------------------------------------
 * One-call drop-ins.
 * ------------------------------------------------------------------------- */

/* parflex(C, steps, weights, beta, L) (Parflex.py:1510-1547,
 * Parflex_gpu.py:656-854) on a HOST cost matrix: copies C to the device,
 * runs both stages and copies the path back.  wp_out receives K x 2 int64
 * points (start first) if K <= wp_cap; *wp_len is always set. */
int pfx_parflex(const double *C_host, int64_t N, int64_t M, int64_t ldc,
                const int64_t *steps, const double *weights, int32_t n_steps,
                double beta, int32_t L, double *best_cost, int64_t *wp_out,
                int64_t wp_cap, int64_t *wp_len);

/* 1 - L2norm(F1)^T L2norm(F2) in FP64 with a fixed summation order
 * (cost_matrix_from_features_gpu, gpu_flexdtw.py:95-109; Parflex.py:1470).
 * F1 is d x N and F2 d x M, row-major by feature (the (d, frames) layout).
 * `norm_scratch` holds d*(N+M) doubles (the normalised features). */
int pfx_cost_matrix_f64(const double *F1, const double *F2, int32_t d,
                        int64_t N, int64_t M, double *norm_scratch, double *C,
                        int64_t ldc, void *stream);

/* FlexDTW.flexdtw's DP on one R x W tile of C with full outputs
 * (FlexDTW.py:326-370; flexdtw_chunk_from_global_C, gpu_flexdtw.py:288-402):
 * D (f64), P (int32 start encoding) and B (int8 step index, -1 when no step
 * won), each R x W row-major on the device. */
int pfx_flexdtw_tile(const double *C, int64_t ldc, int32_t R, int32_t W,
                     const int64_t *steps, const double *weights,
                     int32_t n_steps, double *D, int32_t *P, int8_t *B,
                     void *stream);

/* pfx_flexdtw_tile's DP with no device allocation: the same inputs and
 * outputs, but the kernel's scratch (tile edge rows and packed backpointers)
 * is a fixed ~1.1 MB device array inside the library instead of a
 * cudaMallocAsync per call.  For callers that cannot allocate device memory
 * (a real-time aligner that must not block on the allocator per audio block,
 * a host that reserves all device memory up front).  R and W at most 2048,
 * else PFX_ERR_TOO_LARGE.  All calls on a device share the array: calls that
 * overlap on the GPU race on it, so order them on one stream.  The first call
 * on each device (and in each new CUDA context of it, e.g. after a device
 * reset) looks up the array's address; make it before any stream capture.
 * No counterpart in the reference. */
int pfx_flexdtw_tile_noalloc(const double *C, int64_t ldc, int32_t R, int32_t W,
                             const int64_t *steps, const double *weights,
                             int32_t n_steps, double *D, int32_t *P, int8_t *B,
                             void *stream);

/* ---------------------------------------------------------------------------
 * Batches.  A batch aligns n pairs of feature sequences of uneven lengths
 * that share steps, weights, feature dimension d and DP precision
 * (pfx_precision; the FP32 form takes d <= 256 and builds its cost on the
 * tensor cores as pfx_plan_load_features_bf16 does); pair i has its
 * own shape (N[i], M[i]) and tile length L[i].  It owns, in one device
 * arena, a plan per pair (pfx_batch_plan), the raw feature inputs, one
 * pool of tile-skewed cost slabs and the stage-1 tile queues.
 *
 * By default the cost of every tile is built into the pool by separate
 * cost kernels first: pairs are packed into "waves" whose cost slabs fit the
 * pool (wave_bytes; 0 = 70 % of the device memory the batch's other buffers
 * leave free); per wave, the cost of every pair is built from its features,
 * ONE persistent stage-1 launch runs all tiles of all pairs of the wave
 * (largest first) from a device work queue, and stage 2 of the pairs runs
 * on forked streams, overlapping the next waves.
 *
 * With PFX_BATCH_TILE_COST in `precision` (FP64, d <= 16) the stage-1
 * kernel builds each tile's cost itself: the CTA that claims a tile writes
 * its cost into the CTA's own slab of the pool (one slab per resident CTA),
 * then runs the DP on it.  ONE persistent stage-1 launch then runs all
 * tiles of all pairs, whatever the batch's size, with a pool of about
 * 592 slabs instead of one per tile.
 *
 * pfx_batch_run records this whole sequence once into a CUDA graph and
 * replays it.
 *
 * The reference has no batch entry point: its notebooks loop over pairs
 * calling parflex / tiled_stage1_from_features + run_stage2_from_tiled
 * (Parflex.py:1466-1547; gpu_flexdtw.py:405-470).  Each pair's result is
 * that of those calls on the same pair.
 * ------------------------------------------------------------------------- */
typedef struct pfx_batch pfx_batch;

/* Flag for pfx_batch_create's `precision` (or-ed with PFX_FP64, d <= 16):
 * the stage-1 kernel builds each tile's cost itself, one launch for every
 * tile of every pair, instead of separate cost kernels filling slabs in
 * waves.  Same results; for batches whose slabs would need many waves. */
#define PFX_BATCH_TILE_COST 0x100
/* Flag for pfx_batch_create's `precision` (or-ed with PFX_FP64, not with
 * PFX_BATCH_TILE_COST): the cost is 1 - sum_f a_f b_f formed in the order
 * f = 0, 1, ..., d-1 as a chain of fused multiply-adds (the first product
 * rounded on its own), 13 FP64 operations per cell, instead of separately
 * rounded products and sums (24).  Another fixed, deterministic rounding of
 * the same cosine cost, as a BLAS product would form it; stage 1 and stage 2
 * are the same on either cost. */
#define PFX_BATCH_COST_FMA 0x200

/* nw: stage-1 warps per tile CTA (4, 8 or 16; 0 = chosen from the tile
 * count).  precision: a pfx_precision, optionally or-ed with
 * PFX_BATCH_TILE_COST or PFX_BATCH_COST_FMA.  The batch is created on the current CUDA device. */
int pfx_batch_create(int32_t n, const int64_t *N, const int64_t *M, const int32_t *L,
                     const int64_t *steps, const double *weights, int32_t n_steps,
                     int32_t d, int64_t wave_bytes, int32_t nw, int32_t precision,
                     pfx_batch **out);
void pfx_batch_destroy(pfx_batch *batch);
/* info[0..8] = n, waves, total tiles, DP cells (sum of tile R*W), device
 * bytes, stage-1 warps per CTA, largest wave's tiles, cost-slab pool bytes,
 * 1 when stage 1 builds each tile's cost itself (else 0). */
int pfx_batch_info(const pfx_batch *batch, int64_t *info);
/* Device input buffers of pair i: F1 (d x N[i]) and F2 (d x M[i]),
 * row-major by feature.  Fill them before pfx_batch_run (any stream, but
 * ordered before the run). */
int pfx_batch_features(pfx_batch *batch, int32_t i, double **F1, double **F2);
/* Copies pair i's features from host memory (F1: d x N[i], F2: d x M[i],
 * row-major by feature) into the batch's input buffers, asynchronously on
 * `stream` (page-locked host memory makes it truly asynchronous; a copy
 * into the same pair's buffers may be recorded into a CUDA graph, so that a
 * pair's upload overlaps the work on other pairs). */
int pfx_batch_load_async(pfx_batch *batch, int32_t i, const double *F1, const double *F2,
                         void *stream);
/* The plan of pair i (owned by the batch: do not destroy; do not load a
 * cost into it).  pfx_result / pfx_copy_path / pfx_plan_buffer read pair
 * i's results after pfx_batch_run. */
int pfx_batch_plan(pfx_batch *batch, int32_t i, pfx_plan **plan);
/* Restricts every pair to the tiles set in its mask (masks: the pairs' n1*n2
 * masks concatenated in pair order; device memory when on_device): cost
 * slabs are built and stage 1 runs only there (with separate cost kernels
 * the pool now holds only those slabs, so waves are repacked), other tiles
 * keep +inf edges.  For the
 * learned tile proposer; synchronises `stream`; invalidates the recorded
 * graph.  Either form (FP64 or FP32).  No reference counterpart. */
int pfx_batch_set_masks(pfx_batch *batch, const uint8_t *masks, int32_t on_device,
                        void *stream);
/* After a masked run: adds tiles to pair i's run and aligns it again.
 * `tiles` (host, n1*n2; nonzero = run) names the tiles to add, NULL every
 * tile (the full-tile method).  Stage 1 runs only on the added tiles that
 * have not run since the last pfx_batch_run (the others' outputs are
 * reused), the cost slabs of every run tile are rebuilt in the pool, and
 * stage 2 runs on the pair.  Its result is then read through
 * pfx_batch_plan + pfx_result / pfx_copy_path (until the next
 * pfx_batch_run).  The batch keeps its masks, queues and graph.
 * Synchronises `stream`.  No reference counterpart. */
int pfx_batch_complete(pfx_batch *batch, int32_t i, double beta, const uint8_t *tiles,
                       void *stream);
/* Aligns every pair (asynchronous on `stream`).  use_graph = 1 records the
 * launch sequence into a CUDA graph on the first call (and again when beta
 * changes) and replays it; 0 launches directly. */
int pfx_batch_run(pfx_batch *batch, double beta, int32_t use_graph, void *stream);
/* Device time (ms) of the phases of the last direct (use_graph = 0) run,
 * summed over waves: ms3[0] cost building from features, ms3[1] the stage-1
 * launches, ms3[2] stage 2 as far as it does not overlap later waves (the
 * edge gathers, plus the tail after the last wave's gather).
 * Waits for that run.  No reference counterpart (benchmark hook). */
int pfx_batch_timing(pfx_batch *batch, double *ms3);
/* Synchronises `stream` and copies every pair's result to host arrays:
 * best_cost[n], best_end7[7n] (as in pfx_result), wp_len[n].  Pairs whose
 * scan found no endpoint have best_end7[7i+6] = 0.  Fails if a stage-1
 * wait ran out (the whole batch is then invalid). */
int pfx_batch_results(pfx_batch *batch, void *stream, double *best_cost,
                      int64_t *best_end7, int64_t *wp_len);
/* Copies the paths of all pairs into host memory: pair i's K_i x 2 points
 * start at wp_host + 2*offsets[i] (offsets from the wp_len of
 * pfx_batch_results; capacity `cap` points in total).  Synchronises. */
int pfx_batch_copy_paths(pfx_batch *batch, void *stream, int64_t *wp_host,
                         const int64_t *offsets, int64_t cap);
/* As pfx_batch_copy_paths, with each path as two rows: pair i's K_i row
 * indices at host + 2*offsets[i], then its K_i column indices (lens[i] =
 * K_i from pfx_batch_results).  One device-side gather, one copy.
 * Synchronises. */
int pfx_batch_copy_paths_rows(pfx_batch *batch, void *stream, int64_t *host,
                              const int64_t *offsets, const int64_t *lens, int64_t cap);
/* Masked batch, after a run: the test that decides whether a pair's path
 * may have been cut off by its mask, on the device.  For every block of
 * margin x margin cells the path touches, the tiles that cover a cell of
 * it or of its 8 neighbouring blocks and were not run get near[t] = 1
 * (device, the pairs' (n1 x n2) tile arrays concatenated in pair order),
 * and the pair gets flags[i] = 1 (device, int32[n]).  Asynchronous on
 * `stream`.  No reference counterpart. */
int pfx_batch_check_paths(pfx_batch *batch, int32_t margin, uint8_t *near, int32_t *flags,
                          void *stream);

/* ---------------------------------------------------------------------------
 * Learned tile proposer (no reference counterpart).  A 3-layer CNN reads
 * the 16x average-pooled cost matrix and scores the tiles the optimal path
 * crosses; stage 1 then runs only on proposed tiles (pfx_plan_set_tile_mask)
 * and the full-tile method is the fallback.  These are its hand-written
 * inference and training kernels; images are one sample, [C][H][W], FP32
 * unless a *_bf16 flag selects bf16 activation storage (FP32 arithmetic).
 * All pointers are device memory; all calls are asynchronous on `stream`.
 * ------------------------------------------------------------------------- */
/* out (d x P, P = ceil(n / pool)): per block of `pool` frames, the mean of
 * the L2-normalised frames of F (d x n, FP64, row-major by feature). */
int pfx_pool_features(const double *F, int32_t d, int64_t n, int32_t pool, float *out,
                      void *stream);
/* out (P1 x P2) = 1 - A^T B for A (d x P1), B (d x P2), P1 <= 65535: with
 * pooled features, the block means of the cost matrix. */
int pfx_pooled_cost(const float *A, const float *B, int32_t d, int64_t P1, int64_t P2,
                    float *out, void *stream);
/* In place: x <- (x - row mean - column mean + mean) / std over the
 * P1 x P2 map (the proposer's input).  scratch: P1 + P2 + 2 floats. */
int pfx_pooled_center(float *x, int64_t P1, int64_t P2, float *scratch, void *stream);
/* The proposer's input without the P1 x P2 map: in place, A (d x P1) <-
 * -(A - its row means) / s and B (d x P2) <- B - its row means, where s is
 * the standard deviation of the double-centred map.  Then A^T B is the map
 * pfx_pooled_center makes from pfx_pooled_cost's 1 - A^T B (equal in real
 * arithmetic: the pooled cost is bilinear in the features; FP32 rounding
 * differs).  d <= 16.  scratch: pfx_pooled_center_scratch(P1, P2) bytes of
 * device memory (the chunks' moments; FP64 sums in a fixed order). */
int pfx_pooled_center_features(float *A, float *B, int32_t d, int64_t P1, int64_t P2,
                               void *scratch, void *stream);
/* Bytes of scratch pfx_pooled_center_features needs for a P1 x P2 map. */
int64_t pfx_pooled_center_scratch(int64_t P1, int64_t P2);
/* pfx_conv3x3_forward's first layer (Cin = 1, Cout = 32) on the map
 * x = A^T B (H = P1 rows, W = P2 columns), computed per input patch from the
 * features instead of read from memory.  d <= 16. */
int pfx_conv3x3_forward_features(const float *A, const float *B, int32_t d, int32_t H,
                                 int32_t W, const float *w, const float *b, int32_t Cout,
                                 int32_t stride, int32_t relu, void *y, int32_t y_bf16,
                                 void *stream);
/* y (Cout x Ho x Wo) = act(conv3x3(x) + b), zero padding 1, stride 1, 2 or 4,
 * Ho = (H - 1) / stride + 1; w is [Cout][Cin][3][3]; act = ReLU if relu. */
int pfx_conv3x3_forward(const void *x, int32_t x_bf16, int32_t Cin, int32_t H, int32_t W,
                        const float *w, const float *b, int32_t Cout, int32_t stride,
                        int32_t relu, void *y, int32_t y_bf16, void *stream);
/* Backward of pfx_conv3x3_forward (FP32, Cout <= 64): from dy (gradient at y)
 * and the forward's x and y: dx (overwritten; may be NULL), dw and db
 * (accumulated). */
int pfx_conv3x3_backward(const float *x, int32_t Cin, int32_t H, int32_t W, const float *w,
                         int32_t Cout, int32_t stride, const float *y, int32_t relu,
                         const float *dy, float *dx, float *dw, float *db, void *stream);
/* score[t] = max of the logit map (H x W, `fpp` frames per pixel) over the
 * region of tile t of an N x M alignment cut with tile length L and hop;
 * argmax[t] = the flat pixel index of that max (lowest on ties). */
int pfx_tile_max(const float *logits, int32_t H, int32_t W, int32_t n1, int32_t n2,
                 int64_t hop, int64_t L, int64_t N, int64_t M, int32_t fpp, float *score,
                 int32_t *argmax, void *stream);
/* Weighted BCE with logits over n tiles: *loss += mean loss, dscore = its
 * gradient (positives weighted by pos_weight). */
int pfx_tile_bce(const float *score, const uint8_t *label, int32_t n, float pos_weight,
                 float *loss, float *dscore, void *stream);
/* dlogits[argmax[t]] += dscore[t] (dlogits zeroed by the caller). */
int pfx_tile_max_backward(const float *dscore, const int32_t *argmax, int32_t n,
                          float *dlogits, void *stream);
/* One Adam update (bias-corrected, step >= 1) of n parameters. */
int pfx_adam_step(float *param, const float *grad, float *m, float *v, int64_t n, float lr,
                  float beta1, float beta2, float eps, int32_t step, void *stream);
/* mask[t] = 1 if some tile within distance `dilation` of t (Chebyshev, or
 * Manhattan when `manhattan`) has score > threshold. */
int pfx_tile_mask_from_scores(const float *score, int32_t n1, int32_t n2, float threshold,
                              int32_t dilation, int32_t manhattan, uint8_t *mask,
                              void *stream);

#ifdef __cplusplus
}
#endif
#endif /* PARFLEXDTW_B200_H */
