// Shared definitions for the ParFlex B200 kernels.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/parflexdtw_b200.h"

namespace pfx {

// Tile-grid geometry and DP parameters, passed by value to every kernel.
// Matches the reference tiling: hop = L - 1, tile (i, j) covers rows
// [i*hop, min(i*hop + L, N)) and columns [j*hop, min(j*hop + L, M))
// (Parflex.py:388-431).
struct Geo {
    int64_t N, M;      // cost-matrix rows (F1 frames) and columns (F2 frames)
    int64_t ldc;       // leading dimension of C (elements)
    int32_t L, hop;    // tile length and hop
    int32_t n1, n2;    // tile rows / tile columns
    int32_t S;         // number of steps (1..3)
    int32_t kind[3];   // per step: 0 = (1,1), 1 = (1,2), 2 = (2,1)
    double w[3];       // per step weight
    int64_t b_words;   // packed-backpointer words reserved per tile
};

__host__ __device__ inline int64_t ceil_div64(int64_t a, int64_t b) { return (a + b - 1) / b; }

#ifdef __CUDACC__
// 8-byte asynchronous global -> shared copy (cp.async); `full` false writes 8
// zero bytes and reads nothing (src must still be a valid address).  Copies
// of a thread complete at cp_async_wait_all(); a barrier after it publishes
// them to the CTA.
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool full) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src),
                 "r"(full ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
}
#endif
__host__ __device__ inline int32_t ceil_div32(int32_t a, int32_t b) { return (a + b - 1) / b; }

__host__ __device__ inline void tile_rect(const Geo& g, int ti, int tj, int64_t* r0, int64_t* c0,
                                          int32_t* R, int32_t* W) {
    *r0 = (int64_t)ti * g.hop;
    *c0 = (int64_t)tj * g.hop;
    int64_t R_ = g.N - *r0, W_ = g.M - *c0;
    *R = (int32_t)(R_ < g.L ? R_ : g.L);
    *W = (int32_t)(W_ < g.L ? W_ : g.L);
}

// Stage-1 wavefront schedule of one tile (see stage1_f64.cu): strips of 32
// rows, each strip sweeps "local time" tau = c + lane over span steps, strip k
// starts lag*k steps after the CTA starts.  Backpointers are packed 2 bits per
// cell into 32-bit words laid out [strip][period][lane], one period = 16
// consecutive local-time steps of one lane (row).
constexpr int kBlk = 16;  // steps between CTA barriers == cells per B word
struct Sched {
    int32_t nS, span, nP, lag;
};
__host__ __device__ inline Sched make_sched(int32_t R, int32_t W, int32_t nwarps) {
    Sched s;
    s.nS = ceil_div32(R, 32);
    s.span = ceil_div32(W + 31, kBlk) * kBlk;
    s.nP = s.span / kBlk;
    int32_t lag = ceil_div32(ceil_div32(s.span, nwarps), kBlk) * kBlk;
    s.lag = lag < 48 ? 48 : lag;
    return s;
}
// Words one tile of at most L x L cells needs.
__host__ __device__ inline int64_t tile_b_words(int32_t L) {
    Sched s = make_sched(L, L, 1);
    return (int64_t)s.nS * s.nP * 32;
}
// Backpointer code of cell (r, c) of a tile with W columns, from its word slab.
__device__ __forceinline__ int bp_code(const uint32_t* __restrict__ slab, int32_t W, int32_t r,
                                       int32_t c) {
    const int32_t nP = ceil_div32(W + 31, kBlk);
    const int32_t k = r >> 5, lane = r & 31, tau = c + lane;
    const uint32_t word = __ldg(slab + ((int64_t)k * nP + (tau >> 4)) * 32 + lane);
    return (int)((word >> ((tau & 15) * 2)) & 3u);
}

// ---------------------------------------------------------------------------
// Stage-1 schedule with two rows per lane (the plan path).  A strip is 64
// tile rows; lane i of a strip owns rows 64k+2i ("A") and 64k+2i+1 ("B") and
// at local step tau computes (64k+2i, tau-2i) and (64k+2i+1, tau-2i-1), i.e.
// row rho = r mod 64 at column tau - rho.  Backpointer words are laid out
// [strip][period][lane][A|B] (two consecutive words per lane per period).
constexpr int kStripRows = 64;
struct Sched2 {
    int32_t nS, span, nP, lag;
};
__host__ __device__ inline Sched2 make_sched2(int32_t R, int32_t W, int32_t nwarps) {
    Sched2 s;
    s.nS = ceil_div32(R, kStripRows);
    s.span = ceil_div32(W + kStripRows - 1, kBlk) * kBlk;
    s.nP = s.span / kBlk;
    int32_t lag = ceil_div32(ceil_div32(s.span, nwarps), kBlk) * kBlk;
    s.lag = lag < 80 ? 80 : lag;
    return s;
}
__host__ __device__ inline int64_t tile_b_words2(int32_t L) {
    const Sched2 s = make_sched2(L, L, 1);
    return (int64_t)s.nS * s.nP * 2 * 32;
}
// Tile-skewed cost layout: per tile, element (strip k, step tau, lane, half)
// = C[r0 + 64k + 2*lane + half][c0 + tau - 2*lane - half] (0 outside the
// tile), stored at ((k*span + tau)*32 + lane)*2 + half, so one warp-step of
// the stage-1 kernel reads 512 contiguous bytes.  Slab stride per tile is the
// size of an L x L tile.
__host__ __device__ inline int64_t skew_slab_elems(int32_t L) {
    const Sched2 s = make_sched2(L, L, 1);
    return (int64_t)s.nS * s.span * 2 * 32;
}
__host__ __device__ inline int64_t skew_index(int32_t W, int32_t r, int32_t c) {
    const int32_t span = ceil_div32(W + kStripRows - 1, kBlk) * kBlk;
    const int32_t k = r >> 6, rho = r & 63, tau = c + rho;
    return (((int64_t)k * span + tau) * 32 + (rho >> 1)) * 2 + (rho & 1);
}
// Backpointer code of cell (r, c) of a tile with W columns (two-row layout).
__device__ __forceinline__ int64_t bp_word_index2(int32_t W, int32_t r, int32_t tau) {
    const int32_t nP = ceil_div32(W + kStripRows - 1, kBlk);
    const int32_t k = r >> 6, rho = r & 63;
    return (((int64_t)k * nP + (tau >> 4)) * 32 + (rho >> 1)) * 2 + (rho & 1);
}

// Stage-1 outputs.
struct S1Out {
    double* edge_D;   // [tiles][2][L] D on the top / right edge, +inf past the edge
    int32_t* edge_P;  // [tiles][2][L] start encoding on the edges
    uint32_t* Bw;     // [tiles][b_words] packed backpointers
    double* full_D;   // single-tile full outputs (R x W), or null
    int32_t* full_P;
    int8_t* full_B;
    int32_t* status;  // set non-zero by a kernel whose bounded wait ran out, or null
};

// One stage-1 work item: a tile of one alignment, with the addresses of its
// inputs and outputs (the stage-1 kernel claims these from a device queue).
struct TileDesc {
    const void* Csk;    // tile-skewed cost slab (FP64, or FP32 in the FP32 form)
    uint32_t* Bw;       // packed backpointers
    double* eD;         // [2][L] D on the top / right edge
    int32_t* eP;        // [2][L] start encodings on the edges
    int32_t R, W;       // tile rows / columns
    int32_t L;          // edge-array stride (the alignment's tile length)
    int32_t tile;       // tile index within its alignment (row-major)
    // normalised features of the tile's first row / first column, feature f
    // of frame r at fa[f * lda + r] (fb: ldb); read when the stage-1 kernel
    // builds the tile's cost itself (null otherwise)
    const double* fa;
    const double* fb;
    int32_t lda, ldb;
};

// Stage 1 building each tile's FP64 cost itself (d > 0): a CTA writes the
// tile-skewed cost of the tile it claimed into its own slot of `slots`
// (`stride` doubles per slot, one slot per resident CTA: nslots), then runs
// the DP on it.  d = 0: the cost slabs come with the descriptors.
struct CostGen {
    double* slots;
    int64_t stride;
    int32_t nslots;
    int32_t d;
};
constexpr int kGenMaxD = 16;  // feature dimensions the in-kernel cost takes

// Status word values written by kernels.
constexpr int32_t kStatusWaitTimeout = 1;

// Stage-2 device state.  Slot arrays are [n1][n2][2][L].
struct S2Buf {
    const double* edge_D;
    const int32_t* edge_P;
    const uint32_t* Bw;
    double* edge_Cf;     // C at each slot's start cell
    uint8_t* valid;      // sparse compute mask
    double* D_arr;
    double* L_arr;
    double* top_D;       // [M]
    double* top_L;
    double* right_D;     // [N]
    double* right_L;
    double* seg_norm;    // [2][max_segs]
    int64_t* seg_meta;   // [2][max_segs][6] ci cj et idx grow gcol
    int32_t max_segs;
    double* best;        // [1]
    int64_t* best_end;   // [7] grow gcol ci cj et idx found
    int32_t* chain;      // [101][12]
    int32_t* chain_len;  // [1]
    int32_t* seg_pts;    // [101][seg_cap][2]
    int32_t* seg_len;    // [101]
    int64_t seg_cap;
    int64_t* wp;         // [K][2] final path, start first
    int64_t* wp_len;     // [1]
    const int32_t* tile_slot;  // [n1*n2] cost slab of each tile, -1 where stage 1
                               // skipped the tile (null: slab = tile index)
};

// Records `msg` as the calling thread's last error and returns `status`.
int report_status(int status, const char* msg);
// Parses a step list into Geo::S / kind / w (PFX_OK or PFX_ERR_STEPS).
int parse_step_kinds(const int64_t* steps, const double* weights, int32_t n, Geo* g);

// Count of kernels this library has launched (process-wide).
void count_launches(int n);

// Launchers (stage1_f64.cu, stage1_v3.cu, layout.cu, stage2.cu, cost.cu).
// Stage-1 queue kernel over `ntiles` descriptors (all sharing the step set and
// weights of g; tiles at most g.L x g.L); `*head` must be 0 at launch; nw in
// {4, 8, 16} warps per tile.
// `ntiles_dev` (nullable): the queue length read on the device (at most ntiles).
// `gen` (FP64 only, nullable or d = 0: off): every CTA builds the cost of
// the tile it claims from the descriptors' features into its slot of
// gen->slots, which must hold stage1_gen_slots(g, nw, gen->d) slots.
cudaError_t launch_stage1_queue(const TileDesc* descs, int ntiles, const int* ntiles_dev,
                                int* head, const Geo& g, int32_t* status, int nw, bool fp32,
                                cudaStream_t st, const CostGen* gen = nullptr);
// Cost slots the in-kernel-cost form of the queue kernel needs: the CTAs
// that can be resident at once (0: it does not fit).
int stage1_gen_slots(const Geo& g, int nw, int d);
// slot[t] = mask[t] ? t : -1.
cudaError_t launch_mask_slots(const uint8_t* mask, int n, int32_t* slot, cudaStream_t st);
// Keeps the descriptors whose tile is set in `mask`, in order; *count = kept.
cudaError_t launch_compact_descs(const TileDesc* in, int n, const uint8_t* mask, TileDesc* out,
                                 int* count, cudaStream_t st);
// Stage 1 of descs[0, ntiles) on clusters of two 16-warp CTAs (32 warps per
// tile), claimed through *head; for alignments with fewer tiles than SMs.
cudaError_t launch_stage1_cluster(const TileDesc* descs, int ntiles, int* head, const Geo& g,
                                  int32_t* status, bool fp32, cudaStream_t st);
// Clusters of that kernel that can run at once on this device (0: none).
int stage1_cluster_max(const Geo& g, bool fp32);
// Smallest valid warps-per-tile choice heuristic for `ntiles` tiles of length L.
int stage1_queue_warps(int ntiles, int32_t L, int num_sms);
// Cost-building launchers take an optional slot map: tile t's slab is slab
// slot[t] of Csk, and tiles with slot[t] < 0 are skipped (null: slab = t).
// The feature launchers also take an optional list of the nlist tiles to
// build (no CTAs are launched for the others).
cudaError_t launch_relayout_skew(const double* C, int64_t ldc, const Geo& g, double* Csk,
                                 int64_t skew_stride, cudaStream_t st,
                                 const int32_t* slot = nullptr);
// One pair of a multi-pair cost GEMM launch (gemm_bf16.cu): its operands'
// tensor maps, geometry and output slabs, and its first block in the launch.
struct GPair {
    CUtensorMap ma, mb;
    Geo g;
    float* Csk;
    int64_t stride, blk0;
    int32_t nkk, ncb;
};
// Fills *out for pair (A: N x Kp bf16 rows, B: M x Kp) into Csk; returns its
// number of blocks (0 on failure to encode the tensor maps).
int64_t gemm_pair_setup(const void* Abf, const void* Bbf, int Kp, const Geo& g, float* Csk,
                        int64_t stride, int64_t blk0, GPair* out);
// The cost GEMM of npairs pairs (a device table, blocks numbered by blk0) in
// one persistent launch.
cudaError_t launch_gemm_cost_multi(const GPair* pairs, int npairs, int64_t nblk, int Kp,
                                   int32_t* status, cudaStream_t st);
// FP32 form cost from features (gemm_bf16.cu): bf16 rows of L2-normalised
// features, then 1 - A B^T on the tensor cores into FP32 skewed slabs.  cap:
// FP32 elements available from Csk (< 0: n1 * n2 slabs); stores beyond it are
// skipped and flagged in *status.
cudaError_t launch_features_bf16(const double* F, int d, int64_t n, int Kp, void* out,
                                 cudaStream_t st);
// Several feature matrices in one launch: segment s converts F (d x n) into
// out, its blocks numbered from blk0 (features_bf16_blocks(n) per segment,
// segments in order of blk0).
struct FbSeg {
    const double* F;
    int64_t n;
    void* out;
    int64_t blk0;
};
int64_t features_bf16_blocks(int64_t n);
cudaError_t launch_features_bf16_segs(const FbSeg* segs, int nseg, int64_t blocks, int d, int Kp,
                                      cudaStream_t st);
cudaError_t launch_gemm_cost_skew(const void* Abf, const void* Bbf, int Kp, const Geo& g,
                                  float* Csk, int64_t stride, int32_t* status, cudaStream_t st,
                                  const int32_t* slot = nullptr, const int32_t* list = nullptr,
                                  int nlist = 0, int64_t cap = -1);
// FP32 slabs from a row-major FP64 (rounded) or FP32 C (exactly one non-null).
cudaError_t launch_relayout_skew_f32(const double* C64, const float* C32, int64_t ldc,
                                     const Geo& g, float* Csk, int64_t stride, cudaStream_t st,
                                     const int32_t* slot = nullptr);
// fma: the cost as a fixed-order chain of fused multiply-adds (13 FP64
// operations per cell) instead of separately rounded products and sums.
cudaError_t launch_cost_skew(const double* An, const double* Bn, int d, const Geo& g, double* Csk,
                             int64_t skew_stride, cudaStream_t st, const int32_t* slot = nullptr,
                             const int32_t* list = nullptr, int nlist = 0, bool fma = false);
cudaError_t launch_l2norm(const double* F, int d, int64_t n, double* out, cudaStream_t st);
cudaError_t launch_stage1(const double* C, const Geo& g, const S1Out& o, int tile0, int ntiles,
                          int nw, bool full, cudaStream_t st);
size_t stage1_smem_bytes_host(int32_t L, int nw);
int stage1_pick_warps(const Geo& g, int num_sms);
cudaError_t launch_fill(double* p, int64_t n, double v, cudaStream_t st);
cudaError_t launch_stage2(const double* C, const void* Csk, int64_t skew_stride, bool f32,
                          const Geo& g, const S2Buf& b, cudaStream_t st);
// launch_stage2 in two parts: the edge tensors (the only part that reads the
// cost slabs) and the cross-tile propagation.
// With An (normalised features, [d][N] and [d][M]) the overlap costs are
// computed from the features in the cost kernels' order, not read from C or
// the slabs (a batch whose stage 1 built its cost itself keeps no slabs).
cudaError_t launch_stage2_edges(const double* C, const void* Csk, int64_t skew_stride, bool f32,
                                const Geo& g, const S2Buf& b, cudaStream_t st,
                                const double* An = nullptr, const double* Bn = nullptr,
                                int d = 0);
cudaError_t launch_stage2_prop(const Geo& g, const S2Buf& b, cudaStream_t st);
cudaError_t launch_sync_scan(const Geo& g, const S2Buf& b, int64_t buf, cudaStream_t st);
cudaError_t launch_stitch(const Geo& g, const S2Buf& b, cudaStream_t st, int from_best,
                          int64_t si, int64_t sj, int64_t se, int64_t sx);
// The tile chain of the stitched backtrace alone (b.chain, b.chain_len): it
// reads only the start encodings on the tile edges, never the backpointers.
cudaError_t launch_stitch_chain(const Geo& g, const S2Buf& b, cudaStream_t st, int from_best,
                                int64_t si, int64_t sj, int64_t se, int64_t sx);
cudaError_t launch_cost_f64(const double* F1, const double* F2, int d, int64_t N, int64_t M,
                            double* An, double* Bn, double* C, int64_t ldc, cudaStream_t st);

}  // namespace pfx
