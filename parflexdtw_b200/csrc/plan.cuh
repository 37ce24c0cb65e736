// Plan object behind the opaque pfx_plan handle of the C ABI, shared by the
// single-alignment entry points (capi.cu) and the batch (batch.cu).
#pragma once

#include "common.cuh"

struct pfx_plan {
    pfx::Geo g;
    int nw;  // warps per tile CTA of the stage-1 kernel
    int device;
    size_t bytes;
    pfx::S1Out s1;
    pfx::S2Buf s2;
    double* D_prop;
    double* L_prop;
    int64_t n4;  // n1*n2*2*L
    void* blocks[40];
    int nblocks;
    // tile-skewed cost (allocated on first load, or attached by a batch) and
    // normalised features
    void* Csk;            // FP64 slabs, or FP32 in the FP32 form
    int64_t skew_stride;  // elements per tile slab
    int fp32;             // 1: FP32 form (FP32 cost slabs and stage-1 DP)
    double* feat;         // d*(N+M) doubles
    int feat_d;
    void* fbf;            // FP32 form: bf16 features, [N + M][fbf_kp]
    int fbf_kp;
    int cost_loaded;
    int gen_cost;         // batch plan whose stage 1 builds each tile's cost from feat
                          // (no slabs kept: Csk is null)
    // stage-1 tile queue of this plan (descriptors in queue order) and its head
    pfx::TileDesc* descs;
    int* head;
    // stage 1 of few tiles: the largest on 2-CTA clusters, the rest on single
    // CTAs in a second stream (created on first use, plans outside a batch)
    int* head2;
    cudaStream_t aux;
    cudaEvent_t ev_fork, ev_join;
    // tile mask (pfx_plan_set_tile_mask or a masked batch): the mask, each
    // tile's cost slab (-1: skipped), the masked queue and its device length
    uint8_t* tile_mask;
    int32_t* tile_slot;
    int32_t* tile_list;  // masked batch: the kept tiles in tile order, n_kept of them
    int32_t n_kept;
    pfx::TileDesc* descs_sub;
    int* nsub;
    int mask_active;
    // tile range (pfx_plan_set_tile_range): cost slabs only for tiles
    // [range_lo, range_hi), packed; range_hi == 0 means every tile has a slab
    int32_t range_lo, range_hi;
    // arena allocation: 0 = cudaMalloc per buffer, 1 = count bytes only,
    // 2 = carve from `arena`
    int arena_mode;
    char* arena;
    size_t arena_off;
};

namespace pfx {
int plan_init(pfx_plan* p, int64_t N, int64_t M, int32_t L, const int64_t* steps,
              const double* weights, int32_t n_steps, int nw, int fp32);
// Descriptors of every tile, largest first; with a host slot map, tile t's
// slab is slab slot[t] of Csk (nullptr where slot[t] < 0).
void plan_tile_descs(const pfx_plan* p, const void* Csk, TileDesc* out,
                     const int32_t* slot = nullptr);
inline int64_t plan_slab_bytes(const pfx_plan* p) {
    const int64_t slabs = p->range_hi > 0 ? (int64_t)p->range_hi - p->range_lo
                                          : (int64_t)p->g.n1 * p->g.n2;
    return slabs * p->skew_stride * (p->fp32 ? 4 : 8);
}
int num_sms_cur();
}  // namespace pfx
