// Batches of alignments: many pairs of uneven lengths, one persistent stage-1
// launch per wave, stage 2 on forked streams, all recorded into a CUDA graph.
//
// The reference aligns one pair per call (Parflex.py:1466-1547,
// gpu_flexdtw.py:405-470); a batch gives every pair exactly the result of
// those calls.  Device memory: one arena holds every pair's plan buffers
// (edge tensors, 2-bit backpointers, stage-2 slots), raw and normalised
// features, the tile queues and the result block; one pool holds the
// tile-skewed FP64 cost slabs of one wave.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "plan.cuh"

using namespace pfx;

namespace {

constexpr int kSide = 32;     // streams stage 2 of a wave is spread over
constexpr int kCostSide = 3;  // extra streams a wave's per-pair cost work is spread over

struct PairOut {
    const double* best;
    const int64_t* best_end;
    const int64_t* wp_len;
};

// One host-to-device upload scattered to many buffers: segment s copies
// segs[s].bytes bytes from base + segs[s].src to segs[s].dst (16-byte words
// where both ends are aligned).
struct CopySeg {
    int64_t src;
    void* dst;
    int64_t bytes;
};
constexpr int64_t kSegChunk = 1 << 16;  // bytes per segment (one CTA each)

__global__ void __launch_bounds__(256) k_scatter_segments(const char* __restrict__ base,
                                                          const CopySeg* __restrict__ segs,
                                                          int nseg) {
    if ((int)blockIdx.x >= nseg) return;
    const CopySeg g = segs[blockIdx.x];
    const char* src = base + g.src;
    char* dst = static_cast<char*>(g.dst);
    int64_t done = 0;
    if (((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0) {
        const int64_t n16 = g.bytes >> 4;
        const int4* s4 = reinterpret_cast<const int4*>(src);
        int4* d4 = reinterpret_cast<int4*>(dst);
        for (int64_t i = threadIdx.x; i < n16; i += blockDim.x) d4[i] = s4[i];
        done = n16 << 4;
    }
    for (int64_t i = done + threadIdx.x; i < g.bytes; i += blockDim.x) dst[i] = src[i];
}

__global__ void k_gather_results(const PairOut* __restrict__ po, int n, int64_t* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const PairOut p = po[i];
    int64_t* o = out + (int64_t)i * 9;
    o[0] = __double_as_longlong(*p.best);
    for (int k = 0; k < 7; ++k) o[1 + k] = p.best_end[k];
    o[8] = *p.wp_len;
}

// Per pair: its stitched path, tile mask and geometry (path checks and copies).
struct PathRef {
    const int64_t* wp;    // [K][2]
    const int64_t* len;   // K
    const uint8_t* mask;  // [n1 * n2] tiles run by the mask
    int64_t N, M;
    int32_t n1, n2, L, pad;
    int64_t tile_off;  // offset of the pair's tiles in concatenated per-tile arrays
    int64_t row_off;   // offset of the pair's block rows in the row scratch
};

// Block rows of `B` path rows: the column of the first and of the last path
// point in each (the path is monotone, so they bound its interval).
__global__ void k_path_rows(const PathRef* __restrict__ pr, int B, int32_t* __restrict__ lo,
                            int32_t* __restrict__ hi) {
    const PathRef q = pr[blockIdx.y];
    const int64_t K = *q.len;
    const int64_t* wp = q.wp;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < K;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = wp[2 * k] / B;
        if (k == 0 || wp[2 * (k - 1)] / B != a) lo[q.row_off + a] = (int32_t)wp[2 * k + 1];
        if (k == K - 1 || wp[2 * (k + 1)] / B != a) hi[q.row_off + a] = (int32_t)wp[2 * k + 1];
    }
}

// Tiles not run by the mask that cover a cell of the 3 x 3 block
// neighbourhood of a block the path touches: near[tile] = 1, flag[pair] = 1.
__global__ void k_path_near(const PathRef* __restrict__ pr, int B, const int32_t* __restrict__ lo,
                            const int32_t* __restrict__ hi, uint8_t* __restrict__ near,
                            int32_t* __restrict__ flag) {
    const PathRef q = pr[blockIdx.y];
    const int64_t K = *q.len;
    if (K <= 0) return;
    const int64_t a0 = q.wp[0] / B, a1 = q.wp[2 * (K - 1)] / B;
    const int64_t hop = q.L - 1;
    auto lo_tile = [&](int64_t x0, int n) {  // first tile whose cells reach x0
        const int64_t x = x0 - (q.L - 1);
        const int64_t t = x <= 0 ? 0 : (x + hop - 1) / hop;
        return (int)(t < n - 1 ? t : n - 1);
    };
    auto hi_tile = [&](int64_t x1, int n) {  // last tile starting at or before x1
        const int64_t t = x1 / hop;
        return (int)(t < n - 1 ? t : n - 1);
    };
    for (int64_t a = a0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; a <= a1;
         a += (int64_t)gridDim.x * blockDim.x) {
        const int32_t cl = lo[q.row_off + a], ch = hi[q.row_off + a];
        if (cl < 0 || ch < 0) continue;  // no path point in this block row
        const int64_t r0 = (a - 1 > 0 ? a - 1 : 0) * B;
        const int64_t r1 = ((a + 2) * B < q.N ? (a + 2) * B : q.N) - 1;
        const int64_t bl = cl / B - 1;
        const int64_t c0 = (bl > 0 ? bl : 0) * B;
        const int64_t c1 = ((ch / B + 2) * B < q.M ? (ch / B + 2) * B : q.M) - 1;
        const int ilo = lo_tile(r0, q.n1), ihi = hi_tile(r1, q.n1);
        const int jlo = lo_tile(c0, q.n2), jhi = hi_tile(c1, q.n2);
        bool any = false;
        for (int i = ilo; i <= ihi; ++i)
            for (int j = jlo; j <= jhi; ++j) {
                const int t = i * q.n2 + j;
                if (!q.mask[t]) {
                    near[q.tile_off + t] = 1;
                    any = true;
                }
            }
        if (any) flag[blockIdx.y] = 1;
    }
}

// Paths as rows: pair p's K points go to out[2 o_p .. 2 o_p + 2K) as K row
// indices then K column indices.
__global__ void k_path_to_rows(const PathRef* __restrict__ pr, const int64_t* __restrict__ offs,
                               const int64_t* __restrict__ lens, int64_t* __restrict__ out) {
    const PathRef q = pr[blockIdx.y];
    const int64_t Kd = *q.len, Kh = lens[blockIdx.y];
    const int64_t K = Kd < Kh ? Kd : Kh;
    int64_t* o = out + 2 * offs[blockIdx.y];
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < K;
         k += (int64_t)gridDim.x * blockDim.x) {
        const longlong2 v = reinterpret_cast<const longlong2*>(q.wp)[k];
        o[k] = v.x;
        o[Kh + k] = v.y;
    }
}

int errf(int status, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return report_status(status, buf);
}

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

struct pfx_batch {
    int n = 0, d = 0, nw = 0, device = 0, fp32 = 0, kp = 0;
    // 1: stage 1 builds each tile's FP64 cost itself into the pool, one slab
    // per resident CTA (gen), and every pair runs in one wave
    int gen_cost = 0;
    CostGen gen{nullptr, 0, 0, 0};
    // 1: the FP64 cost as a fixed-order FMA chain (PFX_BATCH_COST_FMA)
    int cost_fma = 0;
    Geo gq;  // step set and weights; L = largest tile length (ring sizing)
    std::vector<pfx_plan> plans;
    char* arena = nullptr;
    size_t arena_bytes = 0;
    double* slabs = nullptr;
    size_t slab_bytes = 0;
    double* fin = nullptr;  // raw features, pair i at fin_off[i]: F1 (d x N) then F2 (d x M)
    std::vector<int64_t> fin_off;
    // waves: pairs of wave w are wave_pairs[wave_first[w] .. wave_first[w+1])
    std::vector<int> wave_pairs, wave_first;
    std::vector<int64_t> wave_desc_off, wave_tiles;
    TileDesc* descs = nullptr;
    int* heads = nullptr;
    int32_t* status = nullptr;
    PairOut* pout = nullptr;
    int64_t* res = nullptr;  // [n][9]
    int64_t total_tiles = 0, cells = 0, max_wave_tiles = 0;
    // streams and graph
    cudaStream_t cap = nullptr;
    cudaStream_t side[kSide] = {};
    cudaEvent_t fork_ev = nullptr;
    cudaEvent_t join_ev[kSide] = {};
    cudaStream_t cside[kCostSide] = {};  // the per-pair cost and edge-gather launches
    cudaEvent_t cfork_ev = nullptr;
    cudaEvent_t cjoin_ev[kCostSide] = {};
    cudaGraphExec_t exec = nullptr;
    double graph_beta = 0.0;
    int64_t graph_kernels = 0;  // kernel launches recorded in the graph
    int masked = 0;             // pfx_batch_set_masks: only masked-in tiles run
    // phase events of the last direct run: per wave, before cost building,
    // before stage 1, after stage 1, after the stage-2 join
    std::vector<cudaEvent_t> phase_ev;
    bool phase_valid = false;
    GPair* gpairs = nullptr;  // FP32 form: per wave, its pairs' cost GEMM table
    std::vector<int> wave_gp_off;
    std::vector<int64_t> wave_gp_blocks;
    FbSeg* fbsegs = nullptr;  // FP32 form: every feature matrix's bf16 conversion
    int fb_nseg = 0;
    int64_t fb_blocks = 0;
    char* stage = nullptr;   // pinned staging of pfx_batch_set_masks' uploads
    char* dstage = nullptr;  // and its device copy (scattered from there)
    size_t stage_bytes = 0;
    // masked batches, per pair: the slot map and kept-tile list of the mask
    // (host copies), and the tiles whose stage 1 ran since the last run
    std::vector<std::vector<int32_t>> mask_slots, mask_lists;
    std::vector<std::vector<uint8_t>> mask_host, done;
    bool ran = false;  // a run since pfx_batch_set_masks
    // path checks and row-layout copies (allocated on first use)
    PathRef* pref = nullptr;
    int32_t* rows = nullptr;  // lo | hi block-row scratch
    size_t rows_cap = 0;
    int64_t* prow = nullptr;  // device staging of row-layout paths, + offsets and lengths
    size_t prow_cap = 0;
};

static void batch_free(pfx_batch* b) {
    if (!b) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(b->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    for (int k = 0; k < kSide; ++k) {
        if (b->side[k]) cudaStreamDestroy(b->side[k]);
        if (b->join_ev[k]) cudaEventDestroy(b->join_ev[k]);
    }
    if (b->fork_ev) cudaEventDestroy(b->fork_ev);
    for (int k = 0; k < kCostSide; ++k) {
        if (b->cside[k]) cudaStreamDestroy(b->cside[k]);
        if (b->cjoin_ev[k]) cudaEventDestroy(b->cjoin_ev[k]);
    }
    if (b->cfork_ev) cudaEventDestroy(b->cfork_ev);
    for (cudaEvent_t e : b->phase_ev) cudaEventDestroy(e);
    if (b->cap) cudaStreamDestroy(b->cap);
    if (b->arena) cudaFree(b->arena);
    if (b->slabs) cudaFree(b->slabs);
    if (b->stage) cudaFreeHost(b->stage);
    if (b->dstage) cudaFree(b->dstage);
    if (b->fbsegs) cudaFree(b->fbsegs);
    if (b->gpairs) cudaFree(b->gpairs);
    if (b->pref) cudaFree(b->pref);
    if (b->rows) cudaFree(b->rows);
    if (b->prow) cudaFree(b->prow);
    cudaSetDevice(cur);
    delete b;
}

extern "C" void pfx_batch_destroy(pfx_batch* b) { batch_free(b); }

#define BCK(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            const int st_ = errf(PFX_ERR_CUDA, "%s failed: %s (%s:%d)", #call,             \
                                 cudaGetErrorString(e_), __FILE__, __LINE__);              \
            return st_;                                                                    \
        }                                                                                  \
    } while (0)

extern "C" int pfx_batch_create(int32_t n, const int64_t* N, const int64_t* M, const int32_t* L,
                                const int64_t* steps, const double* weights, int32_t n_steps,
                                int32_t d, int64_t wave_bytes, int32_t nw, int32_t precision,
                                pfx_batch** out) {
    if (!out || !N || !M || !L || !steps || !weights) return errf(PFX_ERR_ARG, "null argument");
    *out = nullptr;
    if (n < 1) return errf(PFX_ERR_ARG, "batch of %d pairs", n);
    const int form = precision & 0xff, flags = precision & ~0xff;
    if ((form != PFX_FP64 && form != PFX_FP32) ||
        (flags & ~(PFX_BATCH_TILE_COST | PFX_BATCH_COST_FMA)))
        return errf(PFX_ERR_ARG,
                    "precision %d: PFX_FP64 (0) or PFX_FP32 (1), optionally | "
                    "PFX_BATCH_TILE_COST or PFX_BATCH_COST_FMA", precision);
    const int fp32 = form == PFX_FP32;
    const int gen_cost = (flags & PFX_BATCH_TILE_COST) != 0;
    const int cost_fma = (flags & PFX_BATCH_COST_FMA) != 0;
    if (gen_cost && (fp32 || d < 1 || d > kGenMaxD))
        return errf(PFX_ERR_ARG, "PFX_BATCH_TILE_COST needs PFX_FP64 and 1 <= d <= %d (d = %d)",
                    kGenMaxD, d);
    if (cost_fma && (fp32 || gen_cost))
        return errf(PFX_ERR_ARG, "PFX_BATCH_COST_FMA needs PFX_FP64 without PFX_BATCH_TILE_COST");
    if (d < 1 || (fp32 && d > 256))
        return errf(PFX_ERR_ARG, "feature dimension %d (the FP32 form takes 1..256)", d);
    const int kp = (d + 63) / 64 * 64;
    // per pair: normalised FP64 features, or the bf16 rows of the FP32 form
    auto feat_bytes = [&](int64_t n_, int64_t m_) {
        return fp32 ? (size_t)(n_ + m_) * kp * 2 : (size_t)d * (n_ + m_) * 8;
    };
    if (nw != 0 && nw != 4 && nw != 8 && nw != 16)
        return errf(PFX_ERR_ARG, "nw=%d: warps per tile must be 4, 8 or 16 (or 0)", nw);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return errf(PFX_ERR_NO_DEVICE, "no CUDA device");
    pfx_batch* b = new pfx_batch();
    cudaGetDevice(&b->device);
    b->n = n;
    b->d = d;
    b->fp32 = fp32;
    b->gen_cost = gen_cost;
    b->cost_fma = cost_fma;
    b->kp = kp;
    b->plans.resize(n);
    int st = PFX_OK;
    int32_t maxL = 0;
    // pass 1: geometry and byte counts
    size_t arena = 0;
    std::vector<size_t> plan_off(n), feat_off(n);
    std::vector<int64_t> slab(n);
    for (int i = 0; i < n; ++i) {
        pfx_plan& p = b->plans[i];
        memset(&p, 0, sizeof(p));
        p.arena_mode = 1;
        if ((st = plan_init(&p, N[i], M[i], L[i], steps, weights, n_steps, nw ? nw : 16, fp32))) {
            batch_free(b);
            return st;
        }
        plan_off[i] = arena;
        arena += round256(p.bytes);
        feat_off[i] = arena;
        arena += round256(feat_bytes(N[i], M[i]));
        slab[i] = plan_slab_bytes(&p);
        maxL = std::max(maxL, p.g.L);
        b->total_tiles += (int64_t)p.g.n1 * p.g.n2;
        for (int t = 0; t < p.g.n1 * p.g.n2; ++t) {
            int64_t r0, c0;
            int32_t R, W;
            tile_rect(p.g, t / p.g.n2, t % p.g.n2, &r0, &c0, &R, &W);
            b->cells += (int64_t)R * W;
        }
    }
    b->gq = b->plans[0].g;
    b->gq.L = maxL;
    for (int i = 1; i < n; ++i) {
        const Geo& g = b->plans[i].g;
        if (g.S != b->gq.S) { batch_free(b); return errf(PFX_ERR_ARG, "steps differ"); }
    }
    // waves: pairs by slab size, largest first, packed in order
    size_t freeb = 0, totalb = 0;
    cudaMemGetInfo(&freeb, &totalb);
    const size_t fin_total = [&] {
        size_t s = 0;
        for (int i = 0; i < n; ++i) s += round256((size_t)d * (N[i] + M[i]) * 8);
        return s;
    }();
    const size_t fixed = arena + fin_total + round256(b->total_tiles * sizeof(TileDesc)) + (1 << 20);
    int64_t budget = wave_bytes;
    // default: 70 % of the memory the batch's other buffers leave free
    if (budget <= 0) budget = (int64_t)((freeb > fixed ? freeb - fixed : 0) / 10 * 7);
    // stage 1 building the cost itself: no slab per tile, one wave
    if (gen_cost) budget = INT64_MAX;
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return slab[a] > slab[c]; });
    if (slab[order[0]] > budget) {
        batch_free(b);
        return errf(PFX_ERR_TOO_LARGE, "pair %d needs %lld B of cost slabs; wave budget %lld B",
                    order[0], (long long)slab[order[0]], (long long)budget);
    }
    std::vector<int64_t> pool_off(n);
    int64_t cur = 0, pool = 0;
    b->wave_first.push_back(0);
    for (int q = 0; q < n; ++q) {
        const int i = order[q];
        if (!gen_cost && cur + slab[i] > budget) {
            b->wave_first.push_back(q);
            cur = 0;
        }
        pool_off[i] = cur;
        if (!gen_cost) cur += (slab[i] + 255) & ~(int64_t)255;
        pool = std::max(pool, cur);
        b->wave_pairs.push_back(i);
    }
    b->wave_first.push_back(n);
    const int waves = (int)b->wave_first.size() - 1;
    // stage-1 warps per tile: from the largest wave's tile count
    for (int w = 0; w < waves; ++w) {
        int64_t t = 0;
        for (int q = b->wave_first[w]; q < b->wave_first[w + 1]; ++q) {
            const Geo& g = b->plans[b->wave_pairs[q]].g;
            t += (int64_t)g.n1 * g.n2;
        }
        b->wave_tiles.push_back(t);
        b->max_wave_tiles = std::max(b->max_wave_tiles, t);
    }
    b->nw = nw ? nw
               : stage1_queue_warps((int)std::min<int64_t>(b->max_wave_tiles, 1 << 30), maxL,
                                    num_sms_cur());
    if (b->nw == 0 || stage1_queue_warps(1, maxL, 1) == 0) {
        batch_free(b);
        return errf(PFX_ERR_TOO_LARGE, "L=%d: the stage-1 rings do not fit in shared memory", maxL);
    }
    if (gen_cost) {
        // one slab (of the largest tile length) per CTA the stage-1 kernel keeps resident
        const int slots = stage1_gen_slots(b->gq, b->nw, d);
        if (slots <= 0) {
            batch_free(b);
            return errf(PFX_ERR_TOO_LARGE, "L=%d, %d warps: the in-kernel cost does not fit", maxL,
                        b->nw);
        }
        b->gen.stride = skew_slab_elems(maxL);
        b->gen.nslots = slots;
        b->gen.d = d;
        pool = (int64_t)slots * b->gen.stride * 8;
    }
    // the remaining arena: raw features, descriptors, heads, status, results
    const size_t off_fin = arena;
    arena += fin_total;
    const size_t off_desc = arena;
    arena += round256(b->total_tiles * sizeof(TileDesc));
    const size_t off_heads = arena;
    arena += round256((size_t)n * sizeof(int));  // up to one wave per pair
    const size_t off_status = arena;
    arena += 256;
    const size_t off_pout = arena;
    arena += round256((size_t)n * sizeof(PairOut));
    const size_t off_res = arena;
    arena += round256((size_t)n * 9 * 8);
    cudaError_t e = cudaMalloc(&b->arena, arena);
    if (e == cudaSuccess) e = cudaMemset(b->arena, 0, arena);
    if (e == cudaSuccess) e = cudaMalloc(&b->slabs, (size_t)pool);
    b->gen.slots = gen_cost ? b->slabs : nullptr;
    if (e != cudaSuccess) {
        batch_free(b);
        return errf(PFX_ERR_CUDA, "batch allocation (%zu + %lld B): %s", arena, (long long)pool,
                    cudaGetErrorString(e));
    }
    b->arena_bytes = arena;
    b->slab_bytes = (size_t)pool;
    b->fin = reinterpret_cast<double*>(b->arena + off_fin);
    b->descs = reinterpret_cast<TileDesc*>(b->arena + off_desc);
    b->heads = reinterpret_cast<int*>(b->arena + off_heads);
    b->status = reinterpret_cast<int32_t*>(b->arena + off_status);
    b->pout = reinterpret_cast<PairOut*>(b->arena + off_pout);
    b->res = reinterpret_cast<int64_t*>(b->arena + off_res);
    // pass 2: carve the plans
    b->fin_off.resize(n);
    std::vector<PairOut> po(n);
    size_t fo = 0;
    for (int i = 0; i < n; ++i) {
        pfx_plan& p = b->plans[i];
        memset(&p, 0, sizeof(p));
        p.arena_mode = 2;
        p.arena = b->arena + plan_off[i];
        if ((st = plan_init(&p, N[i], M[i], L[i], steps, weights, n_steps, b->nw, fp32))) {
            batch_free(b);
            return st;
        }
        if (fp32) {
            p.fbf = b->arena + feat_off[i];
            p.fbf_kp = kp;
        } else {
            p.feat = reinterpret_cast<double*>(b->arena + feat_off[i]);
            p.feat_d = d;
        }
        p.Csk = gen_cost ? nullptr : reinterpret_cast<char*>(b->slabs) + pool_off[i];
        p.gen_cost = gen_cost;
        p.cost_loaded = 1;
        p.s1.status = b->status;
        b->fin_off[i] = (int64_t)(fo / 8);
        fo += round256((size_t)d * (N[i] + M[i]) * 8);
        po[i] = PairOut{p.s2.best, p.s2.best_end, p.s2.wp_len};
    }
    // tile queues: per wave, all tiles of its pairs, largest first
    std::vector<TileDesc> all;
    all.reserve(b->total_tiles);
    for (int w = 0; w < waves; ++w) {
        b->wave_desc_off.push_back((int64_t)all.size());
        std::vector<TileDesc> wv;
        for (int q = b->wave_first[w]; q < b->wave_first[w + 1]; ++q) {
            pfx_plan& p = b->plans[b->wave_pairs[q]];
            std::vector<TileDesc> pd((size_t)p.g.n1 * p.g.n2);
            plan_tile_descs(&p, p.Csk, pd.data());
            // the pair's own queue (pfx_stage1 on the batch plan)
            e = cudaMemcpy(p.descs, pd.data(), pd.size() * sizeof(TileDesc), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) break;
            wv.insert(wv.end(), pd.begin(), pd.end());
        }
        std::stable_sort(wv.begin(), wv.end(), [](const TileDesc& a, const TileDesc& c) {
            return (int64_t)a.R * a.W > (int64_t)c.R * c.W;
        });
        all.insert(all.end(), wv.begin(), wv.end());
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(b->descs, all.data(), all.size() * sizeof(TileDesc), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->pout, po.data(), n * sizeof(PairOut), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && fp32) {
        // the bf16 conversion of every pair's two feature matrices: one launch
        std::vector<FbSeg> segs;
        int64_t blk = 0;
        for (int i = 0; i < n; ++i) {
            const pfx_plan& p = b->plans[i];
            const double* F1 = b->fin + b->fin_off[i];
            char* A = static_cast<char*>(p.fbf);
            segs.push_back(FbSeg{F1, p.g.N, A, blk});
            blk += features_bf16_blocks(p.g.N);
            segs.push_back(FbSeg{F1 + (int64_t)d * p.g.N, p.g.M, A + (size_t)p.g.N * kp * 2, blk});
            blk += features_bf16_blocks(p.g.M);
        }
        b->fb_blocks = blk;
        b->fb_nseg = (int)segs.size();
        e = cudaMalloc(&b->fbsegs, segs.size() * sizeof(FbSeg));
        if (e == cudaSuccess)
            e = cudaMemcpy(b->fbsegs, segs.data(), segs.size() * sizeof(FbSeg),
                           cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess && fp32) {
        // the cost GEMM of a wave's pairs in one launch: per wave, its pairs'
        // tensor maps, geometry and slabs (pairs in wave order, blocks
        // numbered from 0 in each wave)
        std::vector<GPair> gp((size_t)n);
        for (int w = 0; w < waves && e == cudaSuccess; ++w) {
            b->wave_gp_off.push_back(b->wave_first[w]);
            int64_t blk = 0;
            for (int q = b->wave_first[w]; q < b->wave_first[w + 1]; ++q) {
                const pfx_plan& p = b->plans[b->wave_pairs[q]];
                const char* A = static_cast<const char*>(p.fbf);
                const char* B = A + (size_t)p.g.N * kp * 2;
                const int64_t nb = gemm_pair_setup(A, B, kp, p.g, static_cast<float*>(p.Csk),
                                                   p.skew_stride, blk, &gp[q]);
                if (nb <= 0) e = cudaErrorInvalidValue;
                blk += nb;
            }
            b->wave_gp_blocks.push_back(blk);
        }
        if (e == cudaSuccess) e = cudaMalloc(&b->gpairs, gp.size() * sizeof(GPair));
        if (e == cudaSuccess)
            e = cudaMemcpy(b->gpairs, gp.data(), gp.size() * sizeof(GPair),
                           cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemset(b->status, 0, 4);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    for (int k = 0; k < kSide && e == cudaSuccess; ++k) {
        e = cudaStreamCreateWithFlags(&b->side[k], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join_ev[k], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming);
    for (int k = 0; k < kCostSide && e == cudaSuccess; ++k) {
        e = cudaStreamCreateWithFlags(&b->cside[k], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->cjoin_ev[k], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->cfork_ev, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        batch_free(b);
        return errf(PFX_ERR_CUDA, "batch setup: %s", cudaGetErrorString(e));
    }
    *out = b;
    return PFX_OK;
}

extern "C" int pfx_batch_set_masks(pfx_batch* b, const uint8_t* masks, int32_t on_device,
                                   void* stream) {
    if (!b || !masks) return errf(PFX_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    const int n = b->n;
    std::vector<int64_t> moff(n + 1, 0);
    for (int i = 0; i < n; ++i)
        moff[i + 1] = moff[i] + (int64_t)b->plans[i].g.n1 * b->plans[i].g.n2;
    std::vector<uint8_t> m((size_t)moff[n]);
    if (on_device) {
        BCK(cudaMemcpyAsync(m.data(), masks, m.size(), cudaMemcpyDeviceToHost, s));
        BCK(cudaStreamSynchronize(s));
    } else {
        memcpy(m.data(), masks, m.size());
    }
    // slots: kept tiles numbered in tile order; slab bytes per pair
    std::vector<std::vector<int32_t>> slots(n);
    std::vector<int64_t> bytes(n);
    for (int i = 0; i < n; ++i) {
        const pfx_plan& p = b->plans[i];
        const int nt = p.g.n1 * p.g.n2;
        slots[i].assign(nt, -1);
        int kept = 0;
        for (int t = 0; t < nt; ++t)
            if (m[moff[i] + t]) slots[i][t] = kept++;
        bytes[i] = (((int64_t)kept * p.skew_stride * (p.fp32 ? 4 : 8)) + 255) & ~(int64_t)255;
    }
    // waves over the existing slab pool, largest first
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return bytes[a] > bytes[c]; });
    if (!b->gen_cost && bytes[order[0]] > (int64_t)b->slab_bytes)
        return errf(PFX_ERR_TOO_LARGE, "pair %d needs %lld B of cost slabs; pool %zu B", order[0],
                    (long long)bytes[order[0]], b->slab_bytes);
    std::vector<int> wave_pairs, wave_first{0};
    std::vector<int64_t> off(n);
    int64_t cur = 0;
    for (int q = 0; q < n; ++q) {
        const int i = order[q];
        if (!b->gen_cost && cur + bytes[i] > (int64_t)b->slab_bytes) {
            wave_first.push_back(q);
            cur = 0;
        }
        off[i] = cur;
        if (!b->gen_cost) cur += bytes[i];
        wave_pairs.push_back(i);
    }
    wave_first.push_back(n);
    // Everything the device needs is laid out once in pinned staging memory
    // (per pair: slot map, mask, kept-tile list, its queue of every tile and
    // of its kept tiles, their count; then the waves' queues of kept tiles;
    // then the copy table), uploaded with one copy and scattered by one
    // kernel.  Descriptors are built in place.
    auto al16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    std::vector<int32_t> kept_n(n);
    size_t need = 0;
    for (int i = 0; i < n; ++i) {
        const int64_t nt = moff[i + 1] - moff[i];
        int kept = 0;
        for (int64_t t = 0; t < nt; ++t) kept += slots[i][t] >= 0;
        kept_n[i] = kept;
        need += al16(nt * 4) + al16(nt) + al16((size_t)kept * 4) +
                al16(nt * sizeof(TileDesc)) + al16((size_t)kept * sizeof(TileDesc)) + 16;
    }
    int64_t kept_total = 0;
    for (int i = 0; i < n; ++i) kept_total += kept_n[i];
    need += al16((size_t)kept_total * sizeof(TileDesc));
    const size_t table_cap = (size_t)6 * n + (need >> 16) + 16;  // chunks of <= 64 KB
    need += table_cap * sizeof(CopySeg);
    BCK(cudaStreamSynchronize(s));  // the staging buffers may still feed earlier copies
    if (need > b->stage_bytes) {
        if (b->stage) cudaFreeHost(b->stage);
        if (b->dstage) cudaFree(b->dstage);
        b->stage = nullptr;
        b->dstage = nullptr;
        b->stage_bytes = 0;
        BCK(cudaMallocHost(&b->stage, need));
        BCK(cudaMalloc(&b->dstage, need));
        b->stage_bytes = need;
    }
    size_t so = 0;
    std::vector<CopySeg> segs;
    // reserve `bytes` of staging for device address dst (copied later)
    auto reserve = [&](void* dst, size_t bytes) {
        char* h = b->stage + so;
        for (size_t c = 0; c < bytes; c += (size_t)kSegChunk) {
            CopySeg g;
            g.src = (int64_t)(so + c);
            g.dst = static_cast<char*>(dst) + c;
            g.bytes = (int64_t)std::min((size_t)kSegChunk, bytes - c);
            segs.push_back(g);
        }
        so += al16(bytes);
        return h;
    };
    b->mask_slots.assign(n, {});
    b->mask_lists.assign(n, {});
    b->mask_host.assign(n, {});
    b->ran = false;
    // plans: slab base, slot map, mask, kept-tile lists, queues
    std::vector<int64_t> wdo, wt;
    const int waves = (int)wave_first.size() - 1;
    std::vector<std::vector<const TileDesc*>> wave_kept(waves);  // staged descriptors
    for (int w = 0; w < waves; ++w) {
        for (int q = wave_first[w]; q < wave_first[w + 1]; ++q) {
            const int i = wave_pairs[q];
            pfx_plan& p = b->plans[i];
            p.Csk = b->gen_cost ? nullptr : reinterpret_cast<char*>(b->slabs) + off[i];
            const int nt = p.g.n1 * p.g.n2;
            const int kept = kept_n[i];
            memcpy(reserve(p.tile_slot, (size_t)nt * 4), slots[i].data(), (size_t)nt * 4);
            memcpy(reserve(p.tile_mask, (size_t)nt), m.data() + moff[i], (size_t)nt);
            std::vector<int32_t> kl;
            kl.reserve(kept);
            for (int t = 0; t < nt; ++t)
                if (slots[i][t] >= 0) kl.push_back(t);
            if (kept) memcpy(reserve(p.tile_list, (size_t)kept * 4), kl.data(), (size_t)kept * 4);
            p.n_kept = kept;
            b->mask_lists[i] = std::move(kl);
            b->mask_slots[i] = slots[i];
            b->mask_host[i].assign(m.begin() + moff[i], m.begin() + moff[i + 1]);
            // the pair's own queue keeps every tile; its kept tiles, in tile
            // order, are the queue pfx_stage1 runs for the mask
            TileDesc* pd = reinterpret_cast<TileDesc*>(
                reserve(p.descs, (size_t)nt * sizeof(TileDesc)));
            plan_tile_descs(&p, p.Csk, pd, slots[i].data());
            if (kept) {
                TileDesc* sub = reinterpret_cast<TileDesc*>(
                    reserve(p.descs_sub, (size_t)kept * sizeof(TileDesc)));
                int o = 0;
                for (int t = 0; t < nt; ++t)
                    if (slots[i][pd[t].tile] >= 0) {
                        sub[o++] = pd[t];
                        wave_kept[w].push_back(&pd[t]);
                    }
            }
            int32_t* cnt = reinterpret_cast<int32_t*>(reserve(p.nsub, sizeof(int32_t)));
            *cnt = kept;
            p.mask_active = 1;
            p.s2.tile_slot = p.tile_slot;
        }
    }
    // the waves' queues, largest tile first (stable: tile order among equals)
    TileDesc* qall = kept_total ? reinterpret_cast<TileDesc*>(
                                      reserve(b->descs, (size_t)kept_total * sizeof(TileDesc)))
                                : nullptr;
    int64_t qo = 0;
    for (int w = 0; w < waves; ++w) {
        std::vector<const TileDesc*>& kv = wave_kept[w];
        std::stable_sort(kv.begin(), kv.end(), [](const TileDesc* a, const TileDesc* c) {
            return (int64_t)a->R * a->W > (int64_t)c->R * c->W;
        });
        wdo.push_back(qo);
        for (const TileDesc* d : kv) qall[qo++] = *d;
        wt.push_back((int64_t)kv.size());
    }
    if (segs.size() > table_cap)
        return errf(PFX_ERR_TOO_LARGE, "copy table: %zu segments > %zu", segs.size(), table_cap);
    const size_t toff = so;
    memcpy(b->stage + toff, segs.data(), segs.size() * sizeof(CopySeg));
    so += segs.size() * sizeof(CopySeg);
    BCK(cudaMemcpyAsync(b->dstage, b->stage, so, cudaMemcpyHostToDevice, s));
    if (!segs.empty()) {
        k_scatter_segments<<<(unsigned)segs.size(), 256, 0, s>>>(
            b->dstage, reinterpret_cast<const CopySeg*>(b->dstage + toff), (int)segs.size());
        count_launches(1);
        BCK(cudaGetLastError());
    }
    BCK(cudaStreamSynchronize(s));
    b->wave_pairs = wave_pairs;
    b->wave_first = wave_first;
    b->wave_desc_off = wdo;
    b->wave_tiles = wt;
    b->max_wave_tiles = 0;
    for (int64_t x : wt) b->max_wave_tiles = std::max(b->max_wave_tiles, x);
    b->masked = 1;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    for (cudaEvent_t e : b->phase_ev) cudaEventDestroy(e);
    b->phase_ev.clear();
    b->phase_valid = false;
    return PFX_OK;
}

extern "C" int pfx_batch_complete(pfx_batch* b, int32_t i, double beta, const uint8_t* tiles,
                                  void* stream) {
    if (!b) return errf(PFX_ERR_ARG, "null batch");
    if (i < 0 || i >= b->n) return errf(PFX_ERR_ARG, "pair %d of %d", i, b->n);
    if (!b->masked) return errf(PFX_ERR_ARG, "pfx_batch_complete needs a masked batch");
    if (!b->ran) return errf(PFX_ERR_ARG, "pfx_batch_complete needs a run since pfx_batch_set_masks");
    pfx_plan& p = b->plans[i];
    const int nt = p.g.n1 * p.g.n2;
    if (!b->gen_cost && plan_slab_bytes(&p) > (int64_t)b->slab_bytes)
        return errf(PFX_ERR_TOO_LARGE, "pair %d: its cost slabs exceed the pool", i);
    cudaStream_t s = (cudaStream_t)stream;
    BCK(cudaStreamSynchronize(s));  // the pool and the queue buffers are free again
    // tiles whose stage 1 has run: the mask, then every completion since the run
    std::vector<uint8_t>& done = b->done[i];
    std::vector<int32_t> slot((size_t)nt), list;
    std::vector<uint8_t> run((size_t)nt, 0);
    for (int t = 0; t < nt; ++t) {
        const bool want = !tiles || tiles[t];
        run[t] = want && !done[t];
        if (want) done[t] = 1;
        slot[t] = done[t] ? t : -1;  // slab t of the pool (pool offset 0)
        if (done[t]) list.push_back(t);
    }
    // the pair's slot map and tile list point at the pool's start meanwhile
    BCK(cudaMemcpyAsync(p.tile_slot, slot.data(), (size_t)nt * 4, cudaMemcpyHostToDevice, s));
    BCK(cudaMemcpyAsync(p.tile_list, list.data(), list.size() * 4, cudaMemcpyHostToDevice, s));
    const double* F1 = b->fin + b->fin_off[i];
    const double* F2 = F1 + (int64_t)b->d * p.g.N;
    if (b->gen_cost) {
        // stage 1 builds the cost of the tiles it runs from the features the
        // masked run normalised
    } else if (b->fp32) {
        // the bf16 features of the run
        const char* A = static_cast<const char*>(p.fbf);
        const char* B = A + (size_t)p.g.N * b->kp * 2;
        BCK(launch_gemm_cost_skew(A, B, b->kp, p.g, reinterpret_cast<float*>(b->slabs),
                                  p.skew_stride, b->status, s, p.tile_slot, p.tile_list,
                                  (int)list.size()));
    } else {
        double* An = p.feat;
        double* Bn = p.feat + (int64_t)b->d * p.g.N;
        BCK(launch_l2norm(F1, b->d, p.g.N, An, s));
        BCK(launch_l2norm(F2, b->d, p.g.M, Bn, s));
        BCK(launch_cost_skew(An, Bn, b->d, p.g, b->slabs, p.skew_stride, s, p.tile_slot,
                             p.tile_list, (int)list.size(), b->cost_fma != 0));
    }
    // stage 1 on the tiles added now (the others' outputs stand; tiles never
    // run keep the +inf edges of the masked run)
    std::vector<TileDesc> pd((size_t)nt), todo;
    plan_tile_descs(&p, b->gen_cost ? nullptr : b->slabs, pd.data());
    for (const TileDesc& d : pd)
        if (run[d.tile]) todo.push_back(d);
    // queue space past the masked waves' queues: the masked-out tiles of
    // one pair never outnumber the masked-out tiles of the batch
    const int waves = (int)b->wave_first.size() - 1;
    TileDesc* qd = b->descs + b->wave_desc_off[waves - 1] + b->wave_tiles[waves - 1];
    int* head = b->heads + (waves < b->n ? waves : 0);
    if (!todo.empty()) {
        BCK(cudaMemcpyAsync(qd, todo.data(), todo.size() * sizeof(TileDesc),
                            cudaMemcpyHostToDevice, s));
        BCK(cudaMemsetAsync(head, 0, sizeof(int), s));
        // (the in-kernel cost's pool holds slabs for the batch's own warps choice)
        const int nw = b->gen_cost ? 0 : stage1_queue_warps((int)todo.size(), b->gq.L,
                                                            num_sms_cur());
        BCK(launch_stage1_queue(qd, (int)todo.size(), nullptr, head, b->gq, b->status,
                                nw ? nw : b->nw, b->fp32 != 0, s,
                                b->gen_cost ? &b->gen : nullptr));
    }
    void* masked_Csk = p.Csk;
    p.Csk = b->gen_cost ? nullptr : b->slabs;
    int st = pfx_stage2_propagate(&p, nullptr, 0, stream);
    if (!st) st = pfx_stage2_scan(&p, beta, stream);
    if (!st) st = pfx_stage2_stitch(&p, 1, 0, 0, 0, 0, stream);
    // back to the masked state (the batch's queues and graph stay valid)
    p.Csk = masked_Csk;
    const std::vector<int32_t>& ms = b->mask_slots[i];
    const std::vector<int32_t>& ml = b->mask_lists[i];
    BCK(cudaMemcpyAsync(p.tile_slot, ms.data(), ms.size() * 4, cudaMemcpyHostToDevice, s));
    if (!ml.empty())
        BCK(cudaMemcpyAsync(p.tile_list, ml.data(), ml.size() * 4, cudaMemcpyHostToDevice, s));
    BCK(cudaStreamSynchronize(s));  // host vectors fed asynchronous copies
    return st;
}

extern "C" int pfx_batch_info(const pfx_batch* b, int64_t* info) {
    if (!b || !info) return errf(PFX_ERR_ARG, "null argument");
    info[0] = b->n;
    info[1] = (int64_t)b->wave_first.size() - 1;
    info[2] = b->total_tiles;
    info[3] = b->cells;
    info[4] = (int64_t)(b->arena_bytes + b->slab_bytes);
    info[5] = b->nw;
    info[6] = b->max_wave_tiles;
    info[7] = (int64_t)b->slab_bytes;
    info[8] = b->gen_cost;
    return PFX_OK;
}

extern "C" int pfx_batch_features(pfx_batch* b, int32_t i, double** F1, double** F2) {
    if (!b || !F1 || !F2) return errf(PFX_ERR_ARG, "null argument");
    if (i < 0 || i >= b->n) return errf(PFX_ERR_ARG, "pair %d of %d", i, b->n);
    *F1 = b->fin + b->fin_off[i];
    *F2 = *F1 + (int64_t)b->d * b->plans[i].g.N;
    return PFX_OK;
}

extern "C" int pfx_batch_load_async(pfx_batch* b, int32_t i, const double* F1,
                                    const double* F2, void* stream) {
    if (!b || !F1 || !F2) return errf(PFX_ERR_ARG, "null argument");
    if (i < 0 || i >= b->n) return errf(PFX_ERR_ARG, "pair %d of %d", i, b->n);
    cudaStream_t s = (cudaStream_t)stream;
    double* d1 = b->fin + b->fin_off[i];
    double* d2 = d1 + (int64_t)b->d * b->plans[i].g.N;
    BCK(cudaMemcpyAsync(d1, F1, sizeof(double) * (size_t)b->d * b->plans[i].g.N,
                        cudaMemcpyHostToDevice, s));
    BCK(cudaMemcpyAsync(d2, F2, sizeof(double) * (size_t)b->d * b->plans[i].g.M,
                        cudaMemcpyHostToDevice, s));
    return PFX_OK;
}

extern "C" int pfx_batch_plan(pfx_batch* b, int32_t i, pfx_plan** plan) {
    if (!b || !plan) return errf(PFX_ERR_ARG, "null argument");
    if (i < 0 || i >= b->n) return errf(PFX_ERR_ARG, "pair %d of %d", i, b->n);
    *plan = &b->plans[i];
    return PFX_OK;
}

// The launch sequence of one batch run, on stream s (captured or direct;
// `timed` records the phase events, direct runs only).
static int batch_enqueue(pfx_batch* b, double beta, cudaStream_t s, bool timed) {
    const int waves = (int)b->wave_first.size() - 1;
    BCK(cudaMemsetAsync(b->heads, 0, (size_t)waves * sizeof(int), s));
    if (timed && b->phase_ev.empty()) {
        b->phase_ev.resize((size_t)waves * 4 + 1);
        for (auto& e : b->phase_ev) BCK(cudaEventCreate(&e));
    }
    b->phase_valid = false;
    auto mark = [&](int w, int k) -> cudaError_t {
        return timed ? cudaEventRecord(b->phase_ev[(size_t)w * 4 + k], s) : cudaSuccess;
    };
    int st;
    int used_side = 0;  // side streams forked so far (joined at the end)
    // a wave's per-pair launches (cost, edge gathers) spread over s and up to
    // kCostSide more streams, forked from s and joined back into it, so that
    // one pair's kernel tail overlaps the next pair's kernels
    auto cost_fork = [&](int npairs, int* nc) -> cudaError_t {
        *nc = std::min(kCostSide, npairs - 1);
        if (*nc <= 0) return cudaSuccess;
        cudaError_t e = cudaEventRecord(b->cfork_ev, s);
        for (int k = 0; k < *nc && e == cudaSuccess; ++k)
            e = cudaStreamWaitEvent(b->cside[k], b->cfork_ev, 0);
        return e;
    };
    auto cost_join = [&](int nc) -> cudaError_t {
        cudaError_t e = cudaSuccess;
        for (int k = 0; k < nc && e == cudaSuccess; ++k) {
            e = cudaEventRecord(b->cjoin_ev[k], b->cside[k]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(s, b->cjoin_ev[k], 0);
        }
        return e;
    };
    auto cost_stream = [&](int q, int nc) { return q % (nc + 1) == 0 ? s : b->cside[q % (nc + 1) - 1]; };
    for (int w = 0; w < waves; ++w) {
        const int q0 = b->wave_first[w], q1 = b->wave_first[w + 1];
        BCK(mark(w, 0));
        if (w == 0 && b->fp32)  // every pair's bf16 features, one launch
            BCK(launch_features_bf16_segs(b->fbsegs, b->fb_nseg, b->fb_blocks, b->d, b->kp, s));
        if (b->fp32 && !b->masked)  // the wave's cost GEMM, one launch
            BCK(launch_gemm_cost_multi(b->gpairs + b->wave_gp_off[w], q1 - q0,
                                       b->wave_gp_blocks[w], b->kp, b->status, s));
        int nc = 0;
        BCK(cost_fork(q1 - q0, &nc));
        for (int q = q0; q < q1; ++q) {
            const cudaStream_t cs = cost_stream(q - q0, nc);
            const int i = b->wave_pairs[q];
            pfx_plan& p = b->plans[i];
            const double* F1 = b->fin + b->fin_off[i];
            const double* F2 = F1 + (int64_t)b->d * p.g.N;
            const int32_t* slot = b->masked ? p.tile_slot : nullptr;
            const int32_t* list = b->masked ? p.tile_list : nullptr;
            if (b->fp32 && !b->masked) {
                // built above
            } else if (b->fp32) {
                const char* A = static_cast<const char*>(p.fbf);
                const char* B = A + (size_t)p.g.N * b->kp * 2;
                BCK(launch_gemm_cost_skew(A, B, b->kp, p.g, static_cast<float*>(p.Csk),
                                          p.skew_stride, b->status, cs, slot, list, p.n_kept,
                                          b->masked ? (int64_t)p.n_kept * p.skew_stride : -1));
            } else {
                double* An = p.feat;
                double* Bn = p.feat + (int64_t)b->d * p.g.N;
                BCK(launch_l2norm(F1, b->d, p.g.N, An, cs));
                BCK(launch_l2norm(F2, b->d, p.g.M, Bn, cs));
                if (!b->gen_cost)  // (else stage 1 builds each tile's cost)
                    BCK(launch_cost_skew(An, Bn, b->d, p.g, static_cast<double*>(p.Csk),
                                         p.skew_stride, cs, slot, list, p.n_kept,
                                         b->cost_fma != 0));
            }
            if (b->masked) {
                // skipped tiles keep +inf edges and start 0 for stage 2
                BCK(launch_fill(p.s1.edge_D, p.n4, HUGE_VAL, cs));
                BCK(cudaMemsetAsync(p.s1.edge_P, 0, (size_t)p.n4 * 4, cs));
            }
        }
        BCK(cost_join(nc));
        BCK(mark(w, 1));
        BCK(launch_stage1_queue(b->descs + b->wave_desc_off[w], (int)b->wave_tiles[w], nullptr,
                                b->heads + w, b->gq, b->status, b->nw, b->fp32 != 0, s,
                                b->gen_cost ? &b->gen : nullptr));
        BCK(mark(w, 2));
        // stage 2 reads the cost slabs only in its edge gather: that part is
        // joined back into the main stream, so the next wave may overwrite the
        // pool while the rest of this wave's stage 2 runs on the side streams
        BCK(cost_fork(q1 - q0, &nc));
        for (int q = q0; q < q1; ++q) {
            const cudaStream_t cs = cost_stream(q - q0, nc);
            const pfx_plan& p = b->plans[b->wave_pairs[q]];
            if (b->gen_cost)  // no slabs kept: overlap costs from the features
                BCK(launch_stage2_edges(nullptr, nullptr, 0, false, p.g, p.s2, cs, p.feat,
                                        p.feat + (int64_t)b->d * p.g.N, b->d));
            else
                BCK(launch_stage2_edges(nullptr, p.Csk, p.skew_stride, p.fp32 != 0, p.g, p.s2,
                                        cs));
        }
        BCK(cost_join(nc));
        BCK(mark(w, 3));
        BCK(cudaEventRecord(b->fork_ev, s));
        const int nside = std::min(kSide, q1 - q0);
        used_side = std::max(used_side, nside);
        for (int k = 0; k < nside; ++k) BCK(cudaStreamWaitEvent(b->side[k], b->fork_ev, 0));
        for (int q = q0; q < q1; ++q) {
            pfx_plan* p = &b->plans[b->wave_pairs[q]];
            cudaStream_t ss = b->side[(q - q0) % nside];
            BCK(launch_stage2_prop(p->g, p->s2, ss));
            if ((st = pfx_stage2_scan(p, beta, ss))) return st;
            if ((st = pfx_stage2_stitch(p, 1, 0, 0, 0, 0, ss))) return st;
        }
    }
    for (int k = 0; k < used_side; ++k) {
        BCK(cudaEventRecord(b->join_ev[k], b->side[k]));
        BCK(cudaStreamWaitEvent(s, b->join_ev[k], 0));
    }
    if (timed) BCK(cudaEventRecord(b->phase_ev[(size_t)waves * 4], s));
    b->phase_valid = timed;
    return PFX_OK;
}

extern "C" int pfx_batch_run(pfx_batch* b, double beta, int32_t use_graph, void* stream) {
    if (!b) return errf(PFX_ERR_ARG, "null batch");
    cudaStream_t s = (cudaStream_t)stream;
    if (b->masked) {  // completions start again from the mask
        b->done = b->mask_host;
        b->ran = true;
    }
    if (!use_graph) return batch_enqueue(b, beta, s, true);
    if (!b->exec || b->graph_beta != beta) {
        if (b->exec) {
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
        }
        // record on the batch's own stream, ordered after work already on `s`
        BCK(cudaEventRecord(b->fork_ev, s));
        BCK(cudaStreamWaitEvent(b->cap, b->fork_ev, 0));
        BCK(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeRelaxed));
        const int64_t k0 = pfx_kernel_launches();
        const int st = batch_enqueue(b, beta, b->cap, false);
        // recorded launches run at each replay: count them there, not here
        b->graph_kernels = pfx_kernel_launches() - k0;
        count_launches(-(int)b->graph_kernels);
        cudaGraph_t graph = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->cap, &graph);
        if (st) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (e != cudaSuccess) return errf(PFX_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        const cudaError_t ei = cudaGraphInstantiate(&b->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) {
            b->exec = nullptr;
            return errf(PFX_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ei));
        }
        b->graph_beta = beta;
    }
    BCK(cudaGraphLaunch(b->exec, s));
    count_launches((int)b->graph_kernels);
    return PFX_OK;
}

extern "C" int pfx_batch_timing(pfx_batch* b, double* ms3) {
    if (!b || !ms3) return errf(PFX_ERR_ARG, "null argument");
    if (!b->phase_valid) return errf(PFX_ERR_ARG, "no direct (use_graph = 0) run to time");
    const int waves = (int)b->wave_first.size() - 1;
    BCK(cudaEventSynchronize(b->phase_ev[(size_t)waves * 4]));
    ms3[0] = ms3[1] = ms3[2] = 0.0;
    for (int w = 0; w < waves; ++w) {
        for (int k = 0; k < 3; ++k) {
            float t = 0.f;
            BCK(cudaEventElapsedTime(&t, b->phase_ev[(size_t)w * 4 + k],
                                     b->phase_ev[(size_t)w * 4 + k + 1]));
            ms3[k] += t;
        }
    }
    // the rest of stage 2 overlaps the later waves: add only its tail
    float tail = 0.f;
    BCK(cudaEventElapsedTime(&tail, b->phase_ev[(size_t)waves * 4 - 1],
                             b->phase_ev[(size_t)waves * 4]));
    ms3[2] += tail;
    return PFX_OK;
}

extern "C" int pfx_batch_results(pfx_batch* b, void* stream, double* best_cost, int64_t* best_end7,
                                 int64_t* wp_len) {
    if (!b) return errf(PFX_ERR_ARG, "null batch");
    cudaStream_t s = (cudaStream_t)stream;
    k_gather_results<<<(b->n + 127) / 128, 128, 0, s>>>(b->pout, b->n, b->res);
    count_launches(1);
    BCK(cudaGetLastError());
    std::vector<int64_t> h((size_t)b->n * 9);
    int32_t kst = 0;
    BCK(cudaMemcpyAsync(h.data(), b->res, h.size() * 8, cudaMemcpyDeviceToHost, s));
    BCK(cudaMemcpyAsync(&kst, b->status, 4, cudaMemcpyDeviceToHost, s));
    BCK(cudaStreamSynchronize(s));
    if (kst) {
        cudaMemsetAsync(b->status, 0, 4, s);
        return errf(PFX_ERR_CUDA, "stage-1 wavefront wait ran out (status %d); batch invalid", kst);
    }
    for (int i = 0; i < b->n; ++i) {
        const int64_t* r = &h[(size_t)i * 9];
        if (best_cost) memcpy(&best_cost[i], &r[0], 8);
        if (best_end7) memcpy(&best_end7[(size_t)i * 7], &r[1], 56);
        if (wp_len) wp_len[i] = r[8];
    }
    return PFX_OK;
}

static int ensure_pref(pfx_batch* b) {
    if (b->pref) return PFX_OK;
    std::vector<PathRef> h((size_t)b->n);
    int64_t to = 0, ro = 0;
    for (int i = 0; i < b->n; ++i) {
        const pfx_plan& p = b->plans[i];
        h[i] = PathRef{p.s2.wp, p.s2.wp_len, p.tile_mask, p.g.N, p.g.M, p.g.n1, p.g.n2, p.g.L,
                       0, to, ro};
        to += (int64_t)p.g.n1 * p.g.n2;
        ro += p.g.N + 2;  // block rows for any block size >= 1
    }
    BCK(cudaMalloc(&b->pref, h.size() * sizeof(PathRef)));
    BCK(cudaMemcpy(b->pref, h.data(), h.size() * sizeof(PathRef), cudaMemcpyHostToDevice));
    return PFX_OK;
}

extern "C" int pfx_batch_check_paths(pfx_batch* b, int32_t margin, uint8_t* near, int32_t* flags,
                                     void* stream) {
    if (!b || !near || !flags) return errf(PFX_ERR_ARG, "null argument");
    if (margin < 1) return errf(PFX_ERR_ARG, "margin %d", margin);
    if (!b->masked) return errf(PFX_ERR_ARG, "pfx_batch_check_paths needs a masked batch");
    cudaStream_t s = (cudaStream_t)stream;
    int st = ensure_pref(b);
    if (st) return st;
    size_t rows = 0;
    for (int i = 0; i < b->n; ++i) rows += (size_t)b->plans[i].g.N + 2;
    if (rows * 2 > b->rows_cap) {
        BCK(cudaStreamSynchronize(s));
        if (b->rows) cudaFree(b->rows);
        b->rows = nullptr;
        b->rows_cap = 0;
        BCK(cudaMalloc(&b->rows, rows * 2 * sizeof(int32_t)));
        b->rows_cap = rows * 2;
    }
    BCK(cudaMemsetAsync(b->rows, 0xff, rows * 2 * sizeof(int32_t), s));
    BCK(cudaMemsetAsync(near, 0, (size_t)b->total_tiles, s));
    BCK(cudaMemsetAsync(flags, 0, (size_t)b->n * sizeof(int32_t), s));
    k_path_rows<<<dim3(32, b->n), 256, 0, s>>>(b->pref, margin, b->rows, b->rows + rows);
    k_path_near<<<dim3(4, b->n), 256, 0, s>>>(b->pref, margin, b->rows, b->rows + rows, near,
                                              flags);
    count_launches(2);
    BCK(cudaGetLastError());
    return PFX_OK;
}

extern "C" int pfx_batch_copy_paths_rows(pfx_batch* b, void* stream, int64_t* host,
                                         const int64_t* offsets, const int64_t* lens,
                                         int64_t cap) {
    if (!b || !host || !offsets || !lens) return errf(PFX_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    int64_t total = 0;
    for (int i = 0; i < b->n; ++i) {
        if (lens[i] < 0 || offsets[i] < 0 || offsets[i] + lens[i] > cap)
            return errf(PFX_ERR_ARG, "pair %d: path of %lld points at offset %lld exceeds %lld", i,
                        (long long)lens[i], (long long)offsets[i], (long long)cap);
        total = std::max(total, offsets[i] + lens[i]);
    }
    int st = ensure_pref(b);
    if (st) return st;
    const size_t need = (size_t)2 * total + 2 * (size_t)b->n;
    if (need > b->prow_cap) {
        BCK(cudaStreamSynchronize(s));
        if (b->prow) cudaFree(b->prow);
        b->prow = nullptr;
        b->prow_cap = 0;
        const size_t cap2 = need + need / 4 + 1024;
        BCK(cudaMalloc(&b->prow, cap2 * sizeof(int64_t)));
        b->prow_cap = cap2;
    }
    int64_t* d_off = b->prow + b->prow_cap - 2 * (size_t)b->n;
    int64_t* d_len = d_off + b->n;
    std::vector<int64_t> ol((size_t)2 * b->n);
    std::copy(offsets, offsets + b->n, ol.begin());
    std::copy(lens, lens + b->n, ol.begin() + b->n);
    BCK(cudaMemcpyAsync(d_off, ol.data(), ol.size() * 8, cudaMemcpyHostToDevice, s));
    k_path_to_rows<<<dim3(16, b->n), 256, 0, s>>>(b->pref, d_off, d_len, b->prow);
    count_launches(1);
    BCK(cudaGetLastError());
    if (total > 0)
        BCK(cudaMemcpyAsync(host, b->prow, (size_t)2 * total * 8, cudaMemcpyDeviceToHost, s));
    BCK(cudaStreamSynchronize(s));
    return PFX_OK;
}

extern "C" int pfx_batch_copy_paths(pfx_batch* b, void* stream, int64_t* wp_host,
                                    const int64_t* offsets, int64_t cap) {
    if (!b || !wp_host || !offsets) return errf(PFX_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<int64_t> lens(b->n);
    for (int i = 0; i < b->n; ++i)
        BCK(cudaMemcpyAsync(&lens[i], b->plans[i].s2.wp_len, 8, cudaMemcpyDeviceToHost, s));
    BCK(cudaStreamSynchronize(s));
    for (int i = 0; i < b->n; ++i) {
        if (offsets[i] < 0 || offsets[i] + lens[i] > cap)
            return errf(PFX_ERR_ARG, "pair %d: path of %lld points at offset %lld exceeds %lld", i,
                        (long long)lens[i], (long long)offsets[i], (long long)cap);
        if (lens[i] > 0)
            BCK(cudaMemcpyAsync(wp_host + 2 * offsets[i], b->plans[i].s2.wp, (size_t)lens[i] * 16,
                                cudaMemcpyDeviceToHost, s));
    }
    BCK(cudaStreamSynchronize(s));
    return PFX_OK;
}
