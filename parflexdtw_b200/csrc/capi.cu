// extern "C" entry points (declared in include/parflexdtw_b200.h).
#include <stdarg.h>
#include <stdio.h>

#include <algorithm>
#include <atomic>
#include <stdlib.h>
#include <string.h>

#include <cmath>
#include <vector>

#include "plan.cuh"



using namespace pfx;

static thread_local char g_err[512];
static std::atomic<long long> g_launches{0};

void pfx::count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

extern "C" int64_t pfx_kernel_launches(void) { return (int64_t)g_launches.load(); }

static int fail(int status, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return status;
}

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(PFX_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                             \
    } while (0)

static const char* kStatus[] = {"ok",
                                "invalid argument",
                                "unsupported step set",
                                "CUDA error",
                                "Stage 2: No valid endpoint found on global top/right edges.",
                                "tile length too large",
                                "no CUDA device"};

extern "C" const char* pfx_status_string(int s) {
    return (s >= 0 && s <= 6) ? kStatus[s] : "unknown status";
}
extern "C" const char* pfx_last_error(void) { return g_err; }
extern "C" int pfx_version(void) { return 100; }

// Steps -> kinds (0 = (1,1), 1 = (1,2), 2 = (2,1)).
static int parse_steps(const int64_t* steps, const double* weights, int32_t n, Geo* g) {
    if (n < 1 || n > 3) return fail(PFX_ERR_STEPS, "n_steps=%d; the device DP takes 1..3 steps", n);
    for (int s = 0; s < n; ++s) {
        const int64_t a = steps[2 * s], b = steps[2 * s + 1];
        int kd;
        if (a == 1 && b == 1) kd = 0;
        else if (a == 1 && b == 2) kd = 1;
        else if (a == 2 && b == 1) kd = 2;
        else
            return fail(PFX_ERR_STEPS, "step (%lld, %lld) is not one of (1,1), (1,2), (2,1)",
                        (long long)a, (long long)b);
        for (int t = 0; t < s; ++t)
            if (g->kind[t] == kd) return fail(PFX_ERR_STEPS, "step listed twice");
        g->kind[s] = kd;
        g->w[s] = weights[s];
    }
    for (int s = n; s < 3; ++s) { g->kind[s] = 0; g->w[s] = 0.0; }
    g->S = n;
    return PFX_OK;
}

// Internal helpers shared with other translation units of this library.
int pfx::report_status(int status, const char* msg) { return fail(status, "%s", msg); }
int pfx::parse_step_kinds(const int64_t* steps, const double* weights, int32_t n, Geo* g) {
    return parse_steps(steps, weights, n, g);
}

static int make_geo(int64_t N, int64_t M, int32_t L, const int64_t* steps, const double* weights,
                    int32_t n_steps, Geo* g) {
    memset(g, 0, sizeof(*g));
    if (N < 2 || M < 2) return fail(PFX_ERR_ARG, "cost matrix %lld x %lld: need at least 2 x 2", (long long)N, (long long)M);
    if (L < 2) return fail(PFX_ERR_ARG, "L=%d: need L >= 2", L);
    if (N >= (1LL << 31) || M >= (1LL << 31)) return fail(PFX_ERR_ARG, "sequence longer than 2^31");
    int st = parse_steps(steps, weights, n_steps, g);
    if (st) return st;
    g->N = N;
    g->M = M;
    g->ldc = M;
    g->L = L;
    g->hop = L - 1;
    g->n1 = (int32_t)ceil_div64(N - 1, g->hop);
    g->n2 = (int32_t)ceil_div64(M - 1, g->hop);
    g->b_words = tile_b_words2(L);
    return PFX_OK;
}

int pfx::num_sms_cur() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

static int check_smem(int32_t L, int nw) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t need = stage1_smem_bytes_host(L, nw);
    if (need > (size_t)optin)
        return fail(PFX_ERR_TOO_LARGE, "L=%d needs %zu B of shared memory per tile CTA (limit %d)",
                    L, need, optin);
    return PFX_OK;
}

template <typename T>
static int plan_alloc(pfx_plan* p, T** ptr, size_t count) {
    void* q = nullptr;
    const size_t bytes = count * sizeof(T) > 0 ? count * sizeof(T) : 16;
    if (p->arena_mode) {
        // carve from a caller-owned arena (mode 2) or only count (mode 1)
        const size_t rounded = (bytes + 255) & ~(size_t)255;
        *ptr = p->arena_mode == 2 ? reinterpret_cast<T*>(p->arena + p->arena_off) : nullptr;
        p->arena_off += rounded;
        p->bytes += rounded;
        return PFX_OK;
    }
    if (p->nblocks >= (int)(sizeof(p->blocks) / sizeof(p->blocks[0])))
        return fail(PFX_ERR_ARG, "plan buffer table full");
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess)
        return fail(PFX_ERR_CUDA, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    p->blocks[p->nblocks++] = q;
    p->bytes += bytes;
    *ptr = reinterpret_cast<T*>(q);
    return PFX_OK;
}

extern "C" void pfx_plan_destroy(pfx_plan* p) {
    if (!p || p->arena_mode == 2) return;  // plans inside a batch belong to the batch
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(p->device);
    for (int i = 0; i < p->nblocks; ++i) cudaFree(p->blocks[i]);
    if (p->aux) cudaStreamDestroy(p->aux);
    if (p->ev_fork) cudaEventDestroy(p->ev_fork);
    if (p->ev_join) cudaEventDestroy(p->ev_join);
    cudaSetDevice(cur);
    free(p);
}

// Geometry, warps per tile and every buffer of a plan (cudaMalloc, or the
// arena selected by p->arena_mode).  The tile-skewed cost slabs and the tile
// queue are separate (plan_attach_cost).
int pfx::plan_init(pfx_plan* p, int64_t N, int64_t M, int32_t L, const int64_t* steps,
                   const double* weights, int32_t n_steps, int nw, int fp32) {
    int st = make_geo(N, M, L, steps, weights, n_steps, &p->g);
    if (st) return st;
    p->fp32 = fp32 ? 1 : 0;
    cudaGetDevice(&p->device);
    const Geo& g = p->g;
    const int64_t nt = (int64_t)g.n1 * g.n2;
    p->nw = nw ? nw : stage1_queue_warps((int)std::min<int64_t>(nt, 1 << 30), L, num_sms_cur());
    if (p->nw == 0 || stage1_queue_warps(1, L, 1) == 0)
        return fail(PFX_ERR_TOO_LARGE, "L=%d: the stage-1 rings do not fit in shared memory", L);
    p->skew_stride = skew_slab_elems(L);
    p->n4 = nt * 2 * g.L;
    const int64_t ms = std::max<int64_t>(std::max(ceil_div64(M, L), ceil_div64(N, L)), 1);
    p->s2.max_segs = (int32_t)ms;
    p->s2.seg_cap = 2 * (int64_t)L + 8;
    double* eD;
    int32_t* eP;
    uint32_t* Bw;
#define PA(ptr, n)                                                 \
    do {                                                           \
        if ((st = plan_alloc(p, ptr, (size_t)(n)))) return st;     \
    } while (0)
    PA(&eD, p->n4);
    PA(&eP, p->n4);
    PA(&Bw, nt * g.b_words);
    p->s1.edge_D = eD;
    p->s1.edge_P = eP;
    p->s1.Bw = Bw;
    p->s2.edge_D = eD;
    p->s2.edge_P = eP;
    p->s2.Bw = Bw;
    PA(&p->s2.edge_Cf, p->n4);
    PA(&p->s2.valid, p->n4);
    PA(&p->s2.D_arr, p->n4);
    PA(&p->s2.L_arr, p->n4);
    PA(&p->D_prop, p->n4);
    PA(&p->L_prop, p->n4);
    PA(&p->s2.top_D, M);
    PA(&p->s2.top_L, M);
    PA(&p->s2.right_D, N);
    PA(&p->s2.right_L, N);
    PA(&p->s2.seg_norm, 2 * ms);
    PA(&p->s2.seg_meta, 12 * ms);
    PA(&p->s2.best, 1);
    PA(&p->s2.best_end, 7);
    PA(&p->s2.chain, 101 * 12);
    PA(&p->s2.chain_len, 1);
    PA(&p->s2.seg_pts, 101 * p->s2.seg_cap * 2);
    PA(&p->s2.seg_len, 101);
    PA(&p->s2.wp, 101 * p->s2.seg_cap * 2);
    PA(&p->s2.wp_len, 1);
    PA(&p->s1.status, 1);
    PA(&p->descs, nt);
    PA(&p->head, 1);
    PA(&p->head2, 1);
    PA(&p->tile_mask, nt);
    PA(&p->tile_slot, nt);
    PA(&p->tile_list, nt);
    PA(&p->descs_sub, nt);
    PA(&p->nsub, 1);
#undef PA
    if (p->arena_mode) return PFX_OK;  // arenas are zeroed by their owner
    CK(cudaMemset(p->s2.best_end, 0, 7 * sizeof(int64_t)));
    CK(cudaMemset(p->s2.chain_len, 0, sizeof(int32_t)));
    CK(cudaMemset(p->s2.wp_len, 0, sizeof(int64_t)));
    CK(cudaMemset(p->s1.status, 0, sizeof(int32_t)));
    // backpointer words stage 1 never writes (past a tile's rows or steps)
    // read as 0, so that two plans' arrays compare equal
    CK(cudaMemset(p->s1.Bw, 0, (size_t)nt * g.b_words * sizeof(uint32_t)));
    return PFX_OK;
}

// Tile descriptors of plan p with cost slabs at Csk, in queue order (largest
// tile first, then row-major tile index).
void pfx::plan_tile_descs(const pfx_plan* p, const void* Csk, TileDesc* out,
                          const int32_t* slot) {
    const Geo& g = p->g;
    const int nt = g.n1 * g.n2;
    std::vector<int> order(nt);
    for (int t = 0; t < nt; ++t) order[t] = t;
    auto area = [&](int t) {
        int64_t r0, c0;
        int32_t R, W;
        tile_rect(g, t / g.n2, t % g.n2, &r0, &c0, &R, &W);
        return (int64_t)R * W;
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return area(a) > area(b); });
    for (int q = 0; q < nt; ++q) {
        const int t = order[q];
        int64_t r0, c0;
        TileDesc d;
        memset(&d, 0, sizeof(d));
        tile_rect(g, t / g.n2, t % g.n2, &r0, &c0, &d.R, &d.W);
        const int64_t slab = slot ? slot[t] : t;
        d.Csk = (slab < 0 || !Csk)
                    ? nullptr
                    : static_cast<const char*>(Csk) + slab * p->skew_stride * (p->fp32 ? 4 : 8);
        if (p->feat && p->feat_d > 0) {  // for a stage 1 that builds the cost itself
            d.fa = p->feat + r0;
            d.fb = p->feat + (int64_t)p->feat_d * g.N + c0;
            d.lda = (int32_t)g.N;
            d.ldb = (int32_t)g.M;
        }
        d.Bw = p->s1.Bw + (int64_t)t * g.b_words;
        d.eD = p->s1.edge_D + (int64_t)t * 2 * g.L;
        d.eP = p->s1.edge_P + (int64_t)t * 2 * g.L;
        d.L = g.L;
        d.tile = t;
        out[q] = d;
    }
}

extern "C" int pfx_plan_create(int64_t N, int64_t M, int32_t L, const int64_t* steps,
                               const double* weights, int32_t n_steps, pfx_plan** out) {
    return pfx_plan_create_ex(N, M, L, steps, weights, n_steps, PFX_FP64, out);
}

extern "C" int pfx_plan_create_ex(int64_t N, int64_t M, int32_t L, const int64_t* steps,
                                  const double* weights, int32_t n_steps, int32_t precision,
                                  pfx_plan** out) {
    if (!out || !steps || !weights) return fail(PFX_ERR_ARG, "null argument");
    if (precision != PFX_FP64 && precision != PFX_FP32)
        return fail(PFX_ERR_ARG, "precision %d: PFX_FP64 (0) or PFX_FP32 (1)", precision);
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(PFX_ERR_NO_DEVICE, "no CUDA device");
    pfx_plan* p = (pfx_plan*)calloc(1, sizeof(pfx_plan));
    if (!p) return fail(PFX_ERR_ARG, "out of host memory");
    int st = plan_init(p, N, M, L, steps, weights, n_steps, 0, precision == PFX_FP32);
    if (st) {
        pfx_plan_destroy(p);
        return st;
    }
    *out = p;
    return PFX_OK;
}

extern "C" int pfx_plan_set_warps(pfx_plan* p, int32_t nw) {
    if (!p) return fail(PFX_ERR_ARG, "null plan");
    if (nw != 4 && nw != 8 && nw != 16) return fail(PFX_ERR_ARG, "nw=%d: 4, 8 or 16", nw);
    if (stage1_queue_warps(1, p->g.L, 1) == 0 ||
        (nw != 16 && stage1_queue_warps(1 << 30, p->g.L, 1) > nw))
        return fail(PFX_ERR_TOO_LARGE, "L=%d: rings of %d warps do not fit", p->g.L, nw);
    p->nw = nw;
    return PFX_OK;
}

extern "C" int pfx_plan_info(const pfx_plan* p, int64_t* info) {
    if (!p || !info) return fail(PFX_ERR_ARG, "null argument");
    info[0] = p->g.n1;
    info[1] = p->g.n2;
    info[2] = p->g.L;
    info[3] = p->g.hop;
    info[4] = p->g.S;
    info[5] = p->g.b_words;
    info[6] = (int64_t)p->bytes;
    info[7] = p->nw;
    return PFX_OK;
}

extern "C" int pfx_plan_buffer(pfx_plan* p, int which, void** ptr, int64_t* nbytes) {
    if (!p || !ptr || !nbytes) return fail(PFX_ERR_ARG, "null argument");
    const int64_t n4 = p->n4, ms = p->s2.max_segs;
    switch (which) {
        case PFX_BUF_EDGE_D: *ptr = p->s1.edge_D; *nbytes = n4 * 8; break;
        case PFX_BUF_EDGE_P: *ptr = p->s1.edge_P; *nbytes = n4 * 4; break;
        case PFX_BUF_BACKPTR: *ptr = p->s1.Bw; *nbytes = (int64_t)p->g.n1 * p->g.n2 * p->g.b_words * 4; break;
        case PFX_BUF_EDGE_CF: *ptr = p->s2.edge_Cf; *nbytes = n4 * 8; break;
        case PFX_BUF_VALID: *ptr = p->s2.valid; *nbytes = n4; break;
        case PFX_BUF_D_ARR: *ptr = p->s2.D_arr; *nbytes = n4 * 8; break;
        case PFX_BUF_L_ARR: *ptr = p->s2.L_arr; *nbytes = n4 * 8; break;
        case PFX_BUF_TOP_D: *ptr = p->s2.top_D; *nbytes = p->g.M * 8; break;
        case PFX_BUF_TOP_L: *ptr = p->s2.top_L; *nbytes = p->g.M * 8; break;
        case PFX_BUF_RIGHT_D: *ptr = p->s2.right_D; *nbytes = p->g.N * 8; break;
        case PFX_BUF_RIGHT_L: *ptr = p->s2.right_L; *nbytes = p->g.N * 8; break;
        case PFX_BUF_SEG_NORM: *ptr = p->s2.seg_norm; *nbytes = 2 * ms * 8; break;
        case PFX_BUF_SEG_META: *ptr = p->s2.seg_meta; *nbytes = 12 * ms * 8; break;
        case PFX_BUF_D_PROP: *ptr = p->D_prop; *nbytes = n4 * 8; break;
        case PFX_BUF_L_PROP: *ptr = p->L_prop; *nbytes = n4 * 8; break;
        case PFX_BUF_FEAT_BF16:
            if (!p->fbf) return fail(PFX_ERR_ARG, "no bf16 features in the plan");
            *ptr = p->fbf;
            *nbytes = (p->g.N + p->g.M) * p->fbf_kp * 2;
            break;
        case PFX_BUF_COST:
            if (!p->Csk) return fail(PFX_ERR_ARG, "no cost loaded into the plan");
            *ptr = p->Csk;
            *nbytes = plan_slab_bytes(p);
            break;
        default: return fail(PFX_ERR_ARG, "unknown buffer id %d", which);
    }
    return PFX_OK;
}

static int check_ldc(const pfx_plan* p, const double* C, int64_t ldc) {
    if (!C) return fail(PFX_ERR_ARG, "null cost matrix");
    if (ldc < p->g.M) return fail(PFX_ERR_ARG, "ldc=%lld < M=%lld", (long long)ldc, (long long)p->g.M);
    return PFX_OK;
}

// Cost slabs (allocated on first use unless a batch attached its own) and
// the plan's tile queue pointing at them.
static int ensure_cost_buffer(pfx_plan* p) {
    if (p->Csk) return PFX_OK;
    char* slabs = nullptr;
    int st = plan_alloc(p, &slabs, (size_t)plan_slab_bytes(p));
    if (st) return st;
    p->Csk = slabs;
    std::vector<TileDesc> d((size_t)p->g.n1 * p->g.n2);
    plan_tile_descs(p, p->Csk, d.data());
    CK(cudaMemcpy(p->descs, d.data(), d.size() * sizeof(TileDesc), cudaMemcpyHostToDevice));
    return PFX_OK;
}

static const int32_t* active_mask(const pfx_plan* p) {
    return p->mask_active ? p->tile_slot : nullptr;
}

extern "C" int pfx_plan_set_tile_mask(pfx_plan* p, const uint8_t* mask, int32_t on_device,
                                      void* stream) {
    if (!p) return fail(PFX_ERR_ARG, "null plan");
    if (p->range_hi > 0) return fail(PFX_ERR_ARG, "the plan has a tile range: its mask stays");
    if (!mask) {
        p->mask_active = 0;
        p->s2.tile_slot = nullptr;
        return PFX_OK;
    }
    int st;
    if ((st = ensure_cost_buffer(p))) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const int nt = p->g.n1 * p->g.n2;
    CK(cudaMemcpyAsync(p->tile_mask, mask, (size_t)nt,
                       on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    if (!on_device) CK(cudaStreamSynchronize(s));  // the host array may go away
    CK(launch_compact_descs(p->descs, nt, p->tile_mask, p->descs_sub, p->nsub, s));
    // a plan keeps every tile's slab in place: slot = tile where set, -1 elsewhere
    CK(launch_mask_slots(p->tile_mask, nt, p->tile_slot, s));
    p->mask_active = 1;
    p->s2.tile_slot = p->tile_slot;
    return PFX_OK;
}

extern "C" int pfx_plan_set_tile_range(pfx_plan* p, int32_t lo, int32_t hi, void* stream) {
    if (!p) return fail(PFX_ERR_ARG, "null plan");
    const int nt = p->g.n1 * p->g.n2;
    if (lo < 0 || hi > nt || lo >= hi)
        return fail(PFX_ERR_ARG, "tile range [%d, %d) of %d tiles", lo, hi, nt);
    if (p->Csk) return fail(PFX_ERR_ARG, "the plan already holds cost slabs: set the range first");
    p->range_lo = lo;
    p->range_hi = hi;
    char* slabs = nullptr;
    int st = plan_alloc(p, &slabs, (size_t)plan_slab_bytes(p));
    if (st) {
        p->range_lo = p->range_hi = 0;
        return st;
    }
    p->Csk = slabs;
    std::vector<int32_t> slot((size_t)nt, -1);
    std::vector<uint8_t> mask((size_t)nt, 0);
    for (int t = lo; t < hi; ++t) {
        slot[t] = t - lo;
        mask[t] = 1;
    }
    std::vector<TileDesc> d((size_t)nt);
    plan_tile_descs(p, p->Csk, d.data(), slot.data());
    cudaStream_t s = (cudaStream_t)stream;
    CK(cudaMemcpyAsync(p->descs, d.data(), d.size() * sizeof(TileDesc), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(p->tile_mask, mask.data(), (size_t)nt, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(p->tile_slot, slot.data(), (size_t)nt * 4, cudaMemcpyHostToDevice, s));
    CK(launch_compact_descs(p->descs, nt, p->tile_mask, p->descs_sub, p->nsub, s));
    CK(cudaStreamSynchronize(s));  // the host vectors go away
    p->mask_active = 1;
    p->s2.tile_slot = p->tile_slot;
    return PFX_OK;
}

extern "C" int pfx_plan_load_cost(pfx_plan* p, const double* C, int64_t ldc, void* stream) {
    if (!p) return fail(PFX_ERR_ARG, "null plan");
    int st = check_ldc(p, C, ldc);
    if (st) return st;
    if ((st = ensure_cost_buffer(p))) return st;
    if (p->fp32)
        CK(launch_relayout_skew_f32(C, nullptr, ldc, p->g, static_cast<float*>(p->Csk),
                                    p->skew_stride, (cudaStream_t)stream, active_mask(p)));
    else
        CK(launch_relayout_skew(C, ldc, p->g, static_cast<double*>(p->Csk), p->skew_stride,
                                (cudaStream_t)stream, active_mask(p)));
    p->cost_loaded = 1;
    return PFX_OK;
}

extern "C" int pfx_plan_load_cost_f32(pfx_plan* p, const float* C, int64_t ldc, void* stream) {
    if (!p) return fail(PFX_ERR_ARG, "null plan");
    if (!p->fp32) return fail(PFX_ERR_ARG, "pfx_plan_load_cost_f32 needs an FP32 plan");
    if (!C) return fail(PFX_ERR_ARG, "null cost matrix");
    if (ldc < p->g.M) return fail(PFX_ERR_ARG, "ldc=%lld < M=%lld", (long long)ldc, (long long)p->g.M);
    int st;
    if ((st = ensure_cost_buffer(p))) return st;
    CK(launch_relayout_skew_f32(nullptr, C, ldc, p->g, static_cast<float*>(p->Csk),
                                p->skew_stride, (cudaStream_t)stream, active_mask(p)));
    p->cost_loaded = 1;
    return PFX_OK;
}

extern "C" int pfx_plan_load_features(pfx_plan* p, const double* F1, const double* F2, int32_t d,
                                      void* stream) {
    if (!p || !F1 || !F2) return fail(PFX_ERR_ARG, "null argument");
    if (p->fp32) return fail(PFX_ERR_ARG, "FP32 plans build their cost with pfx_plan_load_features_bf16");
    if (d < 1) return fail(PFX_ERR_ARG, "feature dimension %d", d);
    int st;
    if ((st = ensure_cost_buffer(p))) return st;
    if (p->feat && p->feat_d < d) return fail(PFX_ERR_ARG, "feature dimension grew");
    if (!p->feat) {
        if ((st = plan_alloc(p, &p->feat, (size_t)d * (p->g.N + p->g.M)))) return st;
        p->feat_d = d;
    }
    cudaStream_t s = (cudaStream_t)stream;
    double* An = p->feat;
    double* Bn = p->feat + (int64_t)d * p->g.N;
    CK(launch_l2norm(F1, d, p->g.N, An, s));
    CK(launch_l2norm(F2, d, p->g.M, Bn, s));
    CK(launch_cost_skew(An, Bn, d, p->g, static_cast<double*>(p->Csk), p->skew_stride, s,
                        active_mask(p)));
    p->cost_loaded = 1;
    return PFX_OK;
}

extern "C" int pfx_plan_load_features_bf16(pfx_plan* p, const double* F1, const double* F2,
                                           int32_t d, void* stream) {
    if (!p || !F1 || !F2) return fail(PFX_ERR_ARG, "null argument");
    if (!p->fp32) return fail(PFX_ERR_ARG, "pfx_plan_load_features_bf16 needs an FP32 plan");
    if (d < 1 || d > 256)
        return fail(PFX_ERR_ARG, "feature dimension %d: the tensor-core cost takes 1..256", d);
    const int kp = (d + 63) / 64 * 64;
    int st;
    if ((st = ensure_cost_buffer(p))) return st;
    if (p->fbf && p->fbf_kp < kp) return fail(PFX_ERR_ARG, "feature dimension grew");
    if (!p->fbf) {
        char* q = nullptr;
        if ((st = plan_alloc(p, &q, (size_t)(p->g.N + p->g.M) * kp * 2))) return st;
        p->fbf = q;
        p->fbf_kp = kp;
    }
    cudaStream_t s = (cudaStream_t)stream;
    char* A = static_cast<char*>(p->fbf);
    char* B = A + (size_t)p->g.N * p->fbf_kp * 2;
    CK(launch_features_bf16(F1, d, p->g.N, p->fbf_kp, A, s));
    CK(launch_features_bf16(F2, d, p->g.M, p->fbf_kp, B, s));
    CK(launch_gemm_cost_skew(A, B, p->fbf_kp, p->g, static_cast<float*>(p->Csk), p->skew_stride,
                             p->s1.status, s, active_mask(p)));
    p->cost_loaded = 1;
    return PFX_OK;
}

extern "C" int pfx_stage1(pfx_plan* p, const double* C, int64_t ldc, void* stream) {
    if (!p) return fail(PFX_ERR_ARG, "null plan");
    int st;
    if (p->gen_cost)
        return fail(PFX_ERR_ARG, "a batch plan whose stage 1 builds the cost itself keeps no "
                                 "cost slabs: run it through pfx_batch_run");
    if (C && (st = pfx_plan_load_cost(p, C, ldc, stream))) return st;
    if (!p->cost_loaded) return fail(PFX_ERR_ARG, "no cost matrix loaded into the plan");
    cudaStream_t s = (cudaStream_t)stream;
    CK(cudaMemsetAsync(p->head, 0, sizeof(int), s));
    if (p->mask_active) {
        // tiles outside the mask keep +inf edges and start 0
        CK(launch_fill(p->s1.edge_D, p->n4, HUGE_VAL, s));
        CK(cudaMemsetAsync(p->s1.edge_P, 0, (size_t)p->n4 * 4, s));
        CK(launch_stage1_queue(p->descs_sub, p->g.n1 * p->g.n2, p->nsub, p->head, p->g,
                               p->s1.status, p->nw, p->fp32 != 0, s));
    } else {
        const int nt = p->g.n1 * p->g.n2;
        const int sms = num_sms_cur();
        const int maxc = (p->nw == 16 && p->arena_mode == 0 && nt < sms)
                             ? stage1_cluster_max(p->g, p->fp32 != 0)
                             : 0;
        if (maxc > 0) {
            // fewer tiles than SMs: the largest tiles (the queue is ordered
            // largest first) take two SMs each, as many as leave one SM for
            // every other tile and as many clusters as can run at once; the
            // other tiles run at the same time on a second stream
            int nbig = nt < sms - nt ? nt : sms - nt;
            if (nbig > maxc) nbig = maxc;
            if (!p->aux) {
                CK(cudaStreamCreateWithFlags(&p->aux, cudaStreamNonBlocking));
                CK(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
                CK(cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming));
            }
            CK(cudaMemsetAsync(p->head2, 0, sizeof(int), s));
            CK(cudaEventRecord(p->ev_fork, s));
            // the clusters first, so that they find pairs of free SMs
            CK(launch_stage1_cluster(p->descs, nbig, p->head, p->g, p->s1.status,
                                     p->fp32 != 0, s));
            if (nt > nbig) {
                CK(cudaStreamWaitEvent(p->aux, p->ev_fork, 0));
                CK(launch_stage1_queue(p->descs + nbig, nt - nbig, nullptr, p->head2, p->g,
                                       p->s1.status, 16, p->fp32 != 0, p->aux));
                CK(cudaEventRecord(p->ev_join, p->aux));
                CK(cudaStreamWaitEvent(s, p->ev_join, 0));
            }
        } else {
            CK(launch_stage1_queue(p->descs, nt, nullptr, p->head, p->g, p->s1.status, p->nw,
                                   p->fp32 != 0, s));
        }
    }
    return PFX_OK;
}

extern "C" int pfx_stage2_edges(pfx_plan* p, const double* C, int64_t ldc, void* stream) {
    if (!p) return fail(PFX_ERR_ARG, "null plan");
    Geo g = p->g;
    if (C && !p->fp32) {
        int st = check_ldc(p, C, ldc);
        if (st) return st;
        g.ldc = ldc;
    } else if (!p->cost_loaded) {
        return fail(PFX_ERR_ARG, "no cost matrix loaded into the plan");
    }
    if (p->gen_cost) {
        // a batch whose stage 1 built each tile's cost itself keeps no slabs:
        // the overlap costs come from the normalised features
        CK(launch_stage2_edges(nullptr, nullptr, 0, false, g, p->s2, (cudaStream_t)stream,
                               p->feat, p->feat + (int64_t)p->feat_d * g.N, p->feat_d));
        return PFX_OK;
    }
    // the FP32 form reads overlap costs from its own FP32 slabs (the values
    // its DP used), never from an FP64 C
    CK(launch_stage2_edges(p->fp32 ? nullptr : C, p->Csk, p->skew_stride, p->fp32 != 0, g,
                           p->s2, (cudaStream_t)stream));
    return PFX_OK;
}

extern "C" int pfx_stage2_prop(pfx_plan* p, void* stream) {
    if (!p) return fail(PFX_ERR_ARG, "null plan");
    CK(launch_stage2_prop(p->g, p->s2, (cudaStream_t)stream));
    return PFX_OK;
}

extern "C" int pfx_stage2_propagate(pfx_plan* p, const double* C, int64_t ldc, void* stream) {
    int st;
    if ((st = pfx_stage2_edges(p, C, ldc, stream))) return st;
    return pfx_stage2_prop(p, stream);
}

extern "C" int pfx_snapshot_prop(pfx_plan* p, void* stream) {
    if (!p) return fail(PFX_ERR_ARG, "null plan");
    cudaStream_t s = (cudaStream_t)stream;
    CK(cudaMemcpyAsync(p->D_prop, p->s2.D_arr, (size_t)p->n4 * 8, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(p->L_prop, p->s2.L_arr, (size_t)p->n4 * 8, cudaMemcpyDeviceToDevice, s));
    return PFX_OK;
}

static int64_t buffer_global(int64_t N, int64_t M, double beta) {
    // Parflex.py:1520, evaluated in the same order
    const double mn = (double)(N < M ? N : M), mx = (double)(N < M ? M : N);
    const double bg = mn * (1 - (1 - beta) * mn / mx);
    return (int64_t)bg;
}

extern "C" int pfx_stage2_scan(pfx_plan* p, double beta, void* stream) {
    if (!p) return fail(PFX_ERR_ARG, "null plan");
    CK(launch_sync_scan(p->g, p->s2, buffer_global(p->g.N, p->g.M, beta), (cudaStream_t)stream));
    return PFX_OK;
}

extern "C" int pfx_stage2_stitch(pfx_plan* p, int from_best, int64_t i, int64_t j, int64_t edge,
                                 int64_t idx, void* stream) {
    if (!p) return fail(PFX_ERR_ARG, "null plan");
    CK(launch_stitch(p->g, p->s2, (cudaStream_t)stream, from_best, i, j, edge, idx));
    return PFX_OK;
}

extern "C" int pfx_stage2_chain(pfx_plan* p, int from_best, int64_t i, int64_t j, int64_t edge,
                                int64_t idx, int32_t* tiles_host, int32_t cap, int32_t* n_tiles,
                                void* stream) {
    if (!p || !tiles_host || !n_tiles) return fail(PFX_ERR_ARG, "null argument");
    if (cap < 101) return fail(PFX_ERR_ARG, "tiles_host holds %d entries; the chain has up to 101", cap);
    cudaStream_t s = (cudaStream_t)stream;
    CK(launch_stitch_chain(p->g, p->s2, s, from_best, i, j, edge, idx));
    int32_t n = 0;
    int32_t E[12 * 101];
    CK(cudaMemcpyAsync(&n, p->s2.chain_len, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (n < 0 || n > 101) return fail(PFX_ERR_CUDA, "tile chain length %d out of range", n);
    if (n > 0) {
        CK(cudaMemcpyAsync(E, p->s2.chain, sizeof(int32_t) * 12 * n, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
    }
    for (int k = 0; k < n; ++k) {
        tiles_host[2 * k] = E[12 * k];
        tiles_host[2 * k + 1] = E[12 * k + 1];
    }
    *n_tiles = n;
    return PFX_OK;
}

extern "C" int pfx_parflex_device(pfx_plan* p, const double* C, int64_t ldc, double beta,
                                  void* stream) {
    int st;
    if ((st = pfx_stage1(p, C, ldc, stream))) return st;
    if ((st = pfx_stage2_propagate(p, C, ldc, stream))) return st;
    if ((st = pfx_stage2_scan(p, beta, stream))) return st;
    if ((st = pfx_stage2_stitch(p, 1, 0, 0, 0, 0, stream))) return st;
    return PFX_OK;
}

extern "C" int pfx_result(pfx_plan* p, void* stream, double* best_cost, int64_t* best_end7,
                          int64_t* wp_len) {
    if (!p) return fail(PFX_ERR_ARG, "null plan");
    cudaStream_t s = (cudaStream_t)stream;
    double b = 0;
    int64_t e[7];
    int64_t n = 0;
    int32_t kst = 0;
    CK(cudaMemcpyAsync(&kst, p->s1.status, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&b, p->s2.best, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(e, p->s2.best_end, 56, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&n, p->s2.wp_len, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (kst) {
        cudaMemsetAsync(p->s1.status, 0, 4, s);
        return fail(PFX_ERR_CUDA, "a bounded device wait ran out (status %d: 1 stage-1 wavefront, 2 cost GEMM); results invalid",
                    kst);
    }
    if (best_cost) *best_cost = b;
    if (best_end7) memcpy(best_end7, e, sizeof(e));
    if (wp_len) *wp_len = n;
    if (!e[6]) return fail(PFX_ERR_NO_ENDPOINT, "%s", kStatus[PFX_ERR_NO_ENDPOINT]);
    return PFX_OK;
}

extern "C" int pfx_copy_path(pfx_plan* p, void* stream, int64_t* wp_host, int64_t cap) {
    if (!p || !wp_host) return fail(PFX_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    int64_t n = 0;
    CK(cudaMemcpyAsync(&n, p->s2.wp_len, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (n > cap) return fail(PFX_ERR_ARG, "path has %lld points, buffer holds %lld", (long long)n, (long long)cap);
    if (n > 0) CK(cudaMemcpyAsync(wp_host, p->s2.wp, (size_t)n * 16, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return PFX_OK;
}

extern "C" int pfx_parflex(const double* C_host, int64_t N, int64_t M, int64_t ldc,
                           const int64_t* steps, const double* weights, int32_t n_steps,
                           double beta, int32_t L, double* best_cost, int64_t* wp_out,
                           int64_t wp_cap, int64_t* wp_len) {
    if (!C_host || ldc < M) return fail(PFX_ERR_ARG, "bad host cost matrix");
    pfx_plan* p = nullptr;
    int st = pfx_plan_create(N, M, L, steps, weights, n_steps, &p);
    if (st) return st;
    double* Cd = nullptr;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        pfx_plan_destroy(p);
        return fail(PFX_ERR_CUDA, "stream creation failed");
    }
    cudaError_t e = cudaMallocAsync((void**)&Cd, (size_t)N * M * 8, s);
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(Cd, (size_t)M * 8, C_host, (size_t)ldc * 8, (size_t)M * 8, (size_t)N,
                              cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        st = fail(PFX_ERR_CUDA, "cost-matrix upload: %s", cudaGetErrorString(e));
    } else {
        st = pfx_parflex_device(p, Cd, M, beta, s);
        int64_t n = 0;
        if (!st) st = pfx_result(p, s, best_cost, nullptr, &n);
        if (wp_len) *wp_len = n;
        if (!st && wp_out && n <= wp_cap) st = pfx_copy_path(p, s, wp_out, wp_cap);
    }
    if (Cd) cudaFreeAsync(Cd, s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    pfx_plan_destroy(p);
    return st;
}

extern "C" int pfx_cost_matrix_f64(const double* F1, const double* F2, int32_t d, int64_t N,
                                   int64_t M, double* norm_scratch, double* C, int64_t ldc,
                                   void* stream) {
    if (!F1 || !F2 || !norm_scratch || !C) return fail(PFX_ERR_ARG, "null argument");
    if (d < 1 || N < 1 || M < 1 || ldc < M) return fail(PFX_ERR_ARG, "bad shape");
    CK(launch_cost_f64(F1, F2, d, N, M, norm_scratch, norm_scratch + (int64_t)d * N, C, ldc,
                       (cudaStream_t)stream));
    return PFX_OK;
}

extern "C" int pfx_flexdtw_tile(const double* C, int64_t ldc, int32_t R, int32_t W,
                                const int64_t* steps, const double* weights, int32_t n_steps,
                                double* D, int32_t* P, int8_t* B, void* stream) {
    if (!C || !D || !P || !B || !steps || !weights) return fail(PFX_ERR_ARG, "null argument");
    if (R < 1 || W < 1) return fail(PFX_ERR_ARG, "Empty chunk: R=%d, C=%d", R, W);
    if (ldc < W) return fail(PFX_ERR_ARG, "ldc < W");
    Geo g;
    memset(&g, 0, sizeof(g));
    int st = parse_steps(steps, weights, n_steps, &g);
    if (st) return st;
    const int32_t L = R > W ? R : W;
    g.N = R;
    g.M = W;
    g.ldc = ldc;
    g.L = L < 2 ? 2 : L;
    g.hop = g.L - 1;
    g.n1 = 1;
    g.n2 = 1;
    g.b_words = tile_b_words(g.L);
    if ((st = check_smem(g.L, 8))) return st;
    cudaStream_t s = (cudaStream_t)stream;
    S1Out o;
    memset(&o, 0, sizeof(o));
    const size_t eb = (size_t)2 * g.L;
    CK(cudaMallocAsync((void**)&o.edge_D, eb * 8, s));
    CK(cudaMallocAsync((void**)&o.edge_P, eb * 4, s));
    CK(cudaMallocAsync((void**)&o.Bw, (size_t)g.b_words * 4, s));
    o.full_D = D;
    o.full_P = P;
    o.full_B = B;
    cudaError_t e = cudaSuccess;
    if (R == 1 || W == 1) {
        // no DP cells: D = C, P = 0, B = 0 (FlexDTW.py:329-334)
        e = cudaMemcpy2DAsync(D, (size_t)W * 8, C, (size_t)ldc * 8, (size_t)W * 8, (size_t)R,
                              cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(P, 0, (size_t)R * W * 4, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(B, 0, (size_t)R * W, s);
    } else {
        e = launch_stage1(C, g, o, 0, 1, 8, true, s);
    }
    cudaFreeAsync(o.edge_D, s);
    cudaFreeAsync(o.edge_P, s);
    cudaFreeAsync(o.Bw, s);
    if (e != cudaSuccess) return fail(PFX_ERR_CUDA, "tile DP: %s", cudaGetErrorString(e));
    return PFX_OK;
}
