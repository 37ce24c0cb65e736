// pfx_flexdtw_tile_noalloc: the single-tile FlexDTW DP without any device
// memory allocation.
//
// Who needs it: callers that cannot call cudaMalloc.  An online score
// follower that aligns each incoming block of audio frames against a
// reference tile must not block on the allocator or take the implicit
// device-wide synchronisation that cudaMalloc / cudaFree can cause, once per
// block; a host application or plugin framework that reserves all device
// memory up front may forbid the library from allocating at all.
// pfx_flexdtw_tile allocates the kernel's scratch (tile edge rows and packed
// backpointers) with cudaMallocAsync on every call; this variant keeps that
// scratch in one file-scope device array instead.
//
// Limits and sharing:
//   * Tiles up to kMaxTile x kMaxTile (2048 x 2048); larger tiles are
//     rejected with PFX_ERR_TOO_LARGE before anything is launched.
//   * The array (about 1.1 MB) lives in every GPU that loads this library,
//     until the process exits.
//   * Every call on a device uses the same array and the array keeps the
//     last call's contents.  The kernel only writes the scratch and never
//     reads it back, so nothing in it has to be cleared between calls, but
//     calls that overlap on the GPU (issued on different streams without
//     ordering) race on it.  Order such calls on one stream.
//   * The first call on each device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current) and caches it; make
//     that first call before any stream capture.  The cache is keyed on the
//     CUDA context's unique id as well as the device, so a call made after a
//     device reset, or under another context of the same device, looks the
//     address up again in the context it runs in.
#include <cstring>
#include <mutex>

#include "common.cuh"

namespace {

constexpr int32_t kMaxTile = 2048;
constexpr size_t kEdgeDBytes = sizeof(double) * 2 * kMaxTile;
constexpr size_t kEdgePBytes = sizeof(int32_t) * 2 * kMaxTile;
// packed backpointers of a kMaxTile x kMaxTile tile: 32-row strips x
// 16-step periods x 32 lanes (see pfx::tile_b_words)
constexpr size_t kStrips = (kMaxTile + 31) / 32;
constexpr size_t kPeriods = (kMaxTile + 31 + pfx::kBlk - 1) / pfx::kBlk;
constexpr size_t kBWordBytes = sizeof(uint32_t) * kStrips * kPeriods * 32;
constexpr size_t kScratchBytes = kEdgeDBytes + kEdgePBytes + kBWordBytes;

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};  // context id the address belongs to

// Unique id of the calling thread's current context (never reused within a
// process, unlike a context handle), through the driver entry point the
// runtime hands out; false when no context is current or the driver lacks
// the call.
bool current_context_id(unsigned long long* id) {
    using CtxGetId = CUresult (*)(CUcontext, unsigned long long*);
    static CtxGetId fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<CtxGetId>(p);
    }();
    return fn && fn(nullptr, id) == CUDA_SUCCESS;
}

}  // namespace

// The scratch itself.  In host code this name is only a host-side stand-in,
// not a device address (a kernel given it would fault or silently use the
// wrong memory); the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_tile_scratch[kScratchBytes];

namespace {
// Device address of g_tile_scratch on the current device (looked up once per
// device and context, under a lock, with that device current; without a
// context id from the driver it is looked up on every call).
int scratch_address(void** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return pfx::report_status(PFX_ERR_NO_DEVICE, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return pfx::report_status(PFX_ERR_ARG, "device ordinal beyond the scratch table");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    unsigned long long ctx = 0;
    const bool have_ctx = current_context_id(&ctx);
    if (have_ctx && g_scratch_addr[dev] && g_scratch_ctx[dev] == ctx) {
        *out = g_scratch_addr[dev];
        return PFX_OK;
    }
    // first call in this context (the lookup also makes the device's primary
    // context current when the thread had none)
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_tile_scratch);
    if (e != cudaSuccess || !p)
        return pfx::report_status(PFX_ERR_CUDA, e != cudaSuccess ? cudaGetErrorString(e)
                                                                 : "null scratch address");
    if (have_ctx || current_context_id(&ctx)) {
        g_scratch_addr[dev] = p;
        g_scratch_ctx[dev] = ctx;
    }
    *out = p;
    return PFX_OK;
}

}  // namespace

extern "C" int pfx_flexdtw_tile_noalloc(const double* C, int64_t ldc, int32_t R, int32_t W,
                                        const int64_t* steps, const double* weights,
                                        int32_t n_steps, double* D, int32_t* P, int8_t* B,
                                        void* stream) {
    using namespace pfx;
    if (!C || !D || !P || !B || !steps || !weights)
        return report_status(PFX_ERR_ARG, "null argument");
    if (R < 1 || W < 1) return report_status(PFX_ERR_ARG, "Empty chunk");
    if (ldc < W) return report_status(PFX_ERR_ARG, "ldc < W");
    if (R > kMaxTile || W > kMaxTile)
        return report_status(PFX_ERR_TOO_LARGE,
                             "pfx_flexdtw_tile_noalloc takes tiles up to 2048 x 2048 "
                             "(its scratch is a fixed device array); use pfx_flexdtw_tile");
    Geo g;
    memset(&g, 0, sizeof(g));
    int st = parse_step_kinds(steps, weights, n_steps, &g);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    if (R == 1 || W == 1) {
        // no DP cells: D = C, P = 0, B = 0 (FlexDTW.py:329-334)
        cudaError_t e = cudaMemcpy2DAsync(D, (size_t)W * 8, C, (size_t)ldc * 8, (size_t)W * 8,
                                          (size_t)R, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(P, 0, (size_t)R * W * 4, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(B, 0, (size_t)R * W, s);
        return e == cudaSuccess ? PFX_OK : report_status(PFX_ERR_CUDA, cudaGetErrorString(e));
    }
    void* base = nullptr;
    if ((st = scratch_address(&base))) return st;
    const int32_t L = R > W ? R : W;
    g.N = R;
    g.M = W;
    g.ldc = ldc;
    g.L = L;
    g.hop = L - 1;
    g.n1 = 1;
    g.n2 = 1;
    g.b_words = tile_b_words(L);
    S1Out o;
    memset(&o, 0, sizeof(o));
    unsigned char* b = static_cast<unsigned char*>(base);
    o.edge_D = reinterpret_cast<double*>(b);
    o.edge_P = reinterpret_cast<int32_t*>(b + kEdgeDBytes);
    o.Bw = reinterpret_cast<uint32_t*>(b + kEdgeDBytes + kEdgePBytes);
    o.full_D = D;
    o.full_P = P;
    o.full_B = B;
    const cudaError_t e = launch_stage1(C, g, o, 0, 1, 8, true, s);
    return e == cudaSuccess ? PFX_OK : report_status(PFX_ERR_CUDA, cudaGetErrorString(e));
}
