// Tile-skewed cost layout for the stage-1 kernel (see skew_index):
// element (tile, strip k, step tau, lane, half) = C[r0 + 64k + 2*lane + half]
// [c0 + tau - 2*lane - half], zero outside the tile.
//
// One CTA fills a 64-row x (TC + 63)-column window of C in shared memory --
// copied from a row-major C, or computed from the normalised features -- and
// writes the TC skewed steps it covers as contiguous 512-byte rows.
//
// From features the value is 1 - sum_f A[f][row] * B[f][col] with the sum
// taken in the fixed order f = 0, 1, ..., d-1 and every product and sum
// rounded separately: bit-identical to k_cost_f64 and to the fixed-order host
// restatement used by the tests.
#include "common.cuh"

namespace pfx {

constexpr int kTC = 256;               // skewed steps per CTA
constexpr int kWinStride = kTC + 64;   // window columns (TC + 63 used, 1 pad); the
                                       // diagonal read stride 319 is odd: conflict-free
constexpr int kMaxFeat = 16;           // features staged in shared memory

__device__ __forceinline__ void write_skewed(const double* __restrict__ S, double* __restrict__ Cs,
                                             int span, int k, int ts) {
    const int nt = (span - ts) < kTC ? (span - ts) : kTC;
    for (int q = threadIdx.x; q < nt * 64; q += blockDim.x) {
        const int tt = q >> 6, rho = q & 63;
        const int x = tt - rho + 63;  // window column of (rho, ts + tt - rho)
        Cs[((int64_t)k * span + ts + tt) * 64 + rho] = S[rho * kWinStride + x];
    }
}

constexpr int kRegionThreads = 512;

template <bool FEAT>
__global__ void __launch_bounds__(kRegionThreads) k_region_skew(const double* __restrict__ C, int64_t ldc,
                                                     const double* __restrict__ An,
                                                     const double* __restrict__ Bn, int d,
                                                     const Geo g, double* __restrict__ Csk,
                                                     int64_t stride) {
    extern __shared__ __align__(16) double S[];  // [64][kWinStride] (+ features)
    // blockIdx.x enumerates (tile, step chunk) pairs, blockIdx.y the strip
    const int nchunk = ceil_div32(make_sched2(g.L, g.L, 1).span, kTC);
    const int tile = (int)(blockIdx.x / nchunk), k = blockIdx.y;
    const int ts = (int)(blockIdx.x % nchunk) * kTC;
    const int ti = tile / g.n2, tj = tile % g.n2;
    int64_t r0, c0;
    int32_t R, W;
    tile_rect(g, ti, tj, &r0, &c0, &R, &W);
    const Sched2 sc = make_sched2(R, W, 1);
    if (k >= sc.nS || ts >= sc.span) return;
    const int col0 = ts - 63;  // tile-local column of window column 0
    if (!FEAT) {
        // 40 elements per thread, issued as independent loads before the stores
        constexpr int kPer = 64 * kWinStride / kRegionThreads;
        double v[kPer];
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int q = threadIdx.x + u * kRegionThreads;
            const int rho = q / kWinStride, x = q % kWinStride;
            const int r = 64 * k + rho, c = col0 + x;
            v[u] = (r < R && c >= 0 && c < W) ? __ldcs(C + (r0 + r) * ldc + c0 + c) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kPer; ++u) S[threadIdx.x + u * kRegionThreads] = v[u];
    } else {
        double* sA = S + 64 * kWinStride;        // [kMaxFeat][64]
        double* sB = sA + kMaxFeat * 64;         // [kMaxFeat][kWinStride]
        for (int q = threadIdx.x; q < d * 64; q += blockDim.x) {
            const int f = q / 64, rho = q % 64;
            const int r = 64 * k + rho;
            sA[f * 64 + rho] = r < R ? An[(int64_t)f * g.N + r0 + r] : 0.0;
        }
        for (int q = threadIdx.x; q < d * kWinStride; q += blockDim.x) {
            const int f = q / kWinStride, x = q % kWinStride;
            const int c = col0 + x;
            sB[f * kWinStride + x] = (c >= 0 && c < W) ? Bn[(int64_t)f * g.M + c0 + c] : 0.0;
        }
        __syncthreads();
        // 4 rows x 5 window columns (stride XB, so neighbouring threads read
        // neighbouring columns) per thread and pass: 1024 micro-tiles
        constexpr int XB = kWinStride / 5;  // 64
        for (int q = threadIdx.x; q < 16 * XB; q += blockDim.x) {
            const int rg = q / XB, xg = q % XB;
            double acc[4][5];
#pragma unroll
            for (int f = 0; f < kMaxFeat; ++f) {
                if (f >= d) break;
                double a[4], b[5];
#pragma unroll
                for (int u = 0; u < 4; ++u) a[u] = sA[f * 64 + rg * 4 + u];
#pragma unroll
                for (int v = 0; v < 5; ++v) b[v] = sB[f * kWinStride + xg + XB * v];
#pragma unroll
                for (int u = 0; u < 4; ++u)
#pragma unroll
                    for (int v = 0; v < 5; ++v)
                        acc[u][v] = f == 0 ? __dmul_rn(a[u], b[v])
                                           : __dadd_rn(acc[u][v], __dmul_rn(a[u], b[v]));
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int rho = rg * 4 + u, r = 64 * k + rho;
#pragma unroll
                for (int v = 0; v < 5; ++v) {
                    const int x = xg + XB * v, c = col0 + x;
                    S[rho * kWinStride + x] =
                        (r < R && c >= 0 && c < W) ? __dsub_rn(1.0, acc[u][v]) : 0.0;
                }
            }
        }
    }
    __syncthreads();
    write_skewed(S, Csk + (int64_t)tile * stride, sc.span, k, ts);
}

static size_t region_smem(bool feat) {
    size_t b = (size_t)64 * kWinStride * sizeof(double);
    if (feat) b += (size_t)kMaxFeat * (64 + kWinStride) * sizeof(double);
    return b;
}

static dim3 region_grid(const Geo& g) {
    const Sched2 s = make_sched2(g.L, g.L, 1);
    return dim3((unsigned)(ceil_div32(s.span, kTC) * (int64_t)g.n1 * g.n2), (unsigned)s.nS, 1);
}

cudaError_t launch_relayout_skew(const double* C, int64_t ldc, const Geo& g, double* Csk,
                                 int64_t stride, cudaStream_t st) {
    const size_t smem = region_smem(false);
    cudaError_t e = cudaFuncSetAttribute(k_region_skew<false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_region_skew<false><<<region_grid(g), kRegionThreads, smem, st>>>(C, ldc, nullptr, nullptr, 0, g, Csk,
                                                           stride);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_cost_skew(const double* An, const double* Bn, int d, const Geo& g, double* Csk,
                             int64_t stride, cudaStream_t st) {
    if (d < 1 || d > kMaxFeat) return cudaErrorInvalidValue;
    const size_t smem = region_smem(true);
    cudaError_t e = cudaFuncSetAttribute(k_region_skew<true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_region_skew<true><<<region_grid(g), kRegionThreads, smem, st>>>(nullptr, 0, An, Bn, d, g, Csk, stride);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace pfx
