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
// restatement used by the tests.  The FMA variant (FMA = true) forms the
// same sum as a chain of fused multiply-adds in the same order (the first
// product rounded on its own): 13 FP64 operations per cell instead of 24,
// bit-identical to the oracle's fma chain (oracle_cost_fma).
#include "common.cuh"

namespace pfx {

constexpr int kTC = 256;               // skewed steps per CTA
constexpr int kWinStride = kTC + 64;   // window columns (TC + 63 used, 1 pad); the
                                       // diagonal read stride 319 is odd: conflict-free
constexpr int kMaxFeat = 16;           // features staged in shared memory

template <typename T>
__device__ __forceinline__ void write_skewed(const T* __restrict__ S, T* __restrict__ Cs,
                                             int span, int k, int ts) {
    const int nt = (span - ts) < kTC ? (span - ts) : kTC;
    for (int q = threadIdx.x; q < nt * 64; q += blockDim.x) {
        const int tt = q >> 6, rho = q & 63;
        const int x = tt - rho + 63;  // window column of (rho, ts + tt - rho)
        Cs[((int64_t)k * span + ts + tt) * 64 + rho] = S[rho * kWinStride + x];
    }
}

constexpr int kRegionThreads = 512;

// Row-major C (Tin) -> skewed slabs (Tout; FP64 -> FP32 rounds to nearest).
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(kRegionThreads) k_region_skew(const Tin* __restrict__ C,
                                                               int64_t ldc, const Geo g,
                                                               Tout* __restrict__ Csk,
                                                               int64_t stride,
                                                               const int32_t* __restrict__ slot) {
    extern __shared__ __align__(16) unsigned char S_raw[];
    Tout* S = reinterpret_cast<Tout*>(S_raw);  // [64][kWinStride]
    // blockIdx.x enumerates (tile, step chunk) pairs, blockIdx.y the strip
    const int nchunk = ceil_div32(make_sched2(g.L, g.L, 1).span, kTC);
    const int tile = (int)(blockIdx.x / nchunk), k = blockIdx.y;
    const int ts = (int)(blockIdx.x % nchunk) * kTC;
    const int slab = slot ? slot[tile] : tile;  // slab index; < 0: tile skipped
    if (slab < 0) return;
    const int ti = tile / g.n2, tj = tile % g.n2;
    int64_t r0, c0;
    int32_t R, W;
    tile_rect(g, ti, tj, &r0, &c0, &R, &W);
    const Sched2 sc = make_sched2(R, W, 1);
    if (k >= sc.nS || ts >= sc.span) return;
    const int col0 = ts - 63;  // tile-local column of window column 0
    // 40 elements per thread, issued as independent loads before the stores
    constexpr int kPer = 64 * kWinStride / kRegionThreads;
    Tout v[kPer];
#pragma unroll
    for (int u = 0; u < kPer; ++u) {
        const int q = threadIdx.x + u * kRegionThreads;
        const int rho = q / kWinStride, x = q % kWinStride;
        const int r = 64 * k + rho, c = col0 + x;
        v[u] = (r < R && c >= 0 && c < W) ? (Tout)__ldcs(C + (r0 + r) * ldc + c0 + c) : (Tout)0;
    }
#pragma unroll
    for (int u = 0; u < kPer; ++u) S[threadIdx.x + u * kRegionThreads] = v[u];
    __syncthreads();
    write_skewed(S, Csk + (int64_t)slab * stride, sc.span, k, ts);
}

// ---------------------------------------------------------------------------
// Cost from features straight into the skewed layout.  Lane l of a warp owns
// rows 64k + 2l (A) and 64k + 2l + 1 (B) of strip k -- the stage-1 mapping --
// and produces 8 consecutive steps tau per pass: A = (64k+2l, tau-2l),
// B = (64k+2l+1, tau-2l-1), stored as one 16-byte (A, B) pair per lane and
// step, so a warp writes 512 contiguous bytes per step.  B's column at tau
// is A's column at tau-1: one pass reads 9 column vectors for 16 cells of a
// strip (k_cost_skew takes two strips at once: 32 cells).  Column features of the CTA's window are
// staged in shared memory split by column parity; at one instruction every
// lane reads the same parity at consecutive half-indices (conflict-free).
constexpr int kCT = 256;                // steps per CTA
constexpr int kCV = 8;                  // steps per register pass
constexpr int kCostThreads = 256;       // 8 warps x 32 steps
constexpr int kCX = kCT + 66;           // window columns (x = c - ts + 64), even
constexpr int kCH = kCX / 2;            // per parity

// Two strips per CTA (blockIdx.y = strip pair): rows 64k + rho of strips 2kk
// and 2kk + 1 sit at the same column for a given step, so each column vector
// read from shared memory serves four cells of a lane.  The rows' features
// are staged in shared memory too ([f][strip][64 rows], one 16-byte (A, B)
// pair per lane: conflict-free), which keeps the registers to 32 sums.
template <int DMAX, bool FMA>
__global__ void __launch_bounds__(kCostThreads, 2)
    k_cost_skew(const double* __restrict__ An, const double* __restrict__ Bn, const int d,
                const Geo g, double* __restrict__ Csk, const int64_t stride,
                const int32_t* __restrict__ slot, const int32_t* __restrict__ list) {
    extern __shared__ __align__(16) double sB[];  // [d][2][kCH], then sA [d][2][64]
    double* sA = sB + d * kCX;
    const int nchunk = ceil_div32(make_sched2(g.L, g.L, 1).span, kCT);
    const int tile = list ? list[blockIdx.x / nchunk] : (int)(blockIdx.x / nchunk);
    const int kk = blockIdx.y;
    const int ts = (int)(blockIdx.x % nchunk) * kCT;
    const int slab = slot ? slot[tile] : tile;  // slab index; < 0: tile skipped
    if (slab < 0) return;
    int64_t r0, c0;
    int32_t R, W;
    tile_rect(g, tile / g.n2, tile % g.n2, &r0, &c0, &R, &W);
    const int span = ceil_div32(W + kStripRows - 1, kBlk) * kBlk;
    const int nS = ceil_div32(R, kStripRows);
    if (2 * kk >= nS || ts >= span) return;
    const bool two = 2 * kk + 1 < nS;
    // the features, as asynchronous copies all in flight at once (one
    // memory latency per CTA, not one per element of a thread)
    for (int q = threadIdx.x; q < d * kCX; q += kCostThreads) {
        const int f = q / kCX, x = q - f * kCX;
        const int c = ts - 64 + x;
        const bool in = c >= 0 && c < W;
        cp_async8(sB + (f * 2 + (x & 1)) * kCH + (x >> 1), in ? Bn + (int64_t)f * g.M + c0 + c : Bn,
                  in);
    }
    for (int q = threadIdx.x; q < d * 128; q += kCostThreads) {
        const int f = q >> 7, r = 128 * kk + (q & 127);
        cp_async8(sA + q, r < R ? An + (int64_t)f * g.N + r0 + r : An, r < R);
    }
    cp_async_wait_all();
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int rA0 = 128 * kk + 2 * lane, rB0 = rA0 + 1, rA1 = rA0 + 64, rB1 = rA1 + 1;
    const double2* sA2 = reinterpret_cast<const double2*>(sA);  // [f][strip][32 lanes]
    double2* out0 = reinterpret_cast<double2*>(Csk + (int64_t)slab * stride) +
                    (int64_t)(2 * kk) * span * 32 + lane;
    double2* out1 = out0 + (int64_t)span * 32;
#pragma unroll 1
    for (int blk = 0; blk < 32 / kCV; ++blk) {
        const int t0 = ts + 32 * warp + kCV * blk;  // warp-uniform
        if (t0 >= span) break;
        // A's column at t0 + v is window x = t0 - ts + 64 - 2*lane + v (even at v = 0);
        // b[j] holds x = xA0 - 1 + j, j = 0..8 (B at v uses b[v], A uses b[v + 1])
        const int h0 = ((t0 - ts + 64) >> 1) - lane;  // half-index of xA0
        double accA0[kCV], accB0[kCV], accA1[kCV], accB1[kCV];
#pragma unroll
        for (int f = 0; f < DMAX; ++f) {
            if (f >= d) break;
            const double* se = sB + (f * 2) * kCH;  // even x
            const double* so = se + kCH;             // odd x
            double b[kCV + 1];
#pragma unroll
            for (int j = 0; j <= kCV; ++j) {
                // x = 2*h0 - 1 + j: odd for even j (half-index h0 - 1 + j/2), even for odd j
                b[j] = (j & 1) ? se[h0 + (j >> 1)] : so[h0 - 1 + (j >> 1)];
            }
            const double2 a0 = sA2[(f * 2) * 32 + lane], a1 = sA2[(f * 2 + 1) * 32 + lane];
#pragma unroll
            for (int v = 0; v < kCV; ++v) {
                if (FMA && f > 0) {
                    accA0[v] = __fma_rn(a0.x, b[v + 1], accA0[v]);
                    accB0[v] = __fma_rn(a0.y, b[v], accB0[v]);
                    accA1[v] = __fma_rn(a1.x, b[v + 1], accA1[v]);
                    accB1[v] = __fma_rn(a1.y, b[v], accB1[v]);
                } else {
                    const double pA0 = __dmul_rn(a0.x, b[v + 1]);
                    const double pB0 = __dmul_rn(a0.y, b[v]);
                    const double pA1 = __dmul_rn(a1.x, b[v + 1]);
                    const double pB1 = __dmul_rn(a1.y, b[v]);
                    accA0[v] = f == 0 ? pA0 : __dadd_rn(accA0[v], pA0);
                    accB0[v] = f == 0 ? pB0 : __dadd_rn(accB0[v], pB0);
                    accA1[v] = f == 0 ? pA1 : __dadd_rn(accA1[v], pA1);
                    accB1[v] = f == 0 ? pB1 : __dadd_rn(accB1[v], pB1);
                }
            }
        }
#pragma unroll
        for (int v = 0; v < kCV; ++v) {
            const int tau = t0 + v;
            if (tau < span) {
                const int cA = tau - 2 * lane, cB = cA - 1;
                const bool inA = cA >= 0 && cA < W, inB = cB >= 0 && cB < W;
                __stcs(out0 + (int64_t)tau * 32,
                       make_double2((rA0 < R && inA) ? __dsub_rn(1.0, accA0[v]) : 0.0,
                                    (rB0 < R && inB) ? __dsub_rn(1.0, accB0[v]) : 0.0));
                if (two)
                    __stcs(out1 + (int64_t)tau * 32,
                           make_double2((rA1 < R && inA) ? __dsub_rn(1.0, accA1[v]) : 0.0,
                                        (rB1 < R && inB) ? __dsub_rn(1.0, accB1[v]) : 0.0));
            }
        }
    }
}

// Any feature dimension: the same mapping with 64 steps per CTA (one
// 8-step pass per warp), the features taken 16 at a time (columns staged per
// chunk, rows re-read per chunk) while the 16 sums of a lane stay in
// registers, so the fixed summation order f = 0, 1, ..., d-1 is kept.
constexpr int kCT2 = 64;
constexpr int kCX2 = kCT2 + 66;
constexpr int kCH2 = kCX2 / 2;

template <bool FMA>
__global__ void __launch_bounds__(kCostThreads, 2)
    k_cost_skew_chunked(const double* __restrict__ An, const double* __restrict__ Bn, const int d,
                        const Geo g, double* __restrict__ Csk, const int64_t stride,
                        const int32_t* __restrict__ slot, const int32_t* __restrict__ list) {
    __shared__ __align__(16) double sB[kMaxFeat * kCX2];  // [16][2][kCH2]
    const int nchunk = ceil_div32(make_sched2(g.L, g.L, 1).span, kCT2);
    const int tile = list ? list[blockIdx.x / nchunk] : (int)(blockIdx.x / nchunk);
    const int k = blockIdx.y;
    const int ts = (int)(blockIdx.x % nchunk) * kCT2;
    const int slab = slot ? slot[tile] : tile;  // slab index; < 0: tile skipped
    if (slab < 0) return;
    int64_t r0, c0;
    int32_t R, W;
    tile_rect(g, tile / g.n2, tile % g.n2, &r0, &c0, &R, &W);
    const int span = ceil_div32(W + kStripRows - 1, kBlk) * kBlk;
    const int nS = ceil_div32(R, kStripRows);
    if (k >= nS || ts >= span) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int rA = 64 * k + 2 * lane, rB = rA + 1;
    const int t0 = ts + kCV * warp;  // this warp's 8 steps
    const int h0 = ((t0 - ts + 64) >> 1) - lane;
    double accA[kCV], accB[kCV];
    for (int f0 = 0; f0 < d; f0 += kMaxFeat) {
        const int nf = d - f0 < kMaxFeat ? d - f0 : kMaxFeat;
        __syncthreads();  // the previous chunk's columns are consumed
        for (int q = threadIdx.x; q < nf * kCX2; q += kCostThreads) {
            const int f = q / kCX2, x = q - f * kCX2;
            const int c = ts - 64 + x;
            const bool in = c >= 0 && c < W;
            cp_async8(sB + (f * 2 + (x & 1)) * kCH2 + (x >> 1),
                      in ? Bn + (int64_t)(f0 + f) * g.M + c0 + c : Bn, in);
        }
        cp_async_wait_all();
        __syncthreads();
        if (t0 < span) {
#pragma unroll 4
            for (int f = 0; f < nf; ++f) {
                const double aA = rA < R ? __ldg(An + (int64_t)(f0 + f) * g.N + r0 + rA) : 0.0;
                const double aB = rB < R ? __ldg(An + (int64_t)(f0 + f) * g.N + r0 + rB) : 0.0;
                const double* se = sB + (f * 2) * kCH2;
                const double* so = se + kCH2;
                double b[kCV + 1];
#pragma unroll
                for (int j = 0; j <= kCV; ++j)
                    b[j] = (j & 1) ? se[h0 + (j >> 1)] : so[h0 - 1 + (j >> 1)];
                const bool first = f0 + f == 0;
#pragma unroll
                for (int v = 0; v < kCV; ++v) {
                    if (FMA && !first) {
                        accA[v] = __fma_rn(aA, b[v + 1], accA[v]);
                        accB[v] = __fma_rn(aB, b[v], accB[v]);
                    } else {
                        const double pA = __dmul_rn(aA, b[v + 1]);
                        const double pB = __dmul_rn(aB, b[v]);
                        accA[v] = first ? pA : __dadd_rn(accA[v], pA);
                        accB[v] = first ? pB : __dadd_rn(accB[v], pB);
                    }
                }
            }
        }
    }
    if (t0 >= span) return;
    double2* out = reinterpret_cast<double2*>(Csk + (int64_t)slab * stride) + (int64_t)k * span * 32 + lane;
#pragma unroll
    for (int v = 0; v < kCV; ++v) {
        const int tau = t0 + v;
        if (tau < span) {
            const int cA = tau - 2 * lane, cB = cA - 1;
            const double vA = (rA < R && cA >= 0 && cA < W) ? __dsub_rn(1.0, accA[v]) : 0.0;
            const double vB = (rB < R && cB >= 0 && cB < W) ? __dsub_rn(1.0, accB[v]) : 0.0;
            __stcs(out + (int64_t)tau * 32, make_double2(vA, vB));
        }
    }
}

// ntiles: the tiles enumerated (all n1 * n2, or the length of a tile list)
static dim3 region_grid(const Geo& g, int per_cta, int64_t ntiles = -1) {
    const Sched2 s = make_sched2(g.L, g.L, 1);
    if (ntiles < 0) ntiles = (int64_t)g.n1 * g.n2;
    return dim3((unsigned)(ceil_div32(s.span, per_cta) * ntiles), (unsigned)s.nS, 1);
}

template <typename Tin, typename Tout>
static cudaError_t relayout_t(const Tin* C, int64_t ldc, const Geo& g, Tout* Csk, int64_t stride,
                              cudaStream_t st, const int32_t* slot) {
    const size_t smem = (size_t)64 * kWinStride * sizeof(Tout);
    auto kern = k_region_skew<Tin, Tout>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<region_grid(g, kTC), kRegionThreads, smem, st>>>(C, ldc, g, Csk, stride, slot);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_relayout_skew(const double* C, int64_t ldc, const Geo& g, double* Csk,
                                 int64_t stride, cudaStream_t st, const int32_t* slot) {
    return relayout_t(C, ldc, g, Csk, stride, st, slot);
}

cudaError_t launch_relayout_skew_f32(const double* C64, const float* C32, int64_t ldc,
                                     const Geo& g, float* Csk, int64_t stride, cudaStream_t st,
                                     const int32_t* slot) {
    return C32 ? relayout_t(C32, ldc, g, Csk, stride, st, slot)
               : relayout_t(C64, ldc, g, Csk, stride, st, slot);
}

template <bool FMA>
static cudaError_t cost_skew_t(const double* An, const double* Bn, int d, const Geo& g,
                               double* Csk, int64_t stride, cudaStream_t st, const int32_t* slot,
                               const int32_t* list, int64_t nt) {
    if (d > kMaxFeat) {
        k_cost_skew_chunked<FMA><<<region_grid(g, kCT2, nt), kCostThreads, 0, st>>>(
            An, Bn, d, g, Csk, stride, slot, list);
        count_launches(1);
        return cudaGetLastError();
    }
    const size_t smem = (size_t)d * (kCX + 128) * sizeof(double);
    dim3 grid = region_grid(g, kCT, nt);
    grid.y = (grid.y + 1) / 2;  // strip pairs
    cudaError_t e;
    if (d == 12) {
        e = cudaFuncSetAttribute(k_cost_skew<12, FMA>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_cost_skew<12, FMA><<<grid, kCostThreads, smem, st>>>(An, Bn, d, g, Csk, stride, slot,
                                                               list);
    } else {
        e = cudaFuncSetAttribute(k_cost_skew<kMaxFeat, FMA>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        k_cost_skew<kMaxFeat, FMA><<<grid, kCostThreads, smem, st>>>(An, Bn, d, g, Csk, stride,
                                                                     slot, list);
    }
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_cost_skew(const double* An, const double* Bn, int d, const Geo& g, double* Csk,
                             int64_t stride, cudaStream_t st, const int32_t* slot,
                             const int32_t* list, int nlist, bool fma) {
    if (d < 1) return cudaErrorInvalidValue;
    const int64_t nt = list ? nlist : -1;
    if (list && nlist == 0) return cudaSuccess;
    return fma ? cost_skew_t<true>(An, Bn, d, g, Csk, stride, st, slot, list, nt)
               : cost_skew_t<false>(An, Bn, d, g, Csk, stride, st, slot, list, nt);
}

}  // namespace pfx
