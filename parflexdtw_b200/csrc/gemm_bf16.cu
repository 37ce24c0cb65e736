// FP32 form cost: C = 1 - bf16(L2norm(F1))^T bf16(L2norm(F2)) on the 5th-gen
// tensor cores, written straight into the FP32 tile-skewed slabs that the
// FP32 stage-1 kernel reads.
//
// One CTA (4 warps) produces the skewed rows tau in [128 cb, 128 cb + 128) of
// the two 64-row strips 2 kk, 2 kk + 1 of one tile.  Those rows hold the cells
// (rho, tau - rho), rho < 64, i.e. rows 128 kk + [0, 128) and columns
// 128 cb - 64 + [1, 192) of the tile: a 128 x 192 block of C (the 64 extra
// columns overlap the neighbouring CTA; tensor-core work is cheap next to
// the slab write, which bounds this kernel).
//
//   TMA (SWIZZLE_128B, K-major boxes of 64 bf16 x rows; rows outside the
//   sequences, e.g. the negative column offset of the first block, arrive as
//   zeros) -> shared memory -> tcgen05.mma.cta_group::1.kind::f16 (BF16 in,
//   FP32 accumulate, M = 128, N = 192, K = 16 per instruction) into a TMEM
//   accumulator of 192 columns -> tcgen05.ld (32 lanes x 32 columns per warp
//   and step) -> 1 - acc, masked to 0 outside the tile -> shared memory in
//   skewed order (address 65 rho + const: conflict-free) -> 256-byte rows of
//   float2 per warp to global (streaming stores).
//
// Every wait is bounded: a wait that runs out sets the status word, waits
// (bounded) for the CTA's own copies or MMAs still in flight, frees its TMEM
// and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "common.cuh"

namespace pfx {

constexpr int kGRows = 128;              // C rows per CTA (two strips)
constexpr int kGSteps = 128;             // skewed steps per CTA
constexpr int kGCols = kGSteps + 64;     // C columns per CTA (MMA N)
constexpr int kGThreads = 128;
constexpr int kGTmemCols = 256;          // power of two >= kGCols
constexpr int kGAtomBytes = 128;         // SWIZZLE_128B: 64 bf16 of K per row
constexpr int kGWaitLimit = 1 << 22;
constexpr int32_t kStatusGemmWait = 2;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Bounded wait for phase `parity` of an mbarrier (non-blocking test and a
// short sleep per round, ~0.5 s in all); false when it ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (int it = 0; it < kGWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Shared-memory matrix descriptor: K-major, SWIZZLE_128B canonical layout
// (rows 128 B apart, 8-row groups 1024 B apart), version 1, base offset 0.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);  // start address, bits [0, 14)
    d |= (uint64_t)1 << 16;                   // leading byte offset (16 B units), unused here
    d |= (uint64_t)(1024 >> 4) << 32;         // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1 << 46;                   // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                   // layout: SWIZZLE_128B
    return d;
}

// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 D, M x N.
__host__ __device__ constexpr uint32_t mma_idesc_bf16(int M, int N) {
    return (1u << 4)                    // D format F32
           | (1u << 7)                  // A format BF16
           | (1u << 10)                 // B format BF16
           | ((uint32_t)(N >> 3) << 17)  // N / 8
           | ((uint32_t)(M >> 4) << 24);  // M / 16
}

template <int KB>  // feature dimension padded to 64 * KB
__global__ void __launch_bounds__(kGThreads, 1)
    k_gemm_cost_skew(const __grid_constant__ CUtensorMap mapA,
                     const __grid_constant__ CUtensorMap mapB, const Geo g,
                     float* __restrict__ Csk, const int64_t stride,
                     int32_t* __restrict__ status, const int32_t* __restrict__ slot,
                     const int32_t* __restrict__ list) {
    extern __shared__ __align__(1024) unsigned char gsm_raw[];
    // operands (1024-byte aligned atoms), later reused as the skew stage
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(gsm_raw) + 1023) & ~(uintptr_t)1023);
    unsigned char* sA = base;                                  // [KB][128 rows][128 B]
    unsigned char* sB = base + KB * kGRows * kGAtomBytes;     // [KB][192 rows][128 B]
    float* Ssk = reinterpret_cast<float*>(base);               // [2][128 steps][64 rows]
    __shared__ __align__(8) uint64_t bar_tma, bar_mma;
    __shared__ uint32_t tmem_base_slot;

    // CTA -> (tile, strip pair, step block)
    const Sched2 sL = make_sched2(g.L, g.L, 1);
    const int nkk = (sL.nS + 1) / 2, ncb = ceil_div32(sL.span, kGSteps);
    int q = (int)blockIdx.x;
    const int cb = q % ncb;
    q /= ncb;
    const int kk = q % nkk;
    const int tile = list ? list[q / nkk] : q / nkk;
    const int slab = slot ? slot[tile] : tile;  // slab index; < 0: tile skipped
    if (slab < 0) return;  // uniform over the CTA
    int64_t r0, c0;
    int32_t R, W;
    tile_rect(g, tile / g.n2, tile % g.n2, &r0, &c0, &R, &W);
    const int span = ceil_div32(W + kStripRows - 1, kBlk) * kBlk;
    const int nS = ceil_div32(R, kStripRows);
    if (2 * kk >= nS || cb * kGSteps >= span) return;  // uniform over the CTA

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_slot)),
                     "r"(kGTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar_tma, 1);
        mbar_init(&bar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_slot;

    __shared__ int s_fail;
    if (threadIdx.x == 0) {
        s_fail = 0;
        const uint32_t bytes = KB * (kGRows + kGCols) * kGAtomBytes;
        mbar_expect_tx(&bar_tma, bytes);
        const int ya = (int)(r0 + (int64_t)kGRows * kk);
        const int yb = (int)(c0 + (int64_t)kGSteps * cb - 64);
#pragma unroll
        for (int kb = 0; kb < KB; ++kb) {
            tma_load_2d(sA + kb * kGRows * kGAtomBytes, &mapA, 64 * kb, ya, &bar_tma);
            tma_load_2d(sB + kb * kGCols * kGAtomBytes, &mapB, 64 * kb, yb, &bar_tma);
        }
        bool ok = mbar_wait(&bar_tma, 0);
        if (!ok) {
            atomicExch(status, kStatusGemmWait);
            mbar_wait(&bar_tma, 0);  // the copies target this CTA's memory: let them land
            s_fail = 1;
        } else {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            constexpr uint32_t idesc = mma_idesc_bf16(kGRows, kGCols);
#pragma unroll
            for (int kb = 0; kb < KB; ++kb) {
#pragma unroll
                for (int k16 = 0; k16 < 4; ++k16) {
                    const uint64_t da = sw128_desc(smem_u32(sA + kb * kGRows * kGAtomBytes) + 32 * k16);
                    const uint64_t db = sw128_desc(smem_u32(sB + kb * kGCols * kGAtomBytes) + 32 * k16);
                    const uint32_t acc = (kb | k16) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                        "l"(da), "l"(db), "r"(idesc), "r"(acc)
                        : "memory");
                }
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smem_u32(&bar_mma))
                : "memory");
            if (!mbar_wait(&bar_mma, 0)) {
                atomicExch(status, kStatusGemmWait);
                mbar_wait(&bar_mma, 0);
                s_fail = 1;
            }
        }
    }
    __syncthreads();
    if (!s_fail) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // accumulator lanes 32 warp + lane = CTA-local row, columns = window columns
        const int row = 32 * warp + lane;
        const int s = row >> 6, rho = row & 63;
        const int r = kGRows * kk + row;  // tile-local row
        const int cbase = kGSteps * cb - 64;
        const bool row_in = r < R;
#pragma unroll 1
        for (int j0 = 0; j0 < kGCols; j0 += 32) {
            uint32_t v[32];
            const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)j0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                "[%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                  "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                  "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
                  "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                  "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
                  "=r"(v[30]), "=r"(v[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int cw = j0 + j;             // window column
                const int tl = cw - 64 + rho;      // CTA-local step of cell (row, cw)
                if (tl >= 0 && tl < kGSteps) {
                    const int c = cbase + cw;      // tile-local column
                    const float val = (row_in && c >= 0 && c < W)
                                          ? __fsub_rn(1.0f, __uint_as_float(v[j]))
                                          : 0.0f;
                    Ssk[(s * kGSteps + tl) * 64 + rho] = val;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kGTmemCols));
    }
    if (s_fail) return;
    // skewed rows out: 32 lanes x float2 = 256 contiguous bytes per (strip, step)
    float2* out = reinterpret_cast<float2*>(Csk + (int64_t)slab * stride);
#pragma unroll 4
    for (int i = threadIdx.x; i < 2 * kGSteps * 32; i += kGThreads) {
        const int s = i / (kGSteps * 32);
        const int tl = (i / 32) % kGSteps;
        const int l = i & 31;
        const int k = 2 * kk + s, tau = kGSteps * cb + tl;
        if (k < nS && tau < span) {
            const float2 v2 = *reinterpret_cast<const float2*>(&Ssk[(s * kGSteps + tl) * 64 + 2 * l]);
            __stcs(out + ((int64_t)k * span + tau) * 32 + l, v2);
        }
    }
}

// bf16 copy of L2-normalised features: F (d x n, FP64, row-major by feature)
// -> out[n][Kp] (row per frame, zero past d), normalised in FP64 with the
// same summation as the FP64 form, then rounded to nearest bf16.
__global__ void k_features_bf16(const double* __restrict__ F, int d, int64_t n, int Kp,
                                __nv_bfloat16* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double ss = 0.0;
    for (int f = 0; f < d; ++f) {
        const double x = F[(int64_t)f * n + i];
        ss = __dadd_rn(ss, __dmul_rn(x, x));
    }
    const double nr = sqrt(ss);
    for (int f = 0; f < Kp; ++f) {
        const double x = f < d ? (nr > 0.0 ? __ddiv_rn(F[(int64_t)f * n + i], nr) : 0.0) : 0.0;
        out[i * Kp + f] = __double2bfloat16(x);
    }
}

cudaError_t launch_features_bf16(const double* F, int d, int64_t n, int Kp, void* out,
                                 cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_features_bf16<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(
        F, d, n, Kp, static_cast<__nv_bfloat16*>(out));
    count_launches(1);
    return cudaGetLastError();
}

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// Tensor map of a [rows][Kp] bf16 matrix read in boxes of 64 x box_rows.
static bool make_map(CUtensorMap* m, const void* base, int64_t rows, int Kp, int box_rows) {
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)Kp * 2};
    cuuint32_t box[2] = {64, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box,
              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

size_t gemm_cost_smem_bytes(int Kp) {
    const size_t ops = (size_t)(Kp / 64) * (kGRows + kGCols) * kGAtomBytes;
    const size_t stage = (size_t)2 * kGSteps * 64 * sizeof(float);
    // at least ~100 KB: at most two CTAs (2 x 256 TMEM columns) per SM
    size_t b = (ops > stage ? ops : stage) + 1024;
    return b < 100 * 1024 ? 100 * 1024 : b;
}

template <int KB>
static cudaError_t gemm_t(const CUtensorMap& ma, const CUtensorMap& mb, const Geo& g, float* Csk,
                          int64_t stride, int32_t* status, cudaStream_t st, const int32_t* slot,
                          const int32_t* list, int nlist) {
    const size_t smem = gemm_cost_smem_bytes(64 * KB);
    auto kern = k_gemm_cost_skew<KB>;
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const Sched2 s = make_sched2(g.L, g.L, 1);
    const int64_t nblk =
        (list ? (int64_t)nlist : (int64_t)g.n1 * g.n2) * ((s.nS + 1) / 2) *
        ceil_div32(s.span, kGSteps);
    if (nblk > 0x7fffffffLL) return cudaErrorInvalidValue;
    if (nblk == 0) return cudaSuccess;
    kern<<<(unsigned)nblk, kGThreads, smem, st>>>(ma, mb, g, Csk, stride, status, slot, list);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_gemm_cost_skew(const void* Abf, const void* Bbf, int Kp, const Geo& g,
                                  float* Csk, int64_t stride, int32_t* status, cudaStream_t st,
                                  const int32_t* slot, const int32_t* list, int nlist) {
    if (Kp % 64 || Kp < 64 || Kp > 256) return cudaErrorInvalidValue;
    CUtensorMap ma, mb;
    if (!make_map(&ma, Abf, g.N, Kp, kGRows) || !make_map(&mb, Bbf, g.M, Kp, kGCols))
        return cudaErrorInvalidValue;
    switch (Kp / 64) {
        case 1: return gemm_t<1>(ma, mb, g, Csk, stride, status, st, slot, list, nlist);
        case 2: return gemm_t<2>(ma, mb, g, Csk, stride, status, st, slot, list, nlist);
        case 3: return gemm_t<3>(ma, mb, g, Csk, stride, status, st, slot, list, nlist);
        default: return gemm_t<4>(ma, mb, g, Csk, stride, status, st, slot, list, nlist);
    }
}

}  // namespace pfx
