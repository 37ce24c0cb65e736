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
#include <string.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "common.cuh"

namespace pfx {

constexpr int kGRows = 128;              // C rows per CTA (two strips)
constexpr int kGSteps = 128;             // skewed steps per CTA
constexpr int kGCols = kGSteps + 64;     // C columns per CTA (MMA N)
constexpr int kGEpiWarps = 12;           // epilogue warps: 3 per TMEM lane quarter,
                                         // 2 of the 6 column chunks each
constexpr int kGThreads = 32 * (2 + kGEpiWarps);  // + producer warp, MMA warp
constexpr int kGAccCols = 256;           // TMEM columns per accumulator (>= kGCols)
constexpr int kGTmemCols = 2 * kGAccCols;  // two accumulators
constexpr int kGAtomBytes = 128;         // SWIZZLE_128B: 64 bf16 of K per row
constexpr int kGWaitLimit = 1 << 22;
constexpr int32_t kStatusGemmWait = 2;
constexpr int32_t kStatusGemmBounds = 3;  // a block's tile or slab range out of bounds (skipped)

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

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait that also gives up when another role of the CTA aborted.
__device__ __forceinline__ bool mbar_wait_ab(uint64_t* bar, uint32_t parity,
                                             const volatile int* abort) {
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
        if (*abort) return false;
        if (it > 32) __nanosleep(64);
    }
    return false;
}

// (tile, strip pair kk, step block cb) of block q, with the operands and the
// output slabs of its pair; false for blocks past a small tile's strips or
// steps (every role skips them alike).
struct GBlock {
    int slab, kk, cb, nS, span, R, W;
    int64_t r0, c0;
    const CUtensorMap* ma;
    const CUtensorMap* mb;
    float* Csk;
    int64_t stride, cap;
};

__device__ __forceinline__ bool gemm_tile(const Geo& g, int tile, int kk, int cb, GBlock& b) {
    b.kk = kk;
    b.cb = cb;
    tile_rect(g, tile / g.n2, tile % g.n2, &b.r0, &b.c0, &b.R, &b.W);
    b.span = ceil_div32(b.W + kStripRows - 1, kBlk) * kBlk;
    b.nS = ceil_div32(b.R, kStripRows);
    return 2 * b.kk < b.nS && b.cb * kGSteps < b.span;
}

__device__ __forceinline__ bool gemm_block(const Geo& g, const int32_t* slot, const int32_t* list,
                                           int nkk, int ncb, int64_t q, GBlock& b,
                                           int32_t* status) {
    const int cb = (int)(q % ncb);
    q /= ncb;
    const int kk = (int)(q % nkk);
    const int tile = list ? list[q / nkk] : (int)(q / nkk);
    if (tile < 0 || tile >= g.n1 * g.n2) {
        atomicExch(status, kStatusGemmBounds);
        return false;
    }
    b.slab = slot ? slot[tile] : tile;
    if (b.slab < 0) return false;
    return gemm_tile(g, tile, kk, cb, b);
}

// Block q of a multi-pair launch: its pair by binary search on blk0.
__device__ __forceinline__ bool gemm_block_multi(const GPair* pairs, int npairs, int64_t q,
                                                 GBlock& b) {
    int lo = 0, hi = npairs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pairs[mid].blk0 <= q) lo = mid;
        else hi = mid - 1;
    }
    const GPair& P = pairs[lo];
    int64_t ql = q - P.blk0;
    const int cb = (int)(ql % P.ncb);
    ql /= P.ncb;
    const int kk = (int)(ql % P.nkk);
    const int tile = (int)(ql / P.nkk);
    if (tile >= P.g.n1 * P.g.n2) return false;
    b.slab = tile;
    b.ma = &P.ma;
    b.mb = &P.mb;
    b.Csk = P.Csk;
    b.stride = P.stride;
    b.cap = (int64_t)P.g.n1 * P.g.n2 * P.stride;
    return gemm_tile(P.g, tile, kk, cb, b);
}

// Persistent, warp-specialised: warp 0 loads operands (TMA, NST stages),
// warp 1 issues the MMAs into one of two TMEM accumulators, warps 2-5 read
// the other accumulator, skew it through shared memory and store it with
// bulk copies -- so block i's epilogue overlaps block i+1's loads and MMAs.
template <int KB, int NST, int NSK>  // features padded to 64 * KB; operand stages;
                                     // skew staging buffers
__global__ void __launch_bounds__(kGThreads, 1)
    k_gemm_cost_skew(const __grid_constant__ CUtensorMap mapA,
                     const __grid_constant__ CUtensorMap mapB, const Geo g,
                     float* __restrict__ Csk, const int64_t stride,
                     int32_t* __restrict__ status, const int32_t* __restrict__ slot,
                     const int32_t* __restrict__ list, const int64_t nblk, const int64_t cap,
                     const GPair* __restrict__ pairs, const int npairs) {
    extern __shared__ __align__(1024) unsigned char gsm_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(gsm_raw) + 1023) & ~(uintptr_t)1023);
    constexpr uint32_t kABytes = KB * kGRows * kGAtomBytes;  // [KB][128 rows][128 B]
    constexpr uint32_t kBBytes = KB * kGCols * kGAtomBytes;  // [KB][192 rows][128 B]
    constexpr uint32_t kStage = kABytes + kBBytes;
    // NSK buffers of [2 strips][128 steps][64 rows]
    float* Ssk0 = reinterpret_cast<float*>(base + NST * kStage);
    __shared__ __align__(8) uint64_t full[NST], empty[NST], tfull[2], tempty[2];
    __shared__ uint32_t tmem_base_slot;
    __shared__ volatile int s_abort;
    __shared__ int s_issued, s_consumed, s_mma, s_epi, s_go;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_slot)),
                     "r"(kGTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 32) {
        for (int i = 0; i < NST; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int j = 0; j < 2; ++j) {
            mbar_init(&tfull[j], 1);
            mbar_init(&tempty[j], kGEpiWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
        s_issued = s_consumed = s_mma = s_epi = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_slot;
    const Sched2 sL = make_sched2(g.L, g.L, 1);
    const int nkk = (sL.nS + 1) / 2, ncb = ceil_div32(sL.span, kGSteps);
    // block q: of the one pair given by the parameters, or of the pair table
    auto next_block = [&](int64_t q, GBlock& b) -> bool {
        if (pairs) return gemm_block_multi(pairs, npairs, q, b);
        b.ma = &mapA;
        b.mb = &mapB;
        b.Csk = Csk;
        b.stride = stride;
        b.cap = cap;
        return gemm_block(g, slot, list, nkk, ncb, q, b, status);
    };
    auto fail = [&]() {
        atomicExch(status, kStatusGemmWait);
        s_abort = 1;
    };

    if (warp == 0) {  // producer: the whole warp walks the blocks, lane 0 issues
        int i = 0;
        for (int64_t q = blockIdx.x; q < nblk; q += gridDim.x) {
            GBlock b;
            if (!next_block(q, b)) continue;
            const int st = i % NST;
            int ok = 1;
            if (lane == 0) ok = mbar_wait_ab(&empty[st], ((i / NST) & 1) ^ 1, &s_abort);
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) {
                if (lane == 0) fail();
                break;
            }
            if (lane == 0) {
                unsigned char* sA = base + st * kStage;
                unsigned char* sB = sA + kABytes;
                mbar_expect_tx(&full[st], kStage);
                const int ya = (int)(b.r0 + (int64_t)kGRows * b.kk);
                const int yb = (int)(b.c0 + (int64_t)kGSteps * b.cb - 64);
#pragma unroll
                for (int kb = 0; kb < KB; ++kb) {
                    tma_load_2d(sA + kb * kGRows * kGAtomBytes, b.ma, 64 * kb, ya, &full[st]);
                    tma_load_2d(sB + kb * kGCols * kGAtomBytes, b.mb, 64 * kb, yb, &full[st]);
                }
                s_issued = i + 1;
            }
            __syncwarp();
            ++i;
        }
    } else if (warp == 1) {  // MMA issuer: the whole warp walks the blocks, lane 0 issues
        constexpr uint32_t idesc = mma_idesc_bf16(kGRows, kGCols);
        int i = 0;
        for (int64_t q = blockIdx.x; q < nblk; q += gridDim.x) {
            GBlock b;
            if (!next_block(q, b)) continue;
            const int st = i % NST, j = i & 1;
            int ok = 1;
            if (lane == 0) {
                ok = mbar_wait_ab(&full[st], (i / NST) & 1, &s_abort);
                if (ok) {
                    s_consumed = i + 1;
                    ok = mbar_wait_ab(&tempty[j], ((i >> 1) & 1) ^ 1, &s_abort);
                }
            }
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) {
                if (lane == 0) fail();
                break;
            }
            if (lane == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t sA = smem_u32(base + st * kStage), sB = sA + kABytes;
                const uint32_t d = tmem + (uint32_t)(kGAccCols * j);
#pragma unroll
                for (int kb = 0; kb < KB; ++kb) {
#pragma unroll
                    for (int k16 = 0; k16 < 4; ++k16) {
                        const uint64_t da = sw128_desc(sA + kb * kGRows * kGAtomBytes + 32 * k16);
                        const uint64_t db = sw128_desc(sB + kb * kGCols * kGAtomBytes + 32 * k16);
                        const uint32_t acc = (kb | k16) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
                            "l"(da), "l"(db), "r"(idesc), "r"(acc)
                            : "memory");
                    }
                }
                asm volatile(
                    "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
                    "[%0];" ::"r"(smem_u32(&empty[st]))
                    : "memory");
                asm volatile(
                    "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 "
                    "[%0];" ::"r"(smem_u32(&tfull[j]))
                    : "memory");
                s_mma = i + 1;
            }
            __syncwarp();
            ++i;
        }
    } else {  // epilogue: TMEM lanes 32 (warp % 4) + [0, 32), column chunks 2e, 2e + 1
        const int ew = warp - 2;
        const bool leader = ew == 0 && lane == 0;
        const int quarter = warp & 3, e = ew >> 2;
        const int row = 32 * quarter + lane;
        const int sr = row >> 6, rho = row & 63;
        int i = 0;
        for (int64_t q = blockIdx.x; q < nblk; q += gridDim.x) {
            GBlock b;
            if (!next_block(q, b)) continue;
            const int j = i & 1;
            float* Ssk = Ssk0 + (i % NSK) * (2 * kGSteps * 64);
            // one thread waits (for the accumulator, and for the bulk store
            // that last read this staging buffer); the decision reaches every
            // epilogue warp through the named barrier, which none may leave
            if (leader) {
                const bool ok = mbar_wait_ab(&tfull[j], (i >> 1) & 1, &s_abort);
                if (!ok) fail();
                else s_epi = i + 1;
                asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(NSK - 1) : "memory");
                s_go = ok ? 1 : 0;
            }
            __syncwarp();
            asm volatile("bar.sync 1, %0;" ::"r"(32 * kGEpiWarps) : "memory");
            if (!s_go) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const bool row_in = kGRows * b.kk + row < b.R;  // tile-local row inside
            // rows of this warp: rho0 .. rho0 + 31
            const int rho0 = (32 * quarter) & 63;
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const int j0 = 32 * (2 * e + cc);         // first window column
                // steps of the chunk's cells: t0 + jj, t0 = j0 - 64 + rho
                const int tlo = j0 - 64 + rho0, thi = tlo + 31 + 31;
                if (thi < 0 || tlo >= kGSteps) continue;  // no cell of the chunk is kept
                uint32_t v[32];
                const uint32_t taddr = tmem + ((uint32_t)(32 * quarter) << 16) +
                                       (uint32_t)(kGAccCols * j + j0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                    "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                    "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, "
                    "%31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                      "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                      "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
                      "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                      "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]),
                      "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                const int t0 = j0 - 64 + rho;
                const int c0 = kGSteps * b.cb - 64 + j0;  // tile-local column at jj = 0
                float* dst = Ssk + (sr * kGSteps + t0) * 64 + rho;
#pragma unroll
                for (int jj = 0; jj < 32; ++jj)
                    if ((unsigned)(t0 + jj) < (unsigned)kGSteps)
                        dst[jj * 64] = (row_in && c0 + jj >= 0 && c0 + jj < b.W)
                                           ? __fsub_rn(1.0f, __uint_as_float(v[jj]))
                                           : 0.0f;
            }
            // the accumulator is free for block i + 2
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[j]);
            // skewed rows out: (strip, step) rows of 256 B are contiguous per strip
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            asm volatile("bar.sync 1, %0;" ::"r"(32 * kGEpiWarps) : "memory");
            if (leader) {
                float* out = b.Csk + (int64_t)b.slab * b.stride;
                const int tau0 = kGSteps * b.cb;
                const int nt = b.span - tau0 < kGSteps ? b.span - tau0 : kGSteps;
                for (int s2 = 0; s2 < 2; ++s2) {
                    const int k = 2 * b.kk + s2;
                    if (k >= b.nS) break;
                    // the rows stay inside the slab, the slab inside the buffer
                    const int64_t r_lo = ((int64_t)k * b.span + tau0) * 64;
                    const int64_t r_hi = r_lo + (int64_t)nt * 64;
                    if (nt <= 0 || r_hi > b.stride || (int64_t)b.slab * b.stride + r_hi > b.cap) {
                        atomicExch(status, kStatusGemmBounds);
                        continue;
                    }
                    float* gdst = out + r_lo;
                    asm volatile(
                        "cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst),
                        "r"(smem_u32(Ssk + s2 * kGSteps * 64)), "r"(nt * 256)
                        : "memory");
                }
                asm volatile("cp.async.bulk.commit_group;" ::: "memory");
            }
            ++i;
        }
        if (leader) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
    __syncwarp();
    __syncthreads();
    // let this CTA's copies and MMAs in flight land before it exits (bounded;
    // on the normal path only the last MMA commits are still to be observed)
    if (threadIdx.x == 0) {
        for (int i = s_consumed; i < s_issued; ++i) mbar_wait(&full[i % NST], (i / NST) & 1);
    }
    if (threadIdx.x == 32) {
        for (int i = s_mma - NST > 0 ? s_mma - NST : 0; i < s_mma; ++i)
            mbar_wait(&empty[i % NST], (i / NST) & 1);
        for (int i = s_epi; i < s_mma; ++i) mbar_wait(&tfull[i & 1], (i >> 1) & 1);
    }
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kGTmemCols));
    }
}

// bf16 copy of L2-normalised features: F (d x n, FP64, row-major by feature)
// -> out[n][Kp] (row per frame, zero past d), normalised in FP64 with the
// same summation as the FP64 form, then rounded to nearest bf16.  A block
// takes 32 frames: one thread per frame sums its squares (fixed order), then
// all threads produce the block's rows -- contiguous in `out` -- one word
// (two bf16) per thread and step, coalesced.
constexpr int kFbFrames = 32;
constexpr int kFbThreads = 256;

// Block b of a segment list: the segment holding it (segs ordered by blk0).
__device__ __forceinline__ int fb_segment(const FbSeg* segs, int nseg, int64_t b) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (segs[mid].blk0 <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// segs == nullptr: the single segment `one`.
__global__ void __launch_bounds__(kFbThreads)
    k_features_bf16(const FbSeg* __restrict__ segs, int nseg, FbSeg one, int d, int Kp) {
    __shared__ double nrm[kFbFrames];
    const FbSeg sg = segs ? segs[fb_segment(segs, nseg, blockIdx.x)] : one;
    const double* __restrict__ F = sg.F;
    const int64_t n = sg.n;
    const int64_t i0 = (blockIdx.x - sg.blk0) * (int64_t)kFbFrames;
    const int rows = n - i0 < kFbFrames ? (int)(n - i0) : kFbFrames;
    const int t = threadIdx.x;
    if (t < rows) {
        double ss = 0.0;
        for (int f = 0; f < d; ++f) {
            const double x = F[(int64_t)f * n + i0 + t];
            ss = __dadd_rn(ss, __dmul_rn(x, x));
        }
        nrm[t] = sqrt(ss);
    }
    __syncthreads();
    const int W2 = Kp / 2;
    uint32_t* o = reinterpret_cast<uint32_t*>(static_cast<__nv_bfloat16*>(sg.out) + i0 * Kp);
    for (int w = t; w < rows * W2; w += kFbThreads) {
        const int fr = w / W2, f = 2 * (w % W2);
        const double nr = nrm[fr];
        const int64_t i = i0 + fr;
        const double x0 = f < d ? (nr > 0.0 ? __ddiv_rn(F[(int64_t)f * n + i], nr) : 0.0) : 0.0;
        const double x1 =
            f + 1 < d ? (nr > 0.0 ? __ddiv_rn(F[(int64_t)(f + 1) * n + i], nr) : 0.0) : 0.0;
        const __nv_bfloat162 pr = __halves2bfloat162(__double2bfloat16(x0), __double2bfloat16(x1));
        o[w] = *reinterpret_cast<const uint32_t*>(&pr);
    }
}

int64_t features_bf16_blocks(int64_t n) { return (n + kFbFrames - 1) / kFbFrames; }

cudaError_t launch_features_bf16(const double* F, int d, int64_t n, int Kp, void* out,
                                 cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (Kp % 2) return cudaErrorInvalidValue;
    const FbSeg one{F, n, out, 0};
    k_features_bf16<<<(unsigned)features_bf16_blocks(n), kFbThreads, 0, st>>>(nullptr, 1, one, d,
                                                                               Kp);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_features_bf16_segs(const FbSeg* segs, int nseg, int64_t blocks, int d, int Kp,
                                      cudaStream_t st) {
    if (blocks <= 0) return cudaSuccess;
    if (Kp % 2 || blocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    k_features_bf16<<<(unsigned)blocks, kFbThreads, 0, st>>>(segs, nseg, FbSeg{}, d, Kp);
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

// Operand stages and skew staging buffers within the 227 KB of shared memory:
// KB 1: 2 + 2, KB 2: 1 + 2 (the second accumulator already overlaps the next
// block's loads with this block's epilogue; 2 + 1 measured the same), KB 3-4:
// 1 + 1.
constexpr int gemm_stages(int KB) { return KB == 1 ? 2 : 1; }
constexpr int gemm_skew_bufs(int KB) { return KB <= 2 ? 2 : 1; }

size_t gemm_cost_smem_bytes(int Kp) {
    const int KB = Kp / 64;
    const size_t stage = (size_t)KB * (kGRows + kGCols) * kGAtomBytes;
    const size_t skew = (size_t)2 * kGSteps * 64 * sizeof(float);
    return gemm_stages(KB) * stage + gemm_skew_bufs(KB) * skew + 1024;  // + 1024 B alignment
}

template <int KB>
static cudaError_t gemm_t(const CUtensorMap& ma, const CUtensorMap& mb, const Geo& g, float* Csk,
                          int64_t stride, int32_t* status, cudaStream_t st, const int32_t* slot,
                          const int32_t* list, int nlist, int64_t cap) {
    const size_t smem = gemm_cost_smem_bytes(64 * KB);
    auto kern = k_gemm_cost_skew<KB, gemm_stages(KB), gemm_skew_bufs(KB)>;
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const Sched2 s = make_sched2(g.L, g.L, 1);
    const int64_t nblk =
        (list ? (int64_t)nlist : (int64_t)g.n1 * g.n2) * ((s.nS + 1) / 2) *
        ceil_div32(s.span, kGSteps);
    if (nblk == 0) return cudaSuccess;
    // persistent: one CTA per SM (its two accumulators hold all 512 TMEM columns)
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = (int)(nblk < sms ? nblk : (int64_t)sms);
    if (cap < 0) cap = (int64_t)g.n1 * g.n2 * stride;
    kern<<<grid, kGThreads, smem, st>>>(ma, mb, g, Csk, stride, status, slot, list, nblk, cap,
                                        nullptr, 0);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_gemm_cost_skew(const void* Abf, const void* Bbf, int Kp, const Geo& g,
                                  float* Csk, int64_t stride, int32_t* status, cudaStream_t st,
                                  const int32_t* slot, const int32_t* list, int nlist,
                                  int64_t cap) {
    if (Kp % 64 || Kp < 64 || Kp > 256) return cudaErrorInvalidValue;
    CUtensorMap ma, mb;
    if (!make_map(&ma, Abf, g.N, Kp, kGRows) || !make_map(&mb, Bbf, g.M, Kp, kGCols))
        return cudaErrorInvalidValue;
    switch (Kp / 64) {
        case 1: return gemm_t<1>(ma, mb, g, Csk, stride, status, st, slot, list, nlist, cap);
        case 2: return gemm_t<2>(ma, mb, g, Csk, stride, status, st, slot, list, nlist, cap);
        case 3: return gemm_t<3>(ma, mb, g, Csk, stride, status, st, slot, list, nlist, cap);
        default: return gemm_t<4>(ma, mb, g, Csk, stride, status, st, slot, list, nlist, cap);
    }
}

int64_t gemm_pair_setup(const void* Abf, const void* Bbf, int Kp, const Geo& g, float* Csk,
                        int64_t stride, int64_t blk0, GPair* out) {
    memset(out, 0, sizeof(GPair));
    if (!make_map(&out->ma, Abf, g.N, Kp, kGRows) || !make_map(&out->mb, Bbf, g.M, Kp, kGCols))
        return 0;
    const Sched2 s = make_sched2(g.L, g.L, 1);
    out->g = g;
    out->Csk = Csk;
    out->stride = stride;
    out->blk0 = blk0;
    out->nkk = (s.nS + 1) / 2;
    out->ncb = ceil_div32(s.span, kGSteps);
    return (int64_t)g.n1 * g.n2 * out->nkk * out->ncb;
}

template <int KB>
static cudaError_t gemm_multi_t(const GPair* pairs, int npairs, int64_t nblk, int32_t* status,
                                cudaStream_t st) {
    const size_t smem = gemm_cost_smem_bytes(64 * KB);
    auto kern = k_gemm_cost_skew<KB, gemm_stages(KB), gemm_skew_bufs(KB)>;
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (nblk <= 0 || npairs <= 0) return cudaSuccess;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = (int)(nblk < sms ? nblk : (int64_t)sms);
    CUtensorMap none;
    memset(&none, 0, sizeof(none));
    Geo g0;
    memset(&g0, 0, sizeof(g0));
    g0.L = 1;
    kern<<<grid, kGThreads, smem, st>>>(none, none, g0, nullptr, 0, status, nullptr, nullptr,
                                        nblk, 0, pairs, npairs);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_gemm_cost_multi(const GPair* pairs, int npairs, int64_t nblk, int Kp,
                                   int32_t* status, cudaStream_t st) {
    if (Kp % 64 || Kp < 64 || Kp > 256) return cudaErrorInvalidValue;
    switch (Kp / 64) {
        case 1: return gemm_multi_t<1>(pairs, npairs, nblk, status, st);
        case 2: return gemm_multi_t<2>(pairs, npairs, nblk, status, st);
        case 3: return gemm_multi_t<3>(pairs, npairs, nblk, status, st);
        default: return gemm_multi_t<4>(pairs, npairs, nblk, status, st);
    }
}

}  // namespace pfx
