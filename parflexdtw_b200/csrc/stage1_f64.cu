// Stage 1: FlexDTW on every L x L tile, FP64, one CTA per tile.
//
// Recurrence (FlexDTW.py:326-370): D[0,:] = C[0,:], D[:,0] = C[:,0], P = 0 and
// B = 0 on those boundary cells.  For r, c >= 1 and each step s in the
// caller's order with the predecessor in bounds:
//     pathcost = D[pred] + C[r,c] * w[s]                (two IEEE roundings)
//     mdist    = r + c - |P[pred]|
//     q        = pathcost / mdist                       (IEEE division)
// the first step with the smallest q (strict <) wins; D = its pathcost,
// B = s, P = the predecessor's column if it lies on row 0, minus its row if it
// lies on column 0, else the predecessor's P.  No FMA contraction anywhere:
// every product and sum goes through __dmul_rn / __dadd_rn so results are
// bit-identical to the reference's non-fastmath Numba code.
//
// Wavefront mapping.  A warp owns a strip of 32 consecutive rows; lane i owns
// row 32k+i and at local time tau computes column c = tau - i, so a warp sweeps
// one anti-diagonal of its strip per step.  The three step kinds need
//   (1,1): D/P of (r-1, c-1) = lane i-1's output two steps ago
//   (1,2): D/P of (r-1, c-2) = what this lane received as (1,1) one step ago
//   (2,1): D/P of (r-2, c-1) = what lane i-1 received as (1,1) one step ago
// so two warp shuffles (of D and P) per step feed all three candidates.
// Lane 0 takes rows r-1 and r-2 from the strip above, which another warp
// computed: lanes 30 and 31 of every strip write their outputs into a
// per-warp shared-memory ring, and strips start `lag` steps apart so the
// ring slot is always written at least 16 steps (one barrier) before it is
// read and read at least 16 steps before it is overwritten.  All warps of the
// CTA advance in lock step, with one __syncthreads per 16 steps.
//
// Outputs: D and P on the tile's top edge (last row) and right edge (last
// column), and 2-bit backpointer codes for every cell (code 3 = "no step
// won", the reference's B = -1).
#include "common.cuh"
#include "select.cuh"

#include <math_constants.h>

namespace pfx {

template <int NW, bool FULL, bool STD>
__global__ void __launch_bounds__(NW * 32, 1)
    k_stage1_f64(const double* __restrict__ C, const Geo g, const S1Out out, const int tile0) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tile = tile0 + (int)blockIdx.x;
    const int ti = tile / g.n2, tj = tile % g.n2;
    int64_t r0, c0;
    int32_t R, W;
    tile_rect(g, ti, tj, &r0, &c0, &R, &W);
    const Sched sc = make_sched(R, W, NW);
    const int lag = sc.lag;  // ring length per warp == lag
    double* rD31 = reinterpret_cast<double*>(smem_raw);
    double* rD30 = rD31 + NW * lag;
    int* rP31 = reinterpret_cast<int*>(rD30 + NW * lag);
    int* rP30 = rP31 + NW * lag;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int prevw = (warp + NW - 1) % NW;
    const int Ttot = (sc.nS - 1) * lag + sc.span;
    const unsigned FULLM = 0xffffffffu;

    double* eD = out.edge_D + (int64_t)tile * 2 * g.L;
    int32_t* eP = out.edge_P + (int64_t)tile * 2 * g.L;
    uint32_t* Bt = out.Bw + (int64_t)tile * g.b_words;

    // weight of the last step (the reference's weights[-1]) without a
    // dynamically indexed parameter array
    const double w_last = g.S == 1 ? g.w[0] : (g.S == 2 ? g.w[1] : g.w[2]);

    // per-lane wavefront history
    double h1D = 0.0, h2D = 0.0, x1pD = 0.0;
    int h1P = 0, h2P = 0, x1pP = 0;

    for (int Tb = 0; Tb < Ttot; Tb += kBlk) {
        int k = -1;
        if (Tb >= warp * lag) {
            const int j = (Tb - warp * lag) / (NW * lag);
            const int kk = warp + j * NW;
            if (kk < sc.nS && Tb < kk * lag + sc.span) k = kk;
        }
        if (k >= 0) {
            const int tau0 = Tb - k * lag;
            const int r = 32 * k + lane;
            const bool row_ok = r < R;
            const double* Crow = C + (r0 + (row_ok ? r : 0)) * g.ldc + c0;
            double cv[kBlk];
#pragma unroll
            for (int t = 0; t < kBlk; ++t) {
                const int c = tau0 + t - lane;
                cv[t] = (row_ok && c >= 0 && c < W) ? __ldg(Crow + c) : 0.0;
            }
            // warm L1 with the next block's columns of this row
            {
                const int cn0 = tau0 + kBlk - lane, cn1 = cn0 + kBlk - 1;
                if (row_ok && cn0 >= 0 && cn0 < W)
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(Crow + cn0));
                if (row_ok && cn1 >= 0 && cn1 < W)
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(Crow + cn1));
            }
            int Tmod = tau0 % lag;
            uint32_t bits = 0;
#pragma unroll
            for (int t = 0; t < kBlk; ++t) {
                const int c = tau0 + t - lane;
                double x1D = __shfl_up_sync(FULLM, h2D, 1);
                int x1P = __shfl_up_sync(FULLM, h2P, 1);
                double x3D = __shfl_up_sync(FULLM, x1pD, 1);
                int x3P = __shfl_up_sync(FULLM, x1pP, 1);
                if (lane == 0) {
                    const int rs = prevw * lag + (Tmod == 0 ? lag - 1 : Tmod - 1);
                    x1D = rD31[rs];
                    x1P = rP31[rs];
                    x3D = rD30[rs];
                    x3P = rP30[rs];
                }
                const double x2D = x1pD;
                const int x2P = x1pP;
                double oD = 0.0;
                int oP = 0;
                int code = 0;
                const bool act = row_ok && c >= 0 && c < W;
                if (act) {
                    const double cval = cv[t];
                    if (r == 0 || c == 0) {
                        oD = cval;
                    } else {
                        select_step<STD, false>(g, w_last, r, c, cval, x1D, x1P, x2D, x2P, x3D, x3P, oD,
                                         oP, code);
                    }
                    if (lane >= 30) {
                        const int ws = warp * lag + (Tmod >= lane ? Tmod - lane : Tmod - lane + lag);
                        if (lane == 31) {
                            rD31[ws] = oD;
                            rP31[ws] = oP;
                        } else {
                            rD30[ws] = oD;
                            rP30[ws] = oP;
                        }
                    }
                    if (r == R - 1) {
                        eD[c] = oD;
                        eP[c] = oP;
                    }
                    if (c == W - 1) {
                        eD[g.L + r] = oD;
                        eP[g.L + r] = oP;
                    }
                    if (FULL) {
                        const int64_t f = (int64_t)r * W + c;
                        out.full_D[f] = oD;
                        out.full_P[f] = oP;
                        out.full_B[f] = (int8_t)(code == 3 ? -1 : code);
                    }
                }
                bits |= (uint32_t)code << (2 * t);
                h2D = h1D;
                h2P = h1P;
                h1D = oD;
                h1P = oP;
                x1pD = x1D;
                x1pP = x1P;
                Tmod = (Tmod + 1 == lag) ? 0 : Tmod + 1;
            }
            if (row_ok) Bt[((int64_t)k * sc.nP + (tau0 >> 4)) * 32 + lane] = bits;
        }
        __syncthreads();
    }
}

// Shared memory one CTA of NW warps needs for tiles of at most L x L.
inline size_t stage1_smem_bytes(int32_t L, int nw) {
    const Sched s = make_sched(L, L, nw);
    return (size_t)nw * s.lag * (2 * sizeof(double) + 2 * sizeof(int));
}

size_t stage1_smem_bytes_host(int32_t L, int nw) { return stage1_smem_bytes(L, nw); }

template <int NW, bool FULL, bool STD>
static cudaError_t launch_stage1_t(const double* C, const Geo& g, const S1Out& o, int tile0,
                                   int ntiles, cudaStream_t st) {
    const size_t smem = stage1_smem_bytes(g.L, NW);
    cudaError_t e = cudaFuncSetAttribute(k_stage1_f64<NW, FULL, STD>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_stage1_f64<NW, FULL, STD><<<ntiles, NW * 32, smem, st>>>(C, g, o, tile0);
    count_launches(1);
    return cudaGetLastError();
}

// Warps per CTA: 16 when the tile count leaves SMs free (one CTA per SM,
// 16 strips in flight per tile), else 8 (more CTAs resident per SM).
int stage1_pick_warps(const Geo& g, int num_sms) {
    const int64_t tiles = (int64_t)g.n1 * g.n2;
    if (g.L < 256) return 8;
    return tiles <= (int64_t)num_sms ? 16 : 8;
}

cudaError_t launch_stage1(const double* C, const Geo& g, const S1Out& o, int tile0, int ntiles,
                          int nw, bool full, cudaStream_t st) {
    if (ntiles <= 0) return cudaSuccess;
    const bool std_steps = g.S == 3 && g.kind[0] == 0 && g.kind[1] == 1 && g.kind[2] == 2;
    if (full) {
        if (std_steps)
            return nw == 16 ? launch_stage1_t<16, true, true>(C, g, o, tile0, ntiles, st)
                            : launch_stage1_t<8, true, true>(C, g, o, tile0, ntiles, st);
        return nw == 16 ? launch_stage1_t<16, true, false>(C, g, o, tile0, ntiles, st)
                        : launch_stage1_t<8, true, false>(C, g, o, tile0, ntiles, st);
    }
    if (std_steps)
        return nw == 16 ? launch_stage1_t<16, false, true>(C, g, o, tile0, ntiles, st)
                        : launch_stage1_t<8, false, true>(C, g, o, tile0, ntiles, st);
    return nw == 16 ? launch_stage1_t<16, false, false>(C, g, o, tile0, ntiles, st)
                    : launch_stage1_t<8, false, false>(C, g, o, tile0, ntiles, st);
}

}  // namespace pfx
