// Learned tile proposer: the kernels of a small CNN that reads a 16x
// average-pooled cost matrix and scores which L x L tiles the optimal path
// crosses (inference and training: forward, backward, Adam).  No reference
// counterpart; the full-tile method stays the fallback and the reference answer.
//
// Images are one sample, channels-first [C][H][W], FP32 in training; in
// inference the activations between layers may be stored in bf16 (FP32
// arithmetic).  Convolutions are 3x3, zero padding 1, stride 1 or 2.
//
// Pooled cost: 16-frame block means of the L2-normalised features give the
// block mean of C exactly in real arithmetic (C is bilinear in the two
// frames: mean_{r,c}(1 - a_r . b_c) = 1 - mean(a) . mean(b)), so the pooled
// map costs one small (P1 x d) x (d x P2) product instead of the full C.
#include <cuda_bf16.h>

#include "common.cuh"

namespace pfx {

__device__ __forceinline__ float ld_act(const float* p) { return *p; }
__device__ __forceinline__ float ld_act(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ void st_act(float* p, float v) { *p = v; }
__device__ __forceinline__ void st_act(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }

// F (d x n, FP64, row-major by feature) -> out (d x P, FP32): per block of
// `pool` frames the mean of the L2-normalised frames (last block: the frames
// it has).
constexpr int kPoolMaxD = 32;

// pool <= 16 and d <= 16: 16 lanes per pooled block (two blocks per
// warp), lane l holds frame i0 + l; the normalised frames are summed by a
// fixed butterfly over the 16 lanes.
__global__ void __launch_bounds__(256)
    k_pool_features_warp(const double* __restrict__ F, int d, int64_t n, int pool,
                         float* __restrict__ out, int64_t P) {
    const int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 4;  // pooled block
    const int l = threadIdx.x & 15;
    const int64_t i0 = g * pool, i1 = min(n, i0 + pool);
    const int64_t i = i0 + l;
    const bool on = g < P && l < pool && i < i1;
    double x[16];
    double ss = 0.0;
#pragma unroll
    for (int f = 0; f < 16; ++f) {
        x[f] = (on && f < d) ? F[(int64_t)f * n + i] : 0.0;
        ss += x[f] * x[f];
    }
    const double nr = sqrt(ss);
    const double inv = nr > 0.0 ? 1.0 / nr : 0.0;
    double v = 0.0;
    for (int f = 0; f < d; ++f) {
        double a = x[f] * inv;
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (f == l) v = a;  // lane f keeps feature f's sum
    }
    // lanes f < d of each half write their feature (d <= 16 here)
    if (g < P && l < d) out[(int64_t)l * P + g] = (float)(v / (double)(i1 - i0));
}

__global__ void k_pool_features(const double* __restrict__ F, int d, int64_t n, int pool,
                                float* __restrict__ out, int64_t P) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (p >= P) return;
    const int64_t i0 = p * pool, i1 = min(n, i0 + pool);
    if (d <= kPoolMaxD) {
        // one pass over the block's frames: norm, then the normalised sums
        double acc[kPoolMaxD];
#pragma unroll
        for (int f = 0; f < kPoolMaxD; ++f) acc[f] = 0.0;
        for (int64_t i = i0; i < i1; ++i) {
            double x[kPoolMaxD];
            double ss = 0.0;
#pragma unroll
            for (int f = 0; f < kPoolMaxD; ++f) {
                x[f] = f < d ? F[(int64_t)f * n + i] : 0.0;
                ss += x[f] * x[f];
            }
            const double nr = sqrt(ss);
            const double inv = nr > 0.0 ? 1.0 / nr : 0.0;
#pragma unroll
            for (int f = 0; f < kPoolMaxD; ++f) acc[f] += x[f] * inv;
        }
        for (int f = 0; f < d; ++f) out[(int64_t)f * P + p] = (float)(acc[f] / (double)(i1 - i0));
        return;
    }
    for (int f = 0; f < d; ++f) {
        double s = 0.0;
        for (int64_t i = i0; i < i1; ++i) {
            double ss = 0.0;
            for (int g = 0; g < d; ++g) {
                const double x = F[(int64_t)g * n + i];
                ss += x * x;
            }
            const double nr = sqrt(ss);
            s += nr > 0.0 ? F[(int64_t)f * n + i] / nr : 0.0;
        }
        out[(int64_t)f * P + p] = (float)(s / (double)(i1 - i0));
    }
}

// out[i][j] = 1 - sum_f A[f][i] B[f][j]   (A: d x P1, B: d x P2)
// Four rows per thread: each B value read once serves four outputs.
__global__ void k_pooled_cost(const float* __restrict__ A, const float* __restrict__ B, int d,
                              int64_t P1, int64_t P2, float* __restrict__ out) {
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t i0 = blockIdx.y * 4LL;
    if (j >= P2) return;
    const int nr = P1 - i0 < 4 ? (int)(P1 - i0) : 4;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (int f = 0; f < d; ++f) {
        const float bv = B[(int64_t)f * P2 + j];
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (r < nr) acc[r] = fmaf(A[(int64_t)f * P1 + i0 + r], bv, acc[r]);
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
        if (r < nr) out[(i0 + r) * P2 + j] = 1.f - acc[r];
}

// Double centring and standardisation of a P1 x P2 map, in place:
// x <- (x - rowmean - colmean + mean) / std.  Removes the per-block offsets
// that a whole row or column of the pooled cost shares, leaving the
// diagonal ridge of the alignment.  sc: [P1 + P2 + 2] floats of scratch.
__global__ void k_row_mean(const float* __restrict__ x, int64_t P1, int64_t P2,
                           float* __restrict__ rm) {
    const int64_t i = blockIdx.x;
    float s = 0.f;
    for (int64_t j = threadIdx.x; j < P2; j += blockDim.x) s += x[i * P2 + j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ float ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += ws[w];
        rm[i] = t / (float)P2;
    }
}

// 32 columns per CTA; the 32 warps take every 32nd row, partial sums are
// added in a fixed order (deterministic)
__global__ void __launch_bounds__(1024)
    k_col_mean(const float* __restrict__ x, int64_t P1, int64_t P2, float* __restrict__ cm) {
    __shared__ float part[32][33];
    const int64_t j = blockIdx.x * 32LL + threadIdx.x;
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
    if (j < P2) {
        int64_t i = threadIdx.y;
        for (; i + 96 < P1; i += 128) {
            s0 += x[i * P2 + j];
            s1 += x[(i + 32) * P2 + j];
            s2 += x[(i + 64) * P2 + j];
            s3 += x[(i + 96) * P2 + j];
        }
        for (; i < P1; i += 32) s0 += x[i * P2 + j];
    }
    part[threadIdx.y][threadIdx.x] = (s0 + s1) + (s2 + s3);
    __syncthreads();
    if (threadIdx.y == 0 && j < P2) {
        float t = 0.f;
        for (int r = 0; r < 32; ++r) t += part[r][threadIdx.x];
        cm[j] = t / (float)P1;
    }
}

// sc[P1 + P2] = grand mean (mean of the row means), sc[P1 + P2 + 1] = 0
__global__ void k_grand_mean(float* __restrict__ sc, int64_t P1, int64_t P2) {
    float s = 0.f;
    for (int64_t i = threadIdx.x; i < P1; i += blockDim.x) s += sc[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ float ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += ws[w];
        sc[P1 + P2] = t / (float)P1;
        sc[P1 + P2 + 1] = 0.f;
    }
}

// grid-stride; one atomic per CTA for the sum of squares
__global__ void __launch_bounds__(256)
    k_center(float* __restrict__ x, int64_t P1, int64_t P2, float* __restrict__ sc) {
    const int64_t n = P1 * P2;
    float s = 0.f;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = q / P2, j = q - i * P2;
        const float v = x[q] - sc[i] - sc[P1 + j] + sc[P1 + P2];
        x[q] = v;
        s = fmaf(v, v, s);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ float ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < 8; ++w) t += ws[w];
        atomicAdd(sc + P1 + P2 + 1, t);
    }
}

__global__ void k_scale(float* __restrict__ x, int64_t n, const float* __restrict__ ss) {
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= n) return;
    const float var = *ss / (float)n;
    x[q] = var > 0.f ? x[q] * rsqrtf(var) : 0.f;
}

// --------------------------------------------------------------------------
// 3x3 convolution, forward.  A CTA computes a 16 x 16 tile of output pixels
// for up to 32 output channels; per input channel the input patch and that
// channel's weights ([tap][co], read 4 at a time) are staged in shared
// memory.  y = act(conv(x) + b), act = ReLU or identity.
constexpr int kCvT = 16;  // output tile edge

// PX output pixels per thread (columns tx, tx + 16/PX, ... of a 16 x 16
// tile) and CO/CS of the CTA's CO output channels (channel group tc of CS);
// CIB input channels are staged in shared memory per barrier.  Every weight
// vector read from shared memory serves the PX pixels, every input value the
// thread's CO/CS channels.  Each output sums over (ci, tap) in the same
// order whatever CO, CIB, PX and CS, so every variant gives the same bits.
template <int S, int CO, int CIB, int PX, int CS, typename Tin, typename Tout>
__global__ void __launch_bounds__(kCvT * kCvT / PX * CS)
    k_conv3x3_fwd(const Tin* __restrict__ x, int Cin, int H, int W, const float* __restrict__ w,
                  const float* __restrict__ b, int Cout, int Ho, int Wo, int relu,
                  Tout* __restrict__ y) {
    constexpr int NT = kCvT * kCvT / PX * CS;  // threads
    constexpr int TXN = kCvT / PX;             // threads along x
    constexpr int CT = CO / CS;                // channels per thread
    constexpr int PT = (kCvT - 1) * S + 3;  // input patch edge
    __shared__ float patch[CIB][PT * PT];
    __shared__ __align__(16) float ws[CIB][9 * CO];
    const int ox0 = blockIdx.x * kCvT, oy0 = blockIdx.y * kCvT, co0 = blockIdx.z * CO;
    const int tc = threadIdx.x % CS, tp = threadIdx.x / CS;
    const int tx = tp % TXN, ty = tp / TXN;
    const int oy = oy0 + ty;
    const int nco = min(CO, Cout - co0);
    float acc[PX][CT];
#pragma unroll
    for (int p = 0; p < PX; ++p)
#pragma unroll
        for (int c = 0; c < CT; ++c) acc[p][c] = 0.f;
    const int ix0 = ox0 * S - 1, iy0 = oy0 * S - 1;
    for (int ci0 = 0; ci0 < Cin; ci0 += CIB) {
        const int ncb = min(CIB, Cin - ci0);
        __syncthreads();
        // the patch in batches of 8 loads per thread, each batch issued
        // before its stores (one memory latency per batch, not per element)
        constexpr int NQB = 8;
        for (int q0 = 0; q0 < CIB * PT * PT; q0 += NQB * NT) {
            float v[NQB];
#pragma unroll
            for (int u = 0; u < NQB; ++u) {
                const int q = q0 + threadIdx.x + u * NT;
                const int cb = q / (PT * PT), r = q % (PT * PT);
                const int py = r / PT, px = r % PT;
                const int iy = iy0 + py, ix = ix0 + px;
                v[u] = (q < CIB * PT * PT && cb < ncb && iy >= 0 && iy < H && ix >= 0 &&
                        ix < W)
                           ? ld_act(x + ((int64_t)(ci0 + cb) * H + iy) * W + ix)
                           : 0.f;
            }
#pragma unroll
            for (int u = 0; u < NQB; ++u) {
                const int q = q0 + threadIdx.x + u * NT;
                if (q < CIB * PT * PT) (&patch[0][0])[q] = v[u];
            }
        }
        for (int q = threadIdx.x; q < CIB * 9 * CO; q += NT) {
            const int cb = q / (9 * CO), r = q % (9 * CO);
            const int tap = r / CO, c = r % CO;
            ws[cb][r] = (c < nco && cb < ncb)
                            ? w[((int64_t)(co0 + c) * Cin + ci0 + cb) * 9 + tap]
                            : 0.f;
        }
        __syncthreads();
        for (int cb = 0; cb < ncb; ++cb) {
#pragma unroll
            for (int tap = 0; tap < 9; ++tap) {
                float xv[PX];
#pragma unroll
                for (int p = 0; p < PX; ++p)
                    xv[p] = patch[cb][(ty * S + tap / 3) * PT + (tx + p * TXN) * S + tap % 3];
                if constexpr (CT % 4 == 0) {
                    const float4* w4 =
                        reinterpret_cast<const float4*>(&ws[cb][tap * CO + tc * CT]);
#pragma unroll
                    for (int c4 = 0; c4 < CT / 4; ++c4) {
                        const float4 wv = w4[c4];
#pragma unroll
                        for (int p = 0; p < PX; ++p) {
                            acc[p][4 * c4 + 0] = fmaf(wv.x, xv[p], acc[p][4 * c4 + 0]);
                            acc[p][4 * c4 + 1] = fmaf(wv.y, xv[p], acc[p][4 * c4 + 1]);
                            acc[p][4 * c4 + 2] = fmaf(wv.z, xv[p], acc[p][4 * c4 + 2]);
                            acc[p][4 * c4 + 3] = fmaf(wv.w, xv[p], acc[p][4 * c4 + 3]);
                        }
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < CT; ++c) {
                        const float wv = ws[cb][tap * CO + tc * CT + c];
#pragma unroll
                        for (int p = 0; p < PX; ++p) acc[p][c] = fmaf(wv, xv[p], acc[p][c]);
                    }
                }
            }
        }
    }
    if (oy >= Ho) return;
#pragma unroll
    for (int p = 0; p < PX; ++p) {
        const int ox = ox0 + tx + p * TXN;
        if (ox >= Wo) continue;
#pragma unroll
        for (int c = 0; c < CT; ++c) {
            const int cc = tc * CT + c;
            if (cc < nco) {
                float v = acc[p][c] + b[co0 + cc];
                if (relu) v = fmaxf(v, 0.f);
                st_act(y + ((int64_t)(co0 + cc) * Ho + oy) * Wo + ox, v);
            }
        }
    }
}

// The network's input from the pooled features, without the map.  The pooled
// cost 1 - a_i . b_j is bilinear, so its double centring is
// -(a_i - abar) . (b_j - bbar), and the mean square of that map is
// sum_{f,g} GA[f][g] GB[f][g] / (P1 P2) with GA, GB the Gram matrices of the
// centred features.  Two kernels (d <= 16, FP64 sums in a fixed order):
// k_feat_moments gives each chunk of kCfChunk frames of A (d x P1) or B
// (d x P2) its feature sums and its raw Gram matrix (upper triangle);
// k_center_features adds the chunks in order, centres the Gram matrices
// (G - P m m^T), and centres A and B in place, scaling A by -1/std so that
// A^T B is the centred, standardised map.
constexpr int kCfChunk = 64;
constexpr int kCfMom = 16 + 136;  // sums, then the upper-triangle Gram entries

__host__ __device__ inline int feat_chunks(int64_t P) { return (int)((P + kCfChunk - 1) / kCfChunk); }

__device__ __forceinline__ void tri_index(int p, int d, int* f, int* g) {
    int r = p, ff = 0;
    while (r >= d - ff) { r -= d - ff; ++ff; }
    *f = ff;
    *g = ff + r;
}

constexpr int kCfMomThreads = 160;  // >= 16 + 136: one thread per moment

__global__ void __launch_bounds__(kCfMomThreads)
    k_feat_moments(const float* __restrict__ A, const float* __restrict__ B, int d, int64_t P1,
                   int64_t P2, double* __restrict__ mom) {
    __shared__ float X[16][kCfChunk];
    const int ncA = feat_chunks(P1);
    const bool isB = (int)blockIdx.x >= ncA;
    const int c = isB ? (int)blockIdx.x - ncA : (int)blockIdx.x;
    const float* src = isB ? B : A;
    const int64_t P = isB ? P2 : P1;
    const int64_t i0 = (int64_t)c * kCfChunk;
    const int n = P - i0 < kCfChunk ? (int)(P - i0) : kCfChunk;
    for (int q = threadIdx.x; q < d * kCfChunk; q += kCfMomThreads) {
        const int f = q / kCfChunk, i = q % kCfChunk;
        X[f][i] = i < n ? src[(int64_t)f * P + i0 + i] : 0.f;
    }
    __syncthreads();
    const int npair = d * (d + 1) / 2;
    double* out = mom + (int64_t)blockIdx.x * kCfMom;
    const int t = threadIdx.x;
    if (t < d) {
        double acc = 0.0;
        for (int i = 0; i < n; ++i) acc += (double)X[t][i];
        out[t] = acc;
    } else if (t >= 16 && t < 16 + npair) {
        int f, g;
        tri_index(t - 16, d, &f, &g);
        double acc = 0.0;
        for (int i = 0; i < n; ++i) acc += (double)X[f][i] * (double)X[g][i];
        out[t] = acc;
    }
}

constexpr int kCfThreads = 256;
constexpr int kCfPer = 2048;  // frames x features centred per CTA

// Every CTA derives the means and the scale from the chunks' moments (the
// same sums in the same order, so every CTA gets the same values), then
// centres its slice of A and B: slice j covers kCfPer consecutive entries of
// the d x P1 array A followed by the d x P2 array B.
__global__ void __launch_bounds__(kCfThreads)
    k_center_features(float* __restrict__ A, float* __restrict__ B, int d, int64_t P1,
                      int64_t P2, const double* __restrict__ mom) {
    __shared__ double mean[2][16];
    __shared__ double gram[2][136];
    __shared__ float scale;
    const int t = threadIdx.x;
    const int npair = d * (d + 1) / 2;
    const int ncA = feat_chunks(P1), ncB = feat_chunks(P2);
    for (int q = t; q < 2 * kCfMom; q += kCfThreads) {
        const int s = q / kCfMom, k = q % kCfMom;
        const int c0 = s ? ncA : 0, nc = s ? ncB : ncA;
        const bool used = k < d || (k >= 16 && k < 16 + npair);
        double acc = 0.0;
        if (used)
            for (int c = 0; c < nc; ++c) acc += mom[(int64_t)(c0 + c) * kCfMom + k];
        if (k < d) mean[s][k] = acc / (double)(s ? P2 : P1);
        if (k >= 16 && k < 16 + npair) gram[s][k - 16] = acc;
    }
    __syncthreads();
    if (t < 2 * npair) {  // centred Gram: G - P m_f m_g
        const int s = t / npair, p = t % npair;
        int f, g;
        tri_index(p, d, &f, &g);
        gram[s][p] -= (double)(s ? P2 : P1) * mean[s][f] * mean[s][g];
    }
    __syncthreads();
    if (t == 0) {
        double v = 0.0;
        for (int p = 0; p < npair; ++p) {
            int f, g;
            tri_index(p, d, &f, &g);
            v += (f == g ? 1.0 : 2.0) * gram[0][p] * gram[1][p];
        }
        v /= (double)P1 * (double)P2;
        scale = v > 0.0 ? (float)(-1.0 / sqrt(v)) : 0.f;
    }
    __syncthreads();
    const int64_t nA = (int64_t)d * P1, n = nA + (int64_t)d * P2;
    const int64_t q0 = (int64_t)blockIdx.x * kCfPer;
    const int64_t q1 = q0 + kCfPer < n ? q0 + kCfPer : n;
    for (int64_t q = q0 + t; q < q1; q += kCfThreads) {
        if (q < nA) {
            const int f = (int)(q / P1);
            A[q] = (float)((double)A[q] - mean[0][f]) * scale;
        } else {
            const int f = (int)((q - nA) / P2);
            B[q - nA] = (float)((double)B[q - nA] - mean[1][f]);
        }
    }
}

// The first layer (Cin = 1, CO output channels) on the map x = A^T B: each
// thread computes the 9 inputs of its own output pixel from the CTA's rows of
// A and columns of B staged in shared memory (zero outside the map, as the
// convolution's padding), then the 3 x 3 x CO products in the order of
// k_conv3x3_fwd.
template <int S, int CO, typename Tout>
__global__ void __launch_bounds__(kCvT * kCvT)
    k_conv3x3_fwd_feat(const float* __restrict__ A, const float* __restrict__ B, int d, int H,
                       int W, const float* __restrict__ w, const float* __restrict__ b, int Cout,
                       int Ho, int Wo, int relu, Tout* __restrict__ y) {
    constexpr int NT = kCvT * kCvT;
    constexpr int PT = (kCvT - 1) * S + 3;  // input patch edge
    __shared__ float sA[16][PT], sB[16][PT];
    __shared__ __align__(16) float ws[9 * CO];
    const int ox0 = blockIdx.x * kCvT, oy0 = blockIdx.y * kCvT, co0 = blockIdx.z * CO;
    const int tx = threadIdx.x % kCvT, ty = threadIdx.x / kCvT;
    const int ox = ox0 + tx, oy = oy0 + ty;
    const int nco = min(CO, Cout - co0);
    const int ix0 = ox0 * S - 1, iy0 = oy0 * S - 1;
    for (int q = threadIdx.x; q < d * PT; q += NT) {
        const int f = q / PT, r = q % PT;
        const int iy = iy0 + r, ix = ix0 + r;
        sA[f][r] = (iy >= 0 && iy < H) ? A[(int64_t)f * H + iy] : 0.f;
        sB[f][r] = (ix >= 0 && ix < W) ? B[(int64_t)f * W + ix] : 0.f;
    }
    for (int q = threadIdx.x; q < 9 * CO; q += NT) {
        const int tap = q / CO, c = q % CO;
        ws[q] = c < nco ? w[(int64_t)(co0 + c) * 9 + tap] : 0.f;
    }
    __syncthreads();
    // inputs of taps (ky, kx): rows ty*S + ky, columns tx*S + kx of the patch
    float xin[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) xin[k] = 0.f;
    for (int f = 0; f < d; ++f) {
        float ra[3], cb[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            ra[k] = sA[f][ty * S + k];
            cb[k] = sB[f][tx * S + k];
        }
#pragma unroll
        for (int ky = 0; ky < 3; ++ky)
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) xin[ky * 3 + kx] = fmaf(ra[ky], cb[kx], xin[ky * 3 + kx]);
    }
    float acc[CO];
#pragma unroll
    for (int c = 0; c < CO; ++c) acc[c] = 0.f;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
        const float xv = xin[tap];
        const float4* w4 = reinterpret_cast<const float4*>(&ws[tap * CO]);
#pragma unroll
        for (int c4 = 0; c4 < CO / 4; ++c4) {
            const float4 wv = w4[c4];
            acc[4 * c4 + 0] = fmaf(wv.x, xv, acc[4 * c4 + 0]);
            acc[4 * c4 + 1] = fmaf(wv.y, xv, acc[4 * c4 + 1]);
            acc[4 * c4 + 2] = fmaf(wv.z, xv, acc[4 * c4 + 2]);
            acc[4 * c4 + 3] = fmaf(wv.w, xv, acc[4 * c4 + 3]);
        }
    }
    if (ox >= Wo || oy >= Ho) return;
#pragma unroll
    for (int c = 0; c < CO; ++c) {
        if (c < nco) {
            float v = acc[c] + b[co0 + c];
            if (relu) v = fmaxf(v, 0.f);
            st_act(y + ((int64_t)(co0 + c) * Ho + oy) * Wo + ox, v);
        }
    }
}

// Gradient at the conv output before the activation: dz = dy * (y > 0) for
// ReLU layers, dy otherwise.
__device__ __forceinline__ float dz_at(const float* dy, const float* y, int relu, int64_t i) {
    return relu ? (y[i] > 0.f ? dy[i] : 0.f) : dy[i];
}

// Backward, data: dx[ci][iy][ix] = sum_{co, tap} w[co][ci][tap] dz[co][oy][ox]
// over the outputs whose window covers (iy, ix).  One thread per input pixel.
template <int S>
__global__ void k_conv3x3_bwd_data(const float* __restrict__ w, int Cin, int H, int W, int Cout,
                                   int Ho, int Wo, const float* __restrict__ y,
                                   const float* __restrict__ dy, int relu, float* __restrict__ dx) {
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= (int64_t)Cin * H * W) return;
    const int ix = (int)(q % W), iy = (int)((q / W) % H), ci = (int)(q / ((int64_t)W * H));
    float acc = 0.f;
    for (int ky = 0; ky < 3; ++ky) {
        const int ty = iy + 1 - ky;  // = oy * S
        if (ty < 0 || ty % S) continue;
        const int oy = ty / S;
        if (oy >= Ho) continue;
        for (int kx = 0; kx < 3; ++kx) {
            const int tx = ix + 1 - kx;
            if (tx < 0 || tx % S) continue;
            const int ox = tx / S;
            if (ox >= Wo) continue;
            for (int co = 0; co < Cout; ++co) {
                const int64_t oi = ((int64_t)co * Ho + oy) * Wo + ox;
                acc = fmaf(w[((int64_t)co * Cin + ci) * 9 + ky * 3 + kx], dz_at(dy, y, relu, oi),
                           acc);
            }
        }
    }
    dx[q] = acc;
}

// Backward, weights and bias: dw[co][ci][tap] += sum_pixels dz * x, db[co] +=
// sum dz.  A CTA takes a 16 x 16 output tile and a chunk of 8 input
// channels; per-CTA partial sums go to global memory with atomics.
constexpr int kWgCi = 8;

template <int S>
__global__ void __launch_bounds__(256)
    k_conv3x3_bwd_weight(const float* __restrict__ x, int Cin, int H, int W, int Cout, int Ho,
                         int Wo, const float* __restrict__ y, const float* __restrict__ dy,
                         int relu, float* __restrict__ dw, float* __restrict__ db) {
    constexpr int PT = (kCvT - 1) * S + 3;
    extern __shared__ float sm[];
    float* dz = sm;                          // [Cout][256]
    float* patch = sm + Cout * kCvT * kCvT;  // [kWgCi][PT*PT]
    const int ox0 = blockIdx.x * kCvT, oy0 = blockIdx.y * kCvT, ci0 = blockIdx.z * kWgCi;
    const int nci = min(kWgCi, Cin - ci0);
    for (int q = threadIdx.x; q < Cout * kCvT * kCvT; q += 256) {
        const int co = q / (kCvT * kCvT), p = q % (kCvT * kCvT);
        const int ox = ox0 + p % kCvT, oy = oy0 + p / kCvT;
        dz[q] = (ox < Wo && oy < Ho) ? dz_at(dy, y, relu, ((int64_t)co * Ho + oy) * Wo + ox) : 0.f;
    }
    const int ix0 = ox0 * S - 1, iy0 = oy0 * S - 1;
    for (int q = threadIdx.x; q < nci * PT * PT; q += 256) {
        const int c = q / (PT * PT), r = q % (PT * PT);
        const int iy = iy0 + r / PT, ix = ix0 + r % PT;
        patch[q] = (iy >= 0 && iy < H && ix >= 0 && ix < W)
                       ? x[((int64_t)(ci0 + c) * H + iy) * W + ix]
                       : 0.f;
    }
    __syncthreads();
    const int ncomb = Cout * nci * 9;
    for (int cmb = threadIdx.x; cmb < ncomb; cmb += 256) {
        const int tap = cmb % 9, c = (cmb / 9) % nci, co = cmb / (9 * nci);
        const int ky = tap / 3, kx = tap % 3;
        const float* dzc = dz + co * kCvT * kCvT;
        const float* pc = patch + c * PT * PT;
        float acc = 0.f;
        for (int p = 0; p < kCvT * kCvT; ++p) {
            const int py = p / kCvT, px = p % kCvT;
            acc = fmaf(dzc[p], pc[(py * S + ky) * PT + px * S + kx], acc);
        }
        atomicAdd(dw + ((int64_t)co * Cin + ci0 + c) * 9 + tap, acc);
    }
    if (blockIdx.z == 0) {
        for (int co = threadIdx.x; co < Cout; co += 256) {
            float acc = 0.f;
            for (int p = 0; p < kCvT * kCvT; ++p) acc += dz[co * kCvT * kCvT + p];
            atomicAdd(db + co, acc);
        }
    }
}

// Tile scores: the max logit over each tile's region of the logit map
// (`fpp` frames per logit pixel); argmax = flat pixel index (ties: lowest).
__global__ void __launch_bounds__(256)
    k_tile_max(const float* __restrict__ logits, int H, int W, int n1, int n2, int64_t hop,
               int64_t L, int64_t N, int64_t M, int fpp, float* __restrict__ score,
               int32_t* __restrict__ argmax) {
    const int t = blockIdx.x;
    if (t >= n1 * n2) return;
    const int i = t / n2, j = t % n2;
    const int64_t r0 = i * hop, c0 = j * hop;
    const int64_t r1 = r0 + L < N ? r0 + L : N, c1 = c0 + L < M ? c0 + L : M;
    const int64_t ya = r0 / fpp, yb = (r1 + fpp - 1) / fpp;
    const int64_t xa = c0 / fpp, xb = (c1 + fpp - 1) / fpp;
    const int y0 = (int)(ya < H - 1 ? ya : H - 1), y1 = (int)(yb < H ? yb : H);
    const int x0 = (int)(xa < W - 1 ? xa : W - 1), x1 = (int)(xb < W ? xb : W);
    const int h = max(y1 - y0, 1), wd = max(x1 - x0, 1);
    float best = -INFINITY;
    int bi = y0 * W + x0;
    for (int q = threadIdx.x; q < h * wd; q += blockDim.x) {
        const int idx = (y0 + q / wd) * W + x0 + q % wd;
        const float v = logits[idx];
        if (v > best || (v == best && idx < bi)) {
            best = v;
            bi = idx;
        }
    }
    __shared__ float sv[256];
    __shared__ int si[256];
    sv[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            const float v = sv[threadIdx.x + s];
            const int ix = si[threadIdx.x + s];
            if (v > sv[threadIdx.x] || (v == sv[threadIdx.x] && ix < si[threadIdx.x])) {
                sv[threadIdx.x] = v;
                si[threadIdx.x] = ix;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        score[t] = sv[0];
        argmax[t] = si[0];
    }
}

// Weighted binary cross-entropy with logits: loss += sum_t w_t * l_t / n,
// dscore_t = w_t * (sigmoid(s_t) - y_t) / n, w_t = pos_weight for positives.
__global__ void k_tile_bce(const float* __restrict__ s, const uint8_t* __restrict__ label, int n,
                           float pos_weight, float* __restrict__ loss, float* __restrict__ ds) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (t < n) {
        const float x = s[t], yv = label[t] ? 1.f : 0.f;
        const float wt = label[t] ? pos_weight : 1.f;
        // log(1 + exp(-|x|)) + max(x, 0) - x*y: the stable form
        l = wt * (log1pf(expf(-fabsf(x))) + fmaxf(x, 0.f) - x * yv) / n;
        const float sg = 1.f / (1.f + expf(-x));
        ds[t] = wt * (sg - yv) / n;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

__global__ void k_tile_max_bwd(const float* __restrict__ ds, const int32_t* __restrict__ argmax,
                               int n, float* __restrict__ dlogits) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) atomicAdd(dlogits + argmax[t], ds[t]);
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// mask = dilate(score > threshold) by `dil` tiles (Chebyshev distance, or
// Manhattan distance when `manhattan`).
__global__ void k_tile_mask(const float* __restrict__ score, int n1, int n2, float thr, int dil,
                            int manhattan, uint8_t* __restrict__ mask) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n1 * n2) return;
    const int i = t / n2, j = t % n2;
    uint8_t on = 0;
    for (int a = max(0, i - dil); a <= min(n1 - 1, i + dil) && !on; ++a)
        for (int b = max(0, j - dil); b <= min(n2 - 1, j + dil); ++b)
            if ((!manhattan || abs(a - i) + abs(b - j) <= dil) && score[a * n2 + b] > thr) {
                on = 1;
                break;
            }
    mask[t] = on;
}

// ---------------------------------------------------------------- launchers
static unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

cudaError_t cnn_pool_features(const double* F, int d, int64_t n, int pool, float* out,
                              cudaStream_t st) {
    const int64_t P = (n + pool - 1) / pool;
    if (P <= 0) return cudaSuccess;
    if (pool <= 16 && d <= 16)
        k_pool_features_warp<<<blocks_for(P * 16, 256), 256, 0, st>>>(F, d, n, pool, out, P);
    else
        k_pool_features<<<blocks_for(P, 128), 128, 0, st>>>(F, d, n, pool, out, P);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t cnn_pooled_cost(const float* A, const float* B, int d, int64_t P1, int64_t P2,
                            float* out, cudaStream_t st) {
    if (P1 <= 0 || P2 <= 0) return cudaSuccess;
    k_pooled_cost<<<dim3(blocks_for(P2, 256), (unsigned)blocks_for(P1, 4)), 256, 0, st>>>(
        A, B, d, P1, P2, out);
    count_launches(1);
    return cudaGetLastError();
}

template <int S, int CO, int CIB, int PX, int CS, typename Tin, typename Tout>
static cudaError_t conv_fwd_launch(const void* x, int Cin, int H, int W, const float* w,
                                   const float* b, int Cout, int relu, void* y, cudaStream_t st) {
    const int Ho = (H - 1) / S + 1, Wo = (W - 1) / S + 1;
    const dim3 grid(blocks_for(Wo, kCvT), blocks_for(Ho, kCvT), blocks_for(Cout, CO));
    k_conv3x3_fwd<S, CO, CIB, PX, CS, Tin, Tout><<<grid, kCvT * kCvT / PX * CS, 0, st>>>(
        static_cast<const Tin*>(x), Cin, H, W, w, b, Cout, Ho, Wo, relu, static_cast<Tout*>(y));
    count_launches(1);
    return cudaGetLastError();
}

// 32 output channels per CTA, or one when the layer has fewer than 8; the
// patch of 4 input channels (stride 1, 2) or one (stride 4) per barrier
template <int S, typename Tin, typename Tout>
static cudaError_t conv_fwd_t(const void* x, int Cin, int H, int W, const float* w, const float* b,
                              int Cout, int relu, void* y, cudaStream_t st) {
    constexpr int CIB = S == 4 ? 1 : 4;
    if (Cout < 8)
        return conv_fwd_launch<S, 1, 2 * CIB, 1, 1, Tin, Tout>(x, Cin, H, W, w, b, Cout, relu, y,
                                                               st);
    if (Cin >= 8)  // two pixels x 16 channels per thread: 6 shared loads per 32 FMAs
        return conv_fwd_launch<S, 32, CIB, 2, 2, Tin, Tout>(x, Cin, H, W, w, b, Cout, relu, y,
                                                            st);
    return conv_fwd_launch<S, 32, CIB, 1, 1, Tin, Tout>(x, Cin, H, W, w, b, Cout, relu, y, st);
}

// --------------------------------------------------------------------------
// The inference network's 32 -> 32-channel 3x3 convolution with bf16
// activations (in and out) on the tensor cores: an implicit GEMM, output
// pixels x (tap, input channel) x output channels, with
// mma.sync.m16n8k16 (bf16 operands, FP32 accumulation).  The layer is bound
// by moving its activations, not by its 9216 MACs per pixel, so warp-level
// MMAs out of registers suffice.  Each weight is split into bf16 high and
// low parts (two MMAs), so the products keep the FP32 weight to about 2^-17;
// the sum order differs from k_conv3x3_fwd (results agree to FP32 rounding
// of the sums, not bit for bit).
//
// A CTA computes 8 output rows x 16 columns for all 32 output channels; warp
// w takes rows 2w, 2w + 1 (one m16 tile of 16 pixels each).  Shared memory:
// the input patch as [row][column][channel] with a 36-channel pixel stride
// and the weights as [tap][co][ci] (hi and lo) with a 40-channel row stride,
// so that every fragment load of a warp touches 32 distinct banks.
constexpr int kMmaRows = 8, kMmaCols = 16, kMmaPix = 36, kMmaWRow = 40;

template <int S>
struct MmaConvGeo {
    static constexpr int PR = (kMmaRows - 1) * S + 3;  // patch rows
    static constexpr int PC = (kMmaCols - 1) * S + 3;  // patch columns
    static constexpr int patch_elems = PR * PC * kMmaPix;
    static constexpr int w_elems = 9 * 32 * kMmaWRow;
    static constexpr size_t smem = (size_t)(patch_elems + 2 * w_elems) * 2;
};

__device__ __forceinline__ void mma_bf16_16816(float (&c)[4], uint32_t a0, uint32_t a1,
                                               uint32_t a2, uint32_t a3, uint32_t b0,
                                               uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, "
        "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

template <int S>
__global__ void __launch_bounds__(128)
    k_conv3x3_mma32(const __nv_bfloat16* __restrict__ x, int H, int W,
                    const float* __restrict__ w, const float* __restrict__ b, int Ho, int Wo,
                    int relu, __nv_bfloat16* __restrict__ y) {
    using G = MmaConvGeo<S>;
    extern __shared__ __align__(16) unsigned char cv_smem[];
    __nv_bfloat16* patch = reinterpret_cast<__nv_bfloat16*>(cv_smem);
    __nv_bfloat16* whi = patch + G::patch_elems;
    __nv_bfloat16* wlo = whi + G::w_elems;
    const int ox0 = blockIdx.x * kMmaCols, oy0 = blockIdx.y * kMmaRows;
    const int iy0 = oy0 * S - 1, ix0 = ox0 * S - 1;
    // the patch: a thread takes pixels, each as 16 channel pairs (loads of
    // one channel plane coalesce across the warp's consecutive columns)
    for (int q = threadIdx.x; q < G::PR * G::PC; q += 128) {
        const int r = q / G::PC, c = q - r * G::PC;
        const int iy = iy0 + r, ix = ix0 + c;
        const bool in = iy >= 0 && iy < H && ix >= 0 && ix < W;
        const __nv_bfloat16* src = x + (int64_t)(in ? iy : 0) * W + (in ? ix : 0);
        uint32_t* dst = reinterpret_cast<uint32_t*>(patch + q * kMmaPix);
        unsigned short v[32];
#pragma unroll
        for (int ci = 0; ci < 32; ++ci)
            v[ci] = in ? __bfloat16_as_ushort(src[(int64_t)ci * H * W]) : (unsigned short)0;
#pragma unroll
        for (int k = 0; k < 16; ++k) dst[k] = (uint32_t)v[2 * k] | ((uint32_t)v[2 * k + 1] << 16);
    }
    // the weights, [tap][co][ci], each FP32 weight as bf16 hi + lo
    for (int q = threadIdx.x; q < 9 * 32 * 32; q += 128) {
        const int tap = q / 1024, co = (q >> 5) & 31, ci = q & 31;
        const float v = w[(co * 32 + ci) * 9 + tap];
        const __nv_bfloat16 hi = __float2bfloat16_rn(v);
        const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
        whi[(tap * 32 + co) * kMmaWRow + ci] = hi;
        wlo[(tap * 32 + co) * kMmaWRow + ci] = lo;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[mt][j][e] = 0.f;
    const uint32_t* P32 = reinterpret_cast<const uint32_t*>(patch);
    const uint32_t* H32 = reinterpret_cast<const uint32_t*>(whi);
    const uint32_t* L32 = reinterpret_cast<const uint32_t*>(wlo);
#pragma unroll 1
    for (int tap = 0; tap < 9; ++tap) {
        const int ky = tap / 3, kx = tap - 3 * ky;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int ci0 = 16 * half;
            uint32_t bh[4][2], bl[4][2];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int wi = ((tap * 32 + 8 * j + g) * kMmaWRow + ci0 + 2 * t) >> 1;
                bh[j][0] = H32[wi];
                bh[j][1] = H32[wi + 4];
                bl[j][0] = L32[wi];
                bl[j][1] = L32[wi + 4];
            }
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const int pr = (2 * warp + mt) * S + ky;
                const int p0 = ((pr * G::PC + g * S + kx) * kMmaPix + ci0 + 2 * t) >> 1;
                const int p1 = p0 + ((8 * S * kMmaPix) >> 1);  // pixel g + 8
                const uint32_t a0 = P32[p0], a1 = P32[p1], a2 = P32[p0 + 4], a3 = P32[p1 + 4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    mma_bf16_16816(acc[mt][j], a0, a1, a2, a3, bh[j][0], bh[j][1]);
                    mma_bf16_16816(acc[mt][j], a0, a1, a2, a3, bl[j][0], bl[j][1]);
                }
            }
        }
    }
    // y = act(acc + b): c0, c1 at pixel g, channels 8j + 2t (+1); c2, c3 at pixel g + 8
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const int oy = oy0 + 2 * warp + mt;
        if (oy >= Ho) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int co = 8 * j + 2 * t + (e & 1);
                const int ox = ox0 + g + (e >> 1) * 8;
                if (ox >= Wo) continue;
                float v = acc[mt][j][e] + b[co];
                if (relu) v = fmaxf(v, 0.f);
                y[((int64_t)co * Ho + oy) * Wo + ox] = __float2bfloat16_rn(v);
            }
    }
}

template <int S>
static cudaError_t conv_mma32_launch(const __nv_bfloat16* x, int H, int W, const float* w,
                                     const float* b, int relu, __nv_bfloat16* y,
                                     cudaStream_t st) {
    const int Ho = (H - 1) / S + 1, Wo = (W - 1) / S + 1;
    const size_t smem = MmaConvGeo<S>::smem;
    cudaError_t e = cudaFuncSetAttribute(k_conv3x3_mma32<S>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const dim3 grid(blocks_for(Wo, kMmaCols), blocks_for(Ho, kMmaRows));
    k_conv3x3_mma32<S><<<grid, 128, smem, st>>>(x, H, W, w, b, Ho, Wo, relu, y);
    count_launches(1);
    return cudaGetLastError();
}

// in_bf16 / out_bf16: activation storage types (FP32 otherwise).
cudaError_t cnn_conv_forward(const void* x, int in_bf16, int Cin, int H, int W, const float* w,
                             const float* b, int Cout, int stride, int relu, void* y,
                             int out_bf16, cudaStream_t st) {
    using bf = __nv_bfloat16;
    // the inference network's 32 -> 32 layer (bf16 activations): tensor cores
    if (in_bf16 && out_bf16 && Cin == 32 && Cout == 32 && stride == 2)
        return conv_mma32_launch<2>(static_cast<const bf*>(x), H, W, w, b, relu,
                                    static_cast<bf*>(y), st);
#define PFX_CONV(S)                                                                             \
    if (in_bf16 && out_bf16) return conv_fwd_t<S, bf, bf>(x, Cin, H, W, w, b, Cout, relu, y, st); \
    if (in_bf16) return conv_fwd_t<S, bf, float>(x, Cin, H, W, w, b, Cout, relu, y, st);          \
    if (out_bf16) return conv_fwd_t<S, float, bf>(x, Cin, H, W, w, b, Cout, relu, y, st);         \
    return conv_fwd_t<S, float, float>(x, Cin, H, W, w, b, Cout, relu, y, st);
    if (stride == 1) {
        PFX_CONV(1)
    }
    if (stride == 4) {
        PFX_CONV(4)
    }
    PFX_CONV(2)
#undef PFX_CONV
}

template <int S>
static cudaError_t conv_bwd_t(const float* x, int Cin, int H, int W, const float* w, int Cout,
                              const float* y, int relu, const float* dy, float* dx, float* dw,
                              float* db, cudaStream_t st) {
    const int Ho = (H - 1) / S + 1, Wo = (W - 1) / S + 1;
    if (dx) {
        const int64_t n = (int64_t)Cin * H * W;
        k_conv3x3_bwd_data<S><<<blocks_for(n, 256), 256, 0, st>>>(w, Cin, H, W, Cout, Ho, Wo, y,
                                                                 dy, relu, dx);
        count_launches(1);
    }
    const dim3 grid(blocks_for(Wo, kCvT), blocks_for(Ho, kCvT), blocks_for(Cin, kWgCi));
    constexpr int PT = (kCvT - 1) * S + 3;
    const size_t smem = ((size_t)Cout * kCvT * kCvT + (size_t)kWgCi * PT * PT) * sizeof(float);
    cudaError_t e = cudaFuncSetAttribute(k_conv3x3_bwd_weight<S>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_conv3x3_bwd_weight<S><<<grid, 256, smem, st>>>(x, Cin, H, W, Cout, Ho, Wo, y, dy, relu, dw,
                                                     db);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t cnn_conv_backward(const float* x, int Cin, int H, int W, const float* w, int Cout,
                              int stride, const float* y, int relu, const float* dy, float* dx,
                              float* dw, float* db, cudaStream_t st) {
    if (stride == 1) return conv_bwd_t<1>(x, Cin, H, W, w, Cout, y, relu, dy, dx, dw, db, st);
    if (stride == 4) return conv_bwd_t<4>(x, Cin, H, W, w, Cout, y, relu, dy, dx, dw, db, st);
    return conv_bwd_t<2>(x, Cin, H, W, w, Cout, y, relu, dy, dx, dw, db, st);
}

}  // namespace pfx

// ------------------------------------------------------------------ C ABI
using namespace pfx;

#define PFX_CNN_RET(expr)                                                                  \
    do {                                                                                   \
        const cudaError_t e_ = (expr);                                                     \
        if (e_ != cudaSuccess) return report_status(PFX_ERR_CUDA, cudaGetErrorString(e_)); \
        return PFX_OK;                                                                     \
    } while (0)

#define PFX_CNN_LAUNCHED()                                                                 \
    do {                                                                                   \
        count_launches(1);                                                                 \
        PFX_CNN_RET(cudaGetLastError());                                                   \
    } while (0)

extern "C" int pfx_pool_features(const double* F, int32_t d, int64_t n, int32_t pool, float* out,
                                 void* stream) {
    if (!F || !out || d < 1 || n < 1 || pool < 1)
        return report_status(PFX_ERR_ARG, "pfx_pool_features: bad argument");
    PFX_CNN_RET(cnn_pool_features(F, d, n, pool, out, (cudaStream_t)stream));
}

extern "C" int pfx_pooled_cost(const float* A, const float* B, int32_t d, int64_t P1, int64_t P2,
                               float* out, void* stream) {
    if (!A || !B || !out || d < 1 || P1 < 1 || P2 < 1 || P1 > 65535)
        return report_status(PFX_ERR_ARG, "pfx_pooled_cost: bad argument (P1 <= 65535)");
    PFX_CNN_RET(cnn_pooled_cost(A, B, d, P1, P2, out, (cudaStream_t)stream));
}

extern "C" int pfx_pooled_center(float* x, int64_t P1, int64_t P2, float* scratch,
                                 void* stream) {
    if (!x || !scratch || P1 < 1 || P2 < 1)
        return report_status(PFX_ERR_ARG, "pfx_pooled_center: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t n = P1 * P2;
    k_row_mean<<<(unsigned)P1, 256, 0, st>>>(x, P1, P2, scratch);
    k_col_mean<<<blocks_for(P2, 32), dim3(32, 32), 0, st>>>(x, P1, P2, scratch + P1);
    k_grand_mean<<<1, 1024, 0, st>>>(scratch, P1, P2);
    const int64_t cb = blocks_for(n, 256) < 1184 ? blocks_for(n, 256) : 1184;
    k_center<<<(unsigned)cb, 256, 0, st>>>(x, P1, P2, scratch);
    k_scale<<<blocks_for(n, 256), 256, 0, st>>>(x, n, scratch + P1 + P2 + 1);
    count_launches(5);
    PFX_CNN_RET(cudaGetLastError());
}

extern "C" int64_t pfx_pooled_center_scratch(int64_t P1, int64_t P2) {
    if (P1 < 1 || P2 < 1) return 0;
    return (int64_t)(feat_chunks(P1) + feat_chunks(P2)) * kCfMom * (int64_t)sizeof(double);
}

extern "C" int pfx_pooled_center_features(float* A, float* B, int32_t d, int64_t P1,
                                          int64_t P2, void* scratch, void* stream) {
    if (!A || !B || !scratch || d < 1 || d > 16 || P1 < 1 || P2 < 1)
        return report_status(PFX_ERR_ARG, "pfx_pooled_center_features: bad argument (d <= 16)");
    cudaStream_t st = (cudaStream_t)stream;
    double* mom = static_cast<double*>(scratch);
    k_feat_moments<<<(unsigned)(feat_chunks(P1) + feat_chunks(P2)), kCfMomThreads, 0, st>>>(
        A, B, d, P1, P2, mom);
    const int64_t n = (int64_t)d * (P1 + P2);
    k_center_features<<<(unsigned)((n + kCfPer - 1) / kCfPer), kCfThreads, 0, st>>>(A, B, d, P1,
                                                                                   P2, mom);
    count_launches(2);
    PFX_CNN_RET(cudaGetLastError());
}

extern "C" int pfx_conv3x3_forward_features(const float* A, const float* B, int32_t d, int32_t H,
                                            int32_t W, const float* w, const float* b,
                                            int32_t Cout, int32_t stride, int32_t relu, void* y,
                                            int32_t y_bf16, void* stream) {
    if (!A || !B || !w || !b || !y || d < 1 || d > 16 || Cout != 32 || H < 1 || W < 1 ||
        (stride != 1 && stride != 2 && stride != 4) || (int64_t)H * W > (1LL << 31) / 64)
        return report_status(PFX_ERR_ARG,
                             "pfx_conv3x3_forward_features: bad argument (d <= 16, Cout = 32)");
    cudaStream_t st = (cudaStream_t)stream;
#define PFX_CONV_FEAT(S_)                                                                     \
    do {                                                                                     \
        const int Ho = (H - 1) / S_ + 1, Wo = (W - 1) / S_ + 1;                               \
        const dim3 grid(blocks_for(Wo, kCvT), blocks_for(Ho, kCvT), 1);                       \
        if (y_bf16)                                                                          \
            k_conv3x3_fwd_feat<S_, 32, __nv_bfloat16><<<grid, kCvT * kCvT, 0, st>>>(          \
                A, B, d, H, W, w, b, Cout, Ho, Wo, relu, static_cast<__nv_bfloat16*>(y));    \
        else                                                                                 \
            k_conv3x3_fwd_feat<S_, 32, float><<<grid, kCvT * kCvT, 0, st>>>(                  \
                A, B, d, H, W, w, b, Cout, Ho, Wo, relu, static_cast<float*>(y));            \
    } while (0)
    if (stride == 4)
        PFX_CONV_FEAT(4);
    else if (stride == 2)
        PFX_CONV_FEAT(2);
    else
        PFX_CONV_FEAT(1);
#undef PFX_CONV_FEAT
    PFX_CNN_LAUNCHED();
}

extern "C" int pfx_conv3x3_forward(const void* x, int32_t x_bf16, int32_t Cin, int32_t H,
                                   int32_t W, const float* w, const float* b, int32_t Cout,
                                   int32_t stride, int32_t relu, void* y, int32_t y_bf16,
                                   void* stream) {
    if (!x || !w || !b || !y || Cin < 1 || Cout < 1 || H < 1 || W < 1 ||
        (stride != 1 && stride != 2 && stride != 4) || (int64_t)H * W > (1LL << 31) / 64)
        return report_status(PFX_ERR_ARG, "pfx_conv3x3_forward: bad argument");
    PFX_CNN_RET(cnn_conv_forward(x, x_bf16, Cin, H, W, w, b, Cout, stride, relu, y, y_bf16,
                                 (cudaStream_t)stream));
}

extern "C" int pfx_conv3x3_backward(const float* x, int32_t Cin, int32_t H, int32_t W,
                                    const float* w, int32_t Cout, int32_t stride, const float* y,
                                    int32_t relu, const float* dy, float* dx, float* dw, float* db,
                                    void* stream) {
    if (!x || !w || !y || !dy || !dw || !db || Cin < 1 || Cout < 1 || Cout > 64 || H < 1 ||
        W < 1 || (stride != 1 && stride != 2 && stride != 4))
        return report_status(PFX_ERR_ARG, "pfx_conv3x3_backward: bad argument");
    PFX_CNN_RET(cnn_conv_backward(x, Cin, H, W, w, Cout, stride, y, relu, dy, dx, dw, db,
                                  (cudaStream_t)stream));
}

extern "C" int pfx_tile_max(const float* logits, int32_t H, int32_t W, int32_t n1, int32_t n2,
                            int64_t hop, int64_t L, int64_t N, int64_t M, int32_t fpp,
                            float* score, int32_t* argmax, void* stream) {
    if (!logits || !score || !argmax || n1 < 1 || n2 < 1 || fpp < 1 || H < 1 || W < 1 ||
        hop < 1 || L < 2)
        return report_status(PFX_ERR_ARG, "pfx_tile_max: bad argument");
    k_tile_max<<<(unsigned)(n1 * n2), 256, 0, (cudaStream_t)stream>>>(logits, H, W, n1, n2, hop,
                                                                     L, N, M, fpp, score, argmax);
    PFX_CNN_LAUNCHED();
}

extern "C" int pfx_tile_bce(const float* score, const uint8_t* label, int32_t n, float pos_weight,
                            float* loss, float* dscore, void* stream) {
    if (!score || !label || !loss || !dscore || n < 1)
        return report_status(PFX_ERR_ARG, "pfx_tile_bce: bad argument");
    k_tile_bce<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(score, label, n, pos_weight,
                                                                    loss, dscore);
    PFX_CNN_LAUNCHED();
}

extern "C" int pfx_tile_max_backward(const float* dscore, const int32_t* argmax, int32_t n,
                                     float* dlogits, void* stream) {
    if (!dscore || !argmax || !dlogits || n < 1)
        return report_status(PFX_ERR_ARG, "pfx_tile_max_backward: bad argument");
    k_tile_max_bwd<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(dscore, argmax, n,
                                                                        dlogits);
    PFX_CNN_LAUNCHED();
}

extern "C" int pfx_adam_step(float* param, const float* grad, float* m, float* v, int64_t n,
                             float lr, float beta1, float beta2, float eps, int32_t step,
                             void* stream) {
    if (!param || !grad || !m || !v || n < 1 || step < 1)
        return report_status(PFX_ERR_ARG, "pfx_adam_step: bad argument");
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    k_adam<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(param, grad, m, v, n, lr, beta1,
                                                                beta2, eps, c1, c2);
    PFX_CNN_LAUNCHED();
}

extern "C" int pfx_tile_mask_from_scores(const float* score, int32_t n1, int32_t n2,
                                         float threshold, int32_t dilation, int32_t manhattan,
                                         uint8_t* mask, void* stream) {
    if (!score || !mask || n1 < 1 || n2 < 1 || dilation < 0)
        return report_status(PFX_ERR_ARG, "pfx_tile_mask_from_scores: bad argument");
    k_tile_mask<<<blocks_for((int64_t)n1 * n2, 256), 256, 0, (cudaStream_t)stream>>>(
        score, n1, n2, threshold, dilation, manhattan, mask);
    PFX_CNN_LAUNCHED();
}
