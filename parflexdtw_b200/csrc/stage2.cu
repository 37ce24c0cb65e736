// Stage 2 on the device: edge tensors, sparse valid mask, cross-tile cost
// propagation, overlap sync, global top/right edge scan, and the stitched
// backtrace.  Every rule restates Parflex.py literally; the tile loops of the
// reference become grids over edge slots.  All slot arrays are laid out like
// the reference's 4-D arrays: [n1][n2][2][L] (edge 0 = top edge = the tile's
// last row, indexed by column; edge 1 = right edge = its last column, indexed
// by row).
#include "common.cuh"

#include <math_constants.h>

#include <cmath>

namespace pfx {


__device__ __forceinline__ int64_t slot(const Geo& g, int i, int j, int e, int64_t p) {
    return (((int64_t)i * g.n2 + j) * 2 + e) * g.L + p;
}

__device__ __forceinline__ void decode_start(int32_t s, int32_t* sr, int32_t* sc) {
    // _build_edge_data (Parflex.py:531-546): > 0 bottom edge, < 0 left edge,
    // 0 the corner.
    if (s > 0) { *sr = 0; *sc = s; }
    else if (s < 0) { *sr = -s; *sc = 0; }
    else { *sr = 0; *sc = 0; }
}

// Fill value kernels ------------------------------------------------------
__global__ void k_fill_f64(double* p, int64_t n, double v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

// 1 - sum_f a[f * lda] * b[f * ldb], every product and sum rounded in the
// order f = 0, 1, ..., d-1: the value the cost kernels store for that cell.
__device__ __forceinline__ double cost_from_features(const double* a, int64_t lda,
                                                     const double* b, int64_t ldb, int d) {
    double acc = __dmul_rn(a[0], b[0]);
    for (int f = 1; f < d; ++f) acc = __dadd_rn(acc, __dmul_rn(a[f * lda], b[f * ldb]));
    return __dsub_rn(1.0, acc);
}

// Edge tensors + valid mask (Parflex.py:509-564, 347-373, 582-624) -------
// C: row-major cost (leading dimension g.ldc), or null to read the tile-skewed
// copy Csk (per-tile stride `skew_stride` elements; FP32 elements when `f32`,
// widened exactly to FP64), or, with An non-null, computed from the
// normalised features (An: [d][N], Bn: [d][M]).
__global__ void k_edges(const double* __restrict__ C, const void* __restrict__ Csk,
                        int64_t skew_stride, bool f32, const Geo g, S2Buf b,
                        const double* __restrict__ An, const double* __restrict__ Bn, int d) {
    const int64_t total = (int64_t)g.n1 * g.n2 * 2 * g.L;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pos = q % g.L;
        const int64_t te = q / g.L;
        const int e = (int)(te % 2);
        const int64_t t = te / 2;
        const int i = (int)(t / g.n2), j = (int)(t % g.n2);
        int64_t r0, c0;
        int32_t R, W;
        tile_rect(g, i, j, &r0, &c0, &R, &W);
        const int32_t elen = e == 0 ? W : R;
        if (pos >= elen) { b.edge_Cf[q] = 0.0; continue; }
        const int32_t s = b.edge_P[q];
        int32_t sr, sc;
        decode_start(s, &sr, &sc);
        const int64_t slab = b.tile_slot ? b.tile_slot[t] : t;
        const int64_t si = slab * skew_stride + skew_index(W, sr, sc);
        // a tile stage 1 skipped has no cost slab: its edges are +inf anyway
        b.edge_Cf[q] = slab < 0 ? 0.0
                       : An ? cost_from_features(An + r0 + sr, g.N, Bn + c0 + sc, g.M, d)
                       : (C ? C[(r0 + sr) * g.ldc + c0 + sc]
                            : (f32 ? (double)static_cast<const float*>(Csk)[si]
                                   : static_cast<const double*>(Csk)[si]));
        // mandatory slots: whole top edge of the last tile row, whole right
        // edge of the last tile column, and both ends of every edge
        const bool last = e == 0 ? (i == g.n1 - 1) : (j == g.n2 - 1);
        if (last || pos == 0 || pos == elen - 1) b.valid[q] = 1;
        // starts_bot_edge of tile (i, j) marks the top edge of (i-1, j);
        // starts_left_edge marks the right edge of (i, j-1)
        if (s > 0) {
            if (i >= 1 && s < W) b.valid[slot(g, i - 1, j, 0, s)] = 1;
        } else {
            if (j >= 1) {
                int64_t pr0, pc0;
                int32_t pR, pW;
                tile_rect(g, i, j - 1, &pr0, &pc0, &pR, &pW);
                if (-s < pR) b.valid[slot(g, i, j - 1, 1, -s)] = 1;
            }
        }
    }
}

// Predecessor edge slot holding global cell (gr, gc) of tile (pi, pj)
// (Parflex.py:686-700, 822-839).
__device__ __forceinline__ bool prev_slot(const Geo& g, int pi, int pj, int64_t gr, int64_t gc,
                                          int* pe, int64_t* pp) {
    int64_t r0, c0;
    int32_t R, W;
    tile_rect(g, pi, pj, &r0, &c0, &R, &W);
    const int64_t lr = gr - r0, lc = gc - c0;
    int64_t elen;
    if (lr == R - 1) { *pe = 0; *pp = lc; elen = W; }
    else if (lc == W - 1) { *pe = 1; *pp = lr; elen = R; }
    else return false;
    return *pp >= 0 && *pp < elen;
}

// Stage-2 DP (_nb_initialize_chunks_sparse / _nb_dp_fill_chunks_sparse,
// Parflex.py:632-855), tile anti-diagonal by anti-diagonal: every slot reads
// only slots of tiles (i-1, j) and (i, j-1), so a diagonal's tiles are
// independent.

// Unconditional inheritance of position 0 on the first tile row / column.
__device__ __forceinline__ void prop_inherit(const Geo& g, S2Buf& b, int i, int j) {
    double* D = b.D_arr;
    double* Lr = b.L_arr;
    if (i == 0 && j >= 1) {
        int64_t pr0, pc0;
        int32_t pR, pW;
        tile_rect(g, 0, j - 1, &pr0, &pc0, &pR, &pW);
        D[slot(g, 0, j, 0, 0)] = D[slot(g, 0, j - 1, 0, pW - 1)];
        Lr[slot(g, 0, j, 0, 0)] = Lr[slot(g, 0, j - 1, 0, pW - 1)];
    } else if (j == 0 && i >= 1) {
        int64_t pr0, pc0;
        int32_t pR, pW;
        tile_rect(g, i - 1, 0, &pr0, &pc0, &pR, &pW);
        D[slot(g, i, 0, 1, 0)] = D[slot(g, i - 1, 0, 1, pR - 1)];
        Lr[slot(g, i, 0, 1, 0)] = Lr[slot(g, i - 1, 0, 1, pR - 1)];
    }
}

// Slot q (edge q / L, position q % L) of tile (i, j).
__device__ __forceinline__ void prop_slot(const Geo& g, S2Buf& b, int i, int j, int64_t r0,
                                          int64_t c0, int32_t R, int32_t W, int q) {
    double* D = b.D_arr;
    double* Lr = b.L_arr;
    const int e = q / g.L;
    const int pos = q % g.L;
    const int32_t elen = e == 0 ? W : R;
    if (pos >= elen) return;
    const int64_t k = slot(g, i, j, e, pos);
    if (i == 0 && j == 0) {
        if (!b.valid[k]) return;
    } else if (i == 0 || j == 0) {
        if (pos == 0 || !b.valid[k]) return;
    } else {
        if (!b.valid[k]) return;
        if (pos == 0) {
            int64_t src;
            if (e == 0) {
                int64_t pr0, pc0;
                int32_t pR, pW;
                tile_rect(g, i, j - 1, &pr0, &pc0, &pR, &pW);
                src = slot(g, i, j - 1, 0, pW - 1);
            } else {
                int64_t pr0, pc0;
                int32_t pR, pW;
                tile_rect(g, i - 1, j, &pr0, &pc0, &pR, &pW);
                src = slot(g, i - 1, j, 1, pR - 1);
            }
            const double v = D[src];
            if (isfinite(v)) {
                D[k] = v;
                Lr[k] = Lr[src];
            }
            return;
        }
    }
    int32_t sr, sc;
    decode_start(b.edge_P[k], &sr, &sc);
    const int32_t lr = e == 0 ? R - 1 : pos, lc = e == 0 ? pos : W - 1;
    const double own_len = (double)(abs(lr - sr) + abs(lc - sc));
    int pi, pj;
    if (i == 0 && j == 0) {
        if (sr == 0 || sc == 0) { D[k] = b.edge_D[k]; Lr[k] = own_len; }
        return;
    } else if (i == 0) {
        if (sr == 0) { D[k] = b.edge_D[k]; Lr[k] = own_len; return; }
        if (sc != 0) return;
        pi = 0; pj = j - 1;
    } else if (j == 0) {
        if (sc == 0) { D[k] = b.edge_D[k]; Lr[k] = own_len; return; }
        if (sr != 0) return;
        pi = i - 1; pj = 0;
    } else {
        if (sr == 0) { pi = i - 1; pj = j; }
        else if (sc == 0) { pi = i; pj = j - 1; }
        else { D[k] = b.edge_D[k]; Lr[k] = own_len; return; }
    }
    int pe;
    int64_t pp;
    if (!prev_slot(g, pi, pj, r0 + sr, c0 + sc, &pe, &pp)) return;
    const int64_t src = slot(g, pi, pj, pe, pp);
    const double prev = D[src];
    if (!isfinite(prev)) return;
    D[k] = __dsub_rn(__dadd_rn(prev, b.edge_D[k]), b.edge_Cf[k]);
    Lr[k] = __dadd_rn(__dadd_rn(Lr[src], (double)abs(lr - sr)), (double)abs(lc - sc));
}

// One anti-diagonal a per launch (large grids).
__global__ void k_propagate(const Geo g, S2Buf b, int a) {
    const int ilo = a - (g.n2 - 1) > 0 ? a - (g.n2 - 1) : 0;
    const int i = ilo + (int)blockIdx.y;
    const int j = a - i;
    if (i >= g.n1 || j < 0) return;
    int64_t r0, c0;
    int32_t R, W;
    tile_rect(g, i, j, &r0, &c0, &R, &W);
    if (blockIdx.x == 0 && threadIdx.x == 0) prop_inherit(g, b, i, j);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 2 * g.L; q += gridDim.x * blockDim.x)
        prop_slot(g, b, i, j, r0, c0, R, W, q);
}

// Every anti-diagonal in one CTA (small grids: one launch instead of
// n1 + n2 - 1); a CTA barrier orders the diagonals.
constexpr int kPropAllThreads = 1024;

__global__ void __launch_bounds__(kPropAllThreads) k_propagate_all(const Geo g, S2Buf b) {
    const int per = 2 * g.L;
    for (int a = 0; a <= g.n1 + g.n2 - 2; ++a) {
        const int ilo = a - (g.n2 - 1) > 0 ? a - (g.n2 - 1) : 0;
        const int ihi = a < g.n1 - 1 ? a : g.n1 - 1;
        const int nt = ihi - ilo + 1;
        if ((int)threadIdx.x < nt) prop_inherit(g, b, ilo + (int)threadIdx.x, a - ilo - (int)threadIdx.x);
        for (int x = threadIdx.x; x < nt * per; x += kPropAllThreads) {
            const int i = ilo + x / per, j = a - i;
            int64_t r0, c0;
            int32_t R, W;
            tile_rect(g, i, j, &r0, &c0, &R, &W);
            prop_slot(g, b, i, j, r0, c0, R, W, x % per);
        }
        __syncthreads();
    }
}

// sync_tile_overlap_edges (Parflex.py:920-969).  Loops 1 and 2 touch
// disjoint slots (edge 0 / edge 1) and their pairs are disjoint, loop 3 runs
// after both.
__global__ void k_sync(const Geo g, S2Buf b) {
    double* D = b.D_arr;
    double* Lr = b.L_arr;
    const int nt = g.n1 * g.n2;
    for (int t = threadIdx.x; t < 2 * nt; t += blockDim.x) {
        const int which = t / nt, tt = t % nt;
        const int i = tt / g.n2, j = tt % g.n2;
        int64_t r0, c0;
        int32_t R, W;
        tile_rect(g, i, j, &r0, &c0, &R, &W);
        int64_t a, c;
        if (which == 0) {
            if (j + 1 >= g.n2) continue;
            a = slot(g, i, j, 0, W - 1);
            c = slot(g, i, j + 1, 0, 0);
        } else {
            if (i + 1 >= g.n1) continue;
            a = slot(g, i, j, 1, R - 1);
            c = slot(g, i + 1, j, 1, 0);
        }
        const bool fa = isfinite(D[a]), fc = isfinite(D[c]);
        if (fa && !fc) { D[c] = D[a]; Lr[c] = Lr[a]; }
        else if (!fa && fc) { D[a] = D[c]; Lr[a] = Lr[c]; }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
        const int i = t / g.n2, j = t % g.n2;
        int64_t r0, c0;
        int32_t R, W;
        tile_rect(g, i, j, &r0, &c0, &R, &W);
        const int64_t tc = slot(g, i, j, 0, W - 1), rc = slot(g, i, j, 1, R - 1);
        const bool ft = isfinite(D[tc]), fr = isfinite(D[rc]);
        if (ft && !fr) { D[rc] = D[tc]; Lr[rc] = Lr[tc]; }
        else if (!ft && fr) { D[tc] = D[rc]; Lr[tc] = Lr[rc]; }
        else if (ft && fr && fabs(D[tc] - D[rc]) > 1e-10) { D[rc] = D[tc]; Lr[rc] = Lr[tc]; }
    }
}

// Global edge scan (_build_edge_lookups + _nb_scan_edges,
// Parflex.py:1110-1222).  Block s scans one L-wide segment of the global
// top edge (s < nseg_top) or right edge.  The first owner of a global top
// column g is tile (n1-1, g == 0 ? 0 : (g-1)/hop) at position g - j*hop (the
// last tile row is the only one containing row N-1, and of two tiles sharing
// column g the lower j is visited first); likewise for right-edge rows.
__global__ void k_scan_segments(const Geo g, S2Buf b, int nseg_top, int64_t buf) {
    const int s = blockIdx.x;
    const bool top = s < nseg_top;
    const int seg = top ? s : s - nseg_top;
    const int64_t G = top ? g.M : g.N;
    const int64_t lo = (int64_t)seg * g.L;
    const int64_t hi = lo + g.L < G ? lo + g.L : G;
    double bn = CUDART_INF;
    int64_t bgi = -1;
    for (int64_t gi = lo + threadIdx.x; gi < hi; gi += blockDim.x) {
        if (buf > 0 && gi < buf) continue;
        const int tj_or_i = gi == 0 ? 0 : (int)((gi - 1) / g.hop);
        const int ci = top ? g.n1 - 1 : tj_or_i;
        const int cj = top ? tj_or_i : g.n2 - 1;
        const int et = top ? 0 : 1;
        const int64_t idx = gi - (int64_t)tj_or_i * g.hop;
        const int64_t k = slot(g, ci, cj, et, idx);
        const double Dv = b.D_arr[k], Lv = b.L_arr[k];
        if (!isfinite(Dv) || Lv <= 0.0) continue;
        if (top && Dv >= 1e9) continue;
        const double nrm = __ddiv_rn(Dv, Lv);
        if (top) { b.top_D[gi] = Dv; b.top_L[gi] = Lv; }
        else { b.right_D[gi] = Dv; b.right_L[gi] = Lv; }
        if (nrm < bn) { bn = nrm; bgi = gi; }  // strided: gi ascends per thread
    }
    // block first-minimum: smaller norm, then smaller index
    __shared__ double sn[1024];
    __shared__ int64_t sg[1024];
    sn[threadIdx.x] = bn;
    sg[threadIdx.x] = bgi;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            const double on = sn[threadIdx.x + w];
            const int64_t og = sg[threadIdx.x + w];
            const double mn = sn[threadIdx.x];
            const int64_t mg = sg[threadIdx.x];
            if (og >= 0 && (mg < 0 || on < mn || (on == mn && og < mg))) {
                sn[threadIdx.x] = on;
                sg[threadIdx.x] = og;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const int row = top ? 0 : 1;
        const int64_t gi = sg[0];
        int64_t* m = b.seg_meta + ((int64_t)row * b.max_segs + seg) * 6;
        if (gi >= 0) {
            const int tj_or_i = gi == 0 ? 0 : (int)((gi - 1) / g.hop);
            b.seg_norm[row * b.max_segs + seg] = sn[0];
            m[0] = top ? g.n1 - 1 : tj_or_i;
            m[1] = top ? tj_or_i : g.n2 - 1;
            m[2] = row;
            m[3] = gi - (int64_t)tj_or_i * g.hop;
            m[4] = top ? g.N - 1 : gi;
            m[5] = top ? gi : g.M - 1;
        } else {
            b.seg_norm[row * b.max_segs + seg] = CUDART_INF;
            for (int f = 0; f < 6; ++f) m[f] = -1;
        }
    }
}

// Global winner from the per-segment winners, in scan order (top segments,
// then right segments); strict < against the running best that starts at
// LARGE = 1e9 (Parflex.py:1167-1168).
__global__ void k_scan_final(const Geo g, S2Buf b, int nseg_top, int nseg_right) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double best = 1e9;
    int64_t found = 0;
    int64_t e[6] = {-1, -1, -1, -1, -1, -1};
    for (int s = 0; s < nseg_top + nseg_right; ++s) {
        const int row = s < nseg_top ? 0 : 1;
        const int seg = s < nseg_top ? s : s - nseg_top;
        const int64_t* m = b.seg_meta + ((int64_t)row * b.max_segs + seg) * 6;
        const double nrm = b.seg_norm[row * b.max_segs + seg];
        if (m[0] >= 0 && nrm < best) {
            best = nrm;
            found = 1;
            e[0] = m[4]; e[1] = m[5]; e[2] = m[0]; e[3] = m[1]; e[4] = m[2]; e[5] = m[3];
        }
    }
    *b.best = best;
    for (int f = 0; f < 6; ++f) b.best_end[f] = e[f];
    b.best_end[6] = found;
}

// Tile chain of the stitched backtrace (backtrace_and_stitch,
// Parflex.py:1032-1103).  The chain needs only the start encodings on the
// tile edges, so it is followed first and the per-tile walks run in
// parallel afterwards.  Entry fields: i j edge idx end_r end_c start_r
// start_c row0 col0 rows cols.
__global__ void k_stitch_chain(const Geo g, S2Buf b, int64_t start_i, int64_t start_j,
                               int64_t start_e, int64_t start_x, int from_best) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int64_t ci = start_i, cj = start_j, ce = start_e, cx = start_x;
    if (from_best) {
        if (!b.best_end[6]) { *b.chain_len = 0; return; }
        ci = b.best_end[2]; cj = b.best_end[3]; ce = b.best_end[4]; cx = b.best_end[5];
    }
    int n = 0;
    for (int it = 0; it < 101; ++it) {
        if (ci < 0 || cj < 0 || ci >= g.n1 || cj >= g.n2) break;
        int64_t r0, c0;
        int32_t R, W;
        tile_rect(g, (int)ci, (int)cj, &r0, &c0, &R, &W);
        const int32_t er = ce == 0 ? R - 1 : (int32_t)cx;
        const int32_t ec = ce == 0 ? (int32_t)cx : W - 1;
        const int32_t sv = b.edge_P[slot(g, (int)ci, (int)cj, (int)ce, cx)];
        const int32_t sr = sv >= 0 ? 0 : -sv, sc = sv >= 0 ? sv : 0;
        int32_t* E = b.chain + n * 12;
        E[0] = (int32_t)ci; E[1] = (int32_t)cj; E[2] = (int32_t)ce; E[3] = (int32_t)cx;
        E[4] = er; E[5] = ec; E[6] = sr; E[7] = sc;
        E[8] = (int32_t)r0; E[9] = (int32_t)c0; E[10] = R; E[11] = W;
        ++n;
        const int64_t gsr = r0 + sr, gsc = c0 + sc;
        if (gsr == 0 || gsc == 0) break;
        const bool corner = sr == 0 && sc == 0;
        int64_t pi, pj, pe;
        if (corner) { pi = ci - 1; pj = cj - 1; pe = 0; }
        else if (sv >= 0) { pi = ci - 1; pj = cj; pe = 0; }
        else { pi = ci; pj = cj - 1; pe = 1; }
        if (pi < 0 || pj < 0 || pi >= g.n1 || pj >= g.n2) break;
        int64_t pr0, pc0;
        int32_t pR, pW;
        tile_rect(g, (int)pi, (int)pj, &pr0, &pc0, &pR, &pW);
        int64_t pidx, pmax;
        if (corner) { pidx = pW - 1; pmax = pW; }
        else {
            pidx = pe == 0 ? gsc - pc0 : gsr - pr0;
            pmax = pe == 0 ? pW : pR;
        }
        if (pidx < 0 || pidx >= pmax) break;
        ci = pi; cj = pj; ce = pe; cx = pidx;
    }
    *b.chain_len = n;
}

// One chain entry per warp: walk the packed backpointers from the entry's
// end cell to its start cell (_nb_backtrace_within_chunk,
// Parflex.py:977-1012), writing global points end-first.  The walk only
// moves up and left, so the warp stages a 64-row x 64-column window of
// backpointer words (rows w0+l and w0+32+l loaded by lane l, five 16-cell
// words each) in its own shared memory, anchored with the current cell at
// its bottom-right corner.  Every lane then follows the same path, reading
// each step's word with one broadcast shared-memory load (no shuffle in the
// step's dependency chain).  The window is reloaded (one coalesced round
// trip) only when the path leaves it, about every 32-63 steps, instead of
// one dependent global load per step.
constexpr int kWalkThreads = 128;

__global__ void __launch_bounds__(kWalkThreads) k_stitch_walk(const Geo g, S2Buf b) {
    __shared__ uint32_t s_win[kWalkThreads / 32][64][5];  // per warp: window row x word
    const int n = *b.chain_len;
    const int lane = threadIdx.x & 31;
    const int e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (e >= n) return;
    uint32_t (*win)[5] = s_win[threadIdx.x >> 5];
    const int32_t* E = b.chain + e * 12;
    const int32_t ti = E[0], tj = E[1];
    int32_t r = E[4], c = E[5];
    const int32_t sr = E[6], sc = E[7], gro = E[8], gco = E[9], R = E[10], W = E[11];
    const uint32_t* slab = b.Bw + ((int64_t)ti * g.n2 + tj) * g.b_words;
    const int32_t nP = ceil_div32(W + kStripRows - 1, kBlk);
    int32_t* out = b.seg_pts + (int64_t)e * b.seg_cap * 2;
    int64_t k = 0;
    const int64_t max_iters = (int64_t)R + W;
    bool done = false;
    int32_t w0r = -1, w0c = 0;  // window origin (row, column); -1 = empty
    for (int64_t it = 0; it < max_iters; ++it) {
        if (lane == 0) { out[2 * k] = r + gro; out[2 * k + 1] = c + gco; }
        ++k;
        if (r == sr && c == sc) { done = true; break; }
        if (w0r < 0 || r < w0r || c < w0c) {
            w0r = r - 63 > 0 ? r - 63 : 0;
            w0c = c - 63 > 0 ? c - 63 : 0;
            __syncwarp();  // every lane is done with the previous window
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int32_t ra = w0r + 32 * h + lane;
                const int32_t pa = (w0c + (ra & 63)) >> 4;  // first period held for row ra
#pragma unroll
                for (int q = 0; q < 5; ++q)
                    win[32 * h + lane][q] =
                        (ra < R && pa + q < nP) ? __ldg(slab + bp_word_index2(W, ra, (pa + q) << 4))
                                                : 0u;
            }
            __syncwarp();
        }
        // word of cell (r, c): row r - w0r (0..63) of the window, period
        // (c + rho) / 16 counted from the row's first period (w0c + rho) / 16,
        // rho = r mod 64 (0..4, since c - w0c is 0..63)
        const int32_t rr = r & 63;
        const uint32_t word = win[r - w0r][((c + rr) >> 4) - ((w0c + rr) >> 4)];
        const int code = (int)((word >> (((c + rr) & 15) * 2)) & 3u);
        if (code >= g.S) { done = false; break; }
        const int kd = code == 0 ? g.kind[0] : (code == 1 ? g.kind[1] : g.kind[2]);
        const int32_t pr = r - (kd == 2 ? 2 : 1), pc = c - (kd == 1 ? 2 : 1);
        if (pr < 0 || pc < 0 || pr >= R || pc >= W) { done = false; break; }
        r = pr; c = pc;
    }
    if (!done && (r != sr || c != sc)) {
        if (lane == 0) { out[2 * k] = sr + gro; out[2 * k + 1] = sc + gco; }
        ++k;
    }
    if (lane == 0) b.seg_len[e] = (int32_t)k;
}

// Concatenate the walks with consecutive-duplicate removal and reverse to
// start-first order.  Inside one walk consecutive points always differ, so
// only the first point of a walk can repeat the last point of the previous.
__global__ void k_stitch_concat(S2Buf b) {
    __shared__ int64_t off[102];
    __shared__ int32_t drop[101];
    const int n = *b.chain_len;
    if (threadIdx.x == 0) {
        int64_t o = 0;
        for (int e = 0; e < n; ++e) {
            int d = 0;
            if (e > 0) {
                const int32_t* prev = b.seg_pts + (int64_t)(e - 1) * b.seg_cap * 2;
                const int32_t* cur = b.seg_pts + (int64_t)e * b.seg_cap * 2;
                const int32_t pl = b.seg_len[e - 1];
                d = (cur[0] == prev[2 * (pl - 1)] && cur[1] == prev[2 * (pl - 1) + 1]) ? 1 : 0;
            }
            drop[e] = d;
            off[e] = o;
            o += b.seg_len[e] - d;
        }
        off[n] = o;
        *b.wp_len = o;
    }
    __syncthreads();
    const int64_t K = off[n];
    for (int e = 0; e < n; ++e) {
        const int32_t* src = b.seg_pts + (int64_t)e * b.seg_cap * 2;
        const int32_t len = b.seg_len[e], d = drop[e];
        for (int m = d + threadIdx.x; m < len; m += blockDim.x) {
            const int64_t q = off[e] + m - d;
            b.wp[2 * (K - 1 - q)] = src[2 * m];
            b.wp[2 * (K - 1 - q) + 1] = src[2 * m + 1];
        }
    }
}

// Host-side launch sequence ------------------------------------------------
cudaError_t launch_fill(double* p, int64_t n, double v, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    int64_t blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    k_fill_f64<<<(int)blocks, 256, 0, st>>>(p, n, v);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_stage2(const double* C, const void* Csk, int64_t skew_stride, bool f32,
                          const Geo& g, const S2Buf& b, cudaStream_t st) {
    cudaError_t e = launch_stage2_edges(C, Csk, skew_stride, f32, g, b, st);
    return e != cudaSuccess ? e : launch_stage2_prop(g, b, st);
}

cudaError_t launch_stage2_edges(const double* C, const void* Csk, int64_t skew_stride, bool f32,
                                const Geo& g, const S2Buf& b, cudaStream_t st, const double* An,
                                const double* Bn, int d) {
    const int64_t nslots = (int64_t)g.n1 * g.n2 * 2 * g.L;
    cudaError_t e;
    if ((e = cudaMemsetAsync(b.valid, 0, (size_t)nslots, st)) != cudaSuccess) return e;
    if ((e = launch_fill(b.D_arr, nslots, HUGE_VAL, st)) != cudaSuccess) return e;
    if ((e = launch_fill(b.L_arr, nslots, HUGE_VAL, st)) != cudaSuccess) return e;
    {
        int64_t blocks = (nslots + 255) / 256;
        if (blocks > 8192) blocks = 8192;
        k_edges<<<(int)blocks, 256, 0, st>>>(C, Csk, skew_stride, f32, g, b, An, Bn, d);
        count_launches(1);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_stage2_prop(const Geo& g, const S2Buf& b, cudaStream_t st) {
    cudaError_t e;
    if ((int64_t)g.n1 * g.n2 * 2 * g.L <= (1 << 18)) {
        k_propagate_all<<<1, kPropAllThreads, 0, st>>>(g, b);
        count_launches(1);
        return cudaGetLastError();
    }
    for (int a = 0; a <= g.n1 + g.n2 - 2; ++a) {
        const int ilo = a - (g.n2 - 1) > 0 ? a - (g.n2 - 1) : 0;
        const int ihi = a < g.n1 - 1 ? a : g.n1 - 1;
        const dim3 grid((unsigned)ceil_div32(2 * g.L, 256), (unsigned)(ihi - ilo + 1));
        k_propagate<<<grid, 256, 0, st>>>(g, b, a);
        count_launches(1);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_sync_scan(const Geo& g, const S2Buf& b, int64_t buf, cudaStream_t st) {
    cudaError_t e;
    k_sync<<<1, 1024, 0, st>>>(g, b);
    count_launches(1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_fill(b.top_D, g.M, NAN, st)) != cudaSuccess) return e;
    if ((e = launch_fill(b.right_D, g.N, NAN, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(b.top_L, 0, sizeof(double) * g.M, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(b.right_L, 0, sizeof(double) * g.N, st)) != cudaSuccess) return e;
    if ((e = launch_fill(b.seg_norm, 2 * (int64_t)b.max_segs, HUGE_VAL, st)) != cudaSuccess)
        return e;
    if ((e = cudaMemsetAsync(b.seg_meta, 0xff, sizeof(int64_t) * 12 * b.max_segs, st)) !=
        cudaSuccess)
        return e;
    const int nst = (int)ceil_div64(g.M, g.L), nsr = (int)ceil_div64(g.N, g.L);
    k_scan_segments<<<nst + nsr, 1024, 0, st>>>(g, b, nst, buf);
    count_launches(1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_scan_final<<<1, 32, 0, st>>>(g, b, nst, nsr);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_stitch_chain(const Geo& g, const S2Buf& b, cudaStream_t st, int from_best,
                                int64_t si, int64_t sj, int64_t se, int64_t sx) {
    k_stitch_chain<<<1, 32, 0, st>>>(g, b, si, sj, se, sx, from_best);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_stitch(const Geo& g, const S2Buf& b, cudaStream_t st, int from_best,
                          int64_t si, int64_t sj, int64_t se, int64_t sx) {
    cudaError_t e;
    if ((e = launch_stitch_chain(g, b, st, from_best, si, sj, se, sx)) != cudaSuccess) return e;
    k_stitch_walk<<<26, kWalkThreads, 0, st>>>(g, b);  // one warp per chain entry (<= 101)
    count_launches(1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_stitch_concat<<<1, 1024, 0, st>>>(b);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace pfx
