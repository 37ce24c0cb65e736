/*
 * parflex_oracle.c -- CPU restatement of ParFlex (tiled FlexDTW + stage 2).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle that the device
 * implementation is checked against, and the CPU baseline that bench.py times
 * beside it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.  The product path (parflexdtw_b200) never calls it.
 *
 * It restates, in plain C, the reference algorithm (ishitajain21/ParFlexDTW):
 *   - FlexDTW.flexdtw tile DP ............ FlexDTW.py:326-378
 *   - find_best_endpoint ................. FlexDTW.py:104-154
 *   - backtrace_flexdtw .................. FlexDTW.py:161-186
 *   - run_flexdtw_on_tiles geometry ...... Parflex.py:376-469
 *   - _build_edge_data ................... Parflex.py:509-564
 *   - _build_valid_mask / starts sets .... Parflex.py:347-373, 582-624
 *   - _nb_initialize_chunks_sparse ....... Parflex.py:632-760
 *   - _nb_dp_fill_chunks_sparse .......... Parflex.py:764-855
 *   - sync_tile_overlap_edges ............ Parflex.py:920-969
 *   - _nb_backtrace_within_chunk ......... Parflex.py:977-1012
 *   - backtrace_and_stitch ............... Parflex.py:1032-1103
 *   - _build_edge_lookups ................ Parflex.py:1110-1150
 *   - _nb_scan_edges ..................... Parflex.py:1154-1222
 *   - stage2_scan_and_stitch / parflex ... Parflex.py:1229-1356, 1510-1547
 *
 * Arithmetic is IEEE FP64 with no contraction (compile with
 * -ffp-contract=off), matching Numba's non-fastmath code for the DP.
 *
 * The FP32 form (oracle_tile_dp_f32, oracle_parflex2 with fp32 = 1) is the
 * same recurrence with every DP value in FP32 -- cost, accumulated cost,
 * path cost and the quotient path cost / path length -- and the weights
 * rounded to FP32; stage 2 then runs in FP64 on the exactly widened FP32
 * edge values.  It has no counterpart in the reference: it defines the
 * device's FP32 DP, which the tests hold to it bit for bit.
 * Parity of this restatement is pinned by tests/test_oracle_golden.py
 * against fixtures produced by the reference itself
 * (tests/golden/make_golden.py).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_MAX_STEPS 8

/* ------------------------------------------------------------------------ */
/* Tile DP (FlexDTW.py:326-370).  C is a tile view with leading dimension   */
/* ldc.  D, P, B are R*W row-major outputs (zero-initialised here, as       */
/* np.zeros does in the reference).                                          */
/* ------------------------------------------------------------------------ */
void oracle_tile_dp(const double *C, int64_t ldc, int64_t R, int64_t W,
                    const int64_t *steps, const double *weights, int S,
                    double *D, int32_t *P, int8_t *B)
{
    memset(D, 0, sizeof(double) * (size_t)(R * W));
    memset(P, 0, sizeof(int32_t) * (size_t)(R * W));
    memset(B, 0, (size_t)(R * W));
    for (int64_t c = 0; c < W; ++c) D[c] = C[c];
    for (int64_t r = 0; r < R; ++r) D[r * W] = C[r * ldc];
    for (int64_t row = 1; row < R; ++row) {
        for (int64_t col = 1; col < W; ++col) {
            const double cval = C[row * ldc + col];
            double mincost = INFINITY;
            int minidx = -1;
            int64_t bestr = -1, bestc = -1;
            for (int s = 0; s < S; ++s) {
                int64_t pr = row - steps[2 * s], pc = col - steps[2 * s + 1];
                if (pr >= 0 && pc >= 0) {
                    double pathcost = D[pr * W + pc] + cval * weights[s];
                    int64_t pp = P[pr * W + pc];
                    int64_t mdist = (pp >= 0) ? row + (col - pp) : (row + pp) + col;
                    double cpm = pathcost / (double)mdist;
                    if (cpm < mincost) {
                        mincost = cpm;
                        minidx = s;
                        bestr = pr;
                        bestc = pc;
                    }
                }
            }
            if (minidx < 0) {
                /* Numba wraps negative indices: D[-1,-1], weights[-1],
                 * P[-1,-1] (the last cell, not yet written). */
                D[row * W + col] = D[R * W - 1] + cval * weights[S - 1];
                B[row * W + col] = -1;
                P[row * W + col] = P[R * W - 1];
                continue;
            }
            D[row * W + col] = D[bestr * W + bestc] + cval * weights[minidx];
            B[row * W + col] = (int8_t)minidx;
            if (bestr == 0)
                P[row * W + col] = (int32_t)bestc;
            else if (bestc == 0)
                P[row * W + col] = (int32_t)(-bestr);
            else
                P[row * W + col] = P[bestr * W + bestc];
        }
    }
}

/* FP32 form of oracle_tile_dp (same recurrence, FP32 values). */
void oracle_tile_dp_f32(const float *C, int64_t ldc, int64_t R, int64_t W,
                        const int64_t *steps, const double *weights, int S,
                        float *D, int32_t *P, int8_t *B)
{
    float w[ORACLE_MAX_STEPS];
    for (int s = 0; s < S; ++s) w[s] = (float)weights[s];
    memset(D, 0, sizeof(float) * (size_t)(R * W));
    memset(P, 0, sizeof(int32_t) * (size_t)(R * W));
    memset(B, 0, (size_t)(R * W));
    for (int64_t c = 0; c < W; ++c) D[c] = C[c];
    for (int64_t r = 0; r < R; ++r) D[r * W] = C[r * ldc];
    for (int64_t row = 1; row < R; ++row) {
        for (int64_t col = 1; col < W; ++col) {
            const float cval = C[row * ldc + col];
            float mincost = INFINITY;
            int minidx = -1;
            int64_t bestr = -1, bestc = -1;
            for (int s = 0; s < S; ++s) {
                int64_t pr = row - steps[2 * s], pc = col - steps[2 * s + 1];
                if (pr >= 0 && pc >= 0) {
                    float pathcost = D[pr * W + pc] + cval * w[s];
                    int64_t pp = P[pr * W + pc];
                    int64_t mdist = (pp >= 0) ? row + (col - pp) : (row + pp) + col;
                    float cpm = pathcost / (float)mdist;
                    if (cpm < mincost) {
                        mincost = cpm;
                        minidx = s;
                        bestr = pr;
                        bestc = pc;
                    }
                }
            }
            if (minidx < 0) {
                D[row * W + col] = D[R * W - 1] + cval * w[S - 1];
                B[row * W + col] = -1;
                P[row * W + col] = P[R * W - 1];
                continue;
            }
            D[row * W + col] = D[bestr * W + bestc] + cval * w[minidx];
            B[row * W + col] = (int8_t)minidx;
            if (bestr == 0)
                P[row * W + col] = (int32_t)bestc;
            else if (bestc == 0)
                P[row * W + col] = (int32_t)(-bestr);
            else
                P[row * W + col] = P[bestr * W + bestc];
        }
    }
}

/* find_best_endpoint (FlexDTW.py:104-154) with an integer buffer. */
double oracle_find_best_endpoint(const double *D, const int32_t *P, int64_t R,
                                 int64_t W, int64_t buffer, int64_t *best_r,
                                 int64_t *best_c)
{
    double best = INFINITY;
    *best_r = -1;
    *best_c = -1;
    /* last row, columns buffer..W-1 */
    for (int64_t i = buffer; i < W; ++i) {
        int64_t r = R - 1, c = i;
        int64_t p = P[r * W + c];
        int64_t rs = p >= 0 ? 0 : -p, cs = p >= 0 ? p : 0;
        double avg = D[r * W + c] / (double)((r - rs) + (c - cs));
        if (avg < best) { best = avg; *best_r = r; *best_c = c; }
    }
    /* last column, rows R-2 down to buffer */
    for (int64_t i = R - 2; i >= buffer; --i) {
        int64_t r = i, c = W - 1;
        int64_t p = P[r * W + c];
        int64_t rs = p >= 0 ? 0 : -p, cs = p >= 0 ? p : 0;
        double avg = D[r * W + c] / (double)((r - rs) + (c - cs));
        if (avg < best) { best = avg; *best_r = r; *best_c = c; }
    }
    return best;
}

/* backtrace_flexdtw (FlexDTW.py:161-186); writes reversed (start-first)
 * path as (row, col) pairs, returns the number of points. */
int64_t oracle_backtrace_tile(const int8_t *B, int64_t R, int64_t W,
                              const int64_t *steps, int S, int64_t r, int64_t c,
                              int64_t *out_rc)
{
    int64_t k = 0;
    out_rc[2 * k] = r; out_rc[2 * k + 1] = c; ++k;
    while (r != 0 && c != 0) {
        int s = B[r * W + c];
        if (s < 0) s += S; /* Numba negative-index wraparound */
        r -= steps[2 * s];
        c -= steps[2 * s + 1];
        out_rc[2 * k] = r; out_rc[2 * k + 1] = c; ++k;
    }
    for (int64_t a = 0, b = k - 1; a < b; ++a, --b) {
        int64_t t0 = out_rc[2 * a], t1 = out_rc[2 * a + 1];
        out_rc[2 * a] = out_rc[2 * b]; out_rc[2 * a + 1] = out_rc[2 * b + 1];
        out_rc[2 * b] = t0; out_rc[2 * b + 1] = t1;
    }
    (void)R;
    return k;
}

/* ------------------------------------------------------------------------ */
/* Stage-1 tiling and stage 2.                                              */
/* ------------------------------------------------------------------------ */
typedef struct {
    /* geometry */
    int64_t N, M, L, hop, n1, n2;
    /* stage-1 products, [n1][n2][2][L] unless stated */
    double *edge_Df;      /* D at the top edge (edge 0) / right edge (edge 1) */
    int32_t *edge_S;      /* signed start encoding P at edge cells */
    int64_t *edge_start_r, *edge_start_c;
    double *edge_Cf_olap; /* C at the start cell */
    int64_t *edge_lens;   /* [n1][n2][2] */
    uint8_t *valid_mask;
    int8_t **tile_B;      /* per tile, R*W backpointers */
    double *tile_best;    /* per-tile find_best_endpoint cost [n1*n2] */
    int64_t *tile_wp_len; /* per-tile path length [n1*n2] */
    /* stage-2 products */
    double *D_prop, *L_prop; /* after init+fill */
    double *D_arr, *L_arr;   /* after overlap sync */
    double *top_D, *top_L;   /* [M] */
    double *right_D, *right_L; /* [N] */
    int64_t max_segs;
    double *seg_best_norm;   /* [2][max_segs] */
    int64_t *seg_best_meta;  /* [2][max_segs][6]: ci cj et idx grow gcol */
    double best_cost;
    int64_t best_end[6];
    int64_t found;
    int64_t *wp;     /* [wp_len][2] */
    int64_t wp_len;
    int64_t *tile_order; /* stitched tiles, [n_stitch][4]: i j edge idx */
    int64_t n_stitch;
} oracle_result;

static inline int64_t idx4(const oracle_result *o, int64_t i, int64_t j,
                           int64_t e, int64_t p)
{
    return ((i * o->n2 + j) * 2 + e) * o->L + p;
}

static inline void tile_bounds(const oracle_result *o, int64_t i, int64_t j,
                               int64_t *s1, int64_t *e1, int64_t *s2,
                               int64_t *e2)
{
    *s1 = i * o->hop;
    *s2 = j * o->hop;
    *e1 = *s1 + o->L < o->N ? *s1 + o->L : o->N;
    *e2 = *s2 + o->L < o->M ? *s2 + o->L : o->M;
}

void oracle_free(oracle_result *o)
{
    if (!o) return;
    free(o->edge_Df); free(o->edge_S); free(o->edge_start_r);
    free(o->edge_start_c); free(o->edge_Cf_olap); free(o->edge_lens);
    free(o->valid_mask);
    if (o->tile_B) {
        for (int64_t t = 0; t < o->n1 * o->n2; ++t) free(o->tile_B[t]);
        free(o->tile_B);
    }
    free(o->tile_best); free(o->tile_wp_len);
    free(o->D_prop); free(o->L_prop); free(o->D_arr); free(o->L_arr);
    free(o->top_D); free(o->top_L); free(o->right_D); free(o->right_L);
    free(o->seg_best_norm); free(o->seg_best_meta);
    free(o->wp); free(o->tile_order);
    memset(o, 0, sizeof(*o));
}

/* Stage 1 (Parflex.py:376-469) + edge tensors (Parflex.py:509-564). */
static int stage1(oracle_result *o, const double *C, int64_t ldc,
                  const int64_t *steps, const double *weights, int S,
                  int threads, int want_tile_wp, int fp32)
{
    const int64_t nt = o->n1 * o->n2, L = o->L;
    int failed = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
#pragma omp parallel
    {
        double *D = (double *)malloc(sizeof(double) * (size_t)(L * L));
        int32_t *P = (int32_t *)malloc(sizeof(int32_t) * (size_t)(L * L));
        float *Cf = fp32 ? (float *)malloc(sizeof(float) * (size_t)(L * L)) : NULL;
        float *Df = fp32 ? (float *)malloc(sizeof(float) * (size_t)(L * L)) : NULL;
        int64_t *wpbuf = want_tile_wp ?
            (int64_t *)malloc(sizeof(int64_t) * (size_t)(4 * L + 8)) : NULL;
        if (!D || !P || (want_tile_wp && !wpbuf) || (fp32 && (!Cf || !Df))) {
#pragma omp atomic write
            failed = 1;
        }
#pragma omp for schedule(dynamic, 1)
        for (int64_t t = 0; t < nt; ++t) {
            if (failed) continue;
            int64_t i = t / o->n2, j = t % o->n2, s1, e1, s2, e2;
            tile_bounds(o, i, j, &s1, &e1, &s2, &e2);
            int64_t R = e1 - s1, W = e2 - s2;
            int8_t *B = (int8_t *)malloc((size_t)(R * W));
            if (!B) {
#pragma omp atomic write
                failed = 1;
                continue;
            }
            const double *Ct = C + s1 * ldc + s2;
            if (fp32) {
                /* C holds FP32 values; the DP runs in FP32, D is widened */
                for (int64_t r = 0; r < R; ++r)
                    for (int64_t c = 0; c < W; ++c) Cf[r * W + c] = (float)Ct[r * ldc + c];
                oracle_tile_dp_f32(Cf, W, R, W, steps, weights, S, Df, P, B);
                for (int64_t q = 0; q < R * W; ++q) D[q] = (double)Df[q];
            } else {
                oracle_tile_dp(Ct, ldc, R, W, steps, weights, S, D, P, B);
            }
            o->tile_B[t] = B;
            if (want_tile_wp) {
                int64_t br, bc;
                o->tile_best[t] = oracle_find_best_endpoint(D, P, R, W, 1, &br, &bc);
                o->tile_wp_len[t] = br >= 0 ?
                    oracle_backtrace_tile(B, R, W, steps, S, br, bc, wpbuf) : 0;
            }
            o->edge_lens[(i * o->n2 + j) * 2 + 0] = W;
            o->edge_lens[(i * o->n2 + j) * 2 + 1] = R;
            for (int e = 0; e < 2; ++e) {
                int64_t elen = e == 0 ? W : R;
                for (int64_t pos = 0; pos < elen; ++pos) {
                    int64_t lr = e == 0 ? R - 1 : pos, lc = e == 0 ? pos : W - 1;
                    int64_t k = idx4(o, i, j, e, pos);
                    int32_t sv = P[lr * W + lc];
                    int64_t sr, sc;
                    if (sv > 0) { sr = 0; sc = sv; }
                    else if (sv < 0) { sr = -(int64_t)sv; sc = 0; }
                    else { sr = 0; sc = 0; }
                    o->edge_Df[k] = D[lr * W + lc];
                    o->edge_S[k] = sv;
                    o->edge_start_r[k] = sr;
                    o->edge_start_c[k] = sc;
                    o->edge_Cf_olap[k] = Ct[sr * ldc + sc];
                }
            }
        }
        free(D); free(P); free(Cf); free(Df); free(wpbuf);
    }
    return failed ? -1 : 0;
}

/* _edge_starts_from_S + _build_valid_mask (Parflex.py:347-373, 582-624). */
static void build_valid_mask(oracle_result *o)
{
    const int64_t n1 = o->n1, n2 = o->n2;
    for (int64_t i = 0; i < n1; ++i) {
        for (int64_t j = 0; j < n2; ++j) {
            int64_t W = o->edge_lens[(i * n2 + j) * 2 + 0];
            int64_t R = o->edge_lens[(i * n2 + j) * 2 + 1];
            /* top edge */
            if (i == n1 - 1) {
                for (int64_t p = 0; p < W; ++p) o->valid_mask[idx4(o, i, j, 0, p)] = 1;
            } else {
                /* starts_bot_edge of tile (i+1, j): S > 0 over its top row and
                 * right column */
                int64_t aW = o->edge_lens[((i + 1) * n2 + j) * 2 + 0];
                int64_t aR = o->edge_lens[((i + 1) * n2 + j) * 2 + 1];
                for (int e = 0; e < 2; ++e) {
                    int64_t elen = e == 0 ? aW : aR;
                    for (int64_t p = 0; p < elen; ++p) {
                        int32_t v = o->edge_S[idx4(o, i + 1, j, e, p)];
                        if (v > 0 && v < W) o->valid_mask[idx4(o, i, j, 0, v)] = 1;
                    }
                }
                o->valid_mask[idx4(o, i, j, 0, 0)] = 1;
                o->valid_mask[idx4(o, i, j, 0, W - 1)] = 1;
            }
            /* right edge */
            if (j == n2 - 1) {
                for (int64_t p = 0; p < R; ++p) o->valid_mask[idx4(o, i, j, 1, p)] = 1;
            } else {
                /* starts_left_edge of tile (i, j+1): |S| for S <= 0 */
                int64_t bW = o->edge_lens[(i * n2 + j + 1) * 2 + 0];
                int64_t bR = o->edge_lens[(i * n2 + j + 1) * 2 + 1];
                for (int e = 0; e < 2; ++e) {
                    int64_t elen = e == 0 ? bW : bR;
                    for (int64_t p = 0; p < elen; ++p) {
                        int32_t v = o->edge_S[idx4(o, i, j + 1, e, p)];
                        if (v <= 0 && -(int64_t)v < R)
                            o->valid_mask[idx4(o, i, j, 1, -(int64_t)v)] = 1;
                    }
                }
                o->valid_mask[idx4(o, i, j, 1, 0)] = 1;
                o->valid_mask[idx4(o, i, j, 1, R - 1)] = 1;
            }
        }
    }
}

/* Locate global start cell (g_start_r, g_start_c) on an edge of tile
 * (pi, pj): edge 0 if it is on the tile's last row, else edge 1 if on its
 * last column, else -1 (Parflex.py:686-700, 822-839). */
static int prev_edge_slot(const oracle_result *o, int64_t pi, int64_t pj,
                          int64_t g_start_r, int64_t g_start_c,
                          int64_t *p_edge, int64_t *p_pos)
{
    int64_t s1, e1, s2, e2;
    tile_bounds(o, pi, pj, &s1, &e1, &s2, &e2);
    int64_t p_lr = g_start_r - s1, p_lc = g_start_c - s2;
    int64_t p_nrow = e1 - s1, p_ncol = e2 - s2, p_elen;
    if (p_lr == p_nrow - 1) { *p_edge = 0; *p_pos = p_lc; p_elen = p_ncol; }
    else if (p_lc == p_ncol - 1) { *p_edge = 1; *p_pos = p_lr; p_elen = p_nrow; }
    else return -1;
    if (*p_pos < 0 || *p_pos >= p_elen) return -1;
    return 0;
}

/* _nb_initialize_chunks_sparse + _nb_dp_fill_chunks_sparse
 * (Parflex.py:632-855). */
static void propagate(oracle_result *o)
{
    const int64_t n1 = o->n1, n2 = o->n2;
    double *D = o->D_prop, *Lr = o->L_prop;
    /* chunk (0, 0) */
    {
        int64_t W = o->edge_lens[0], R = o->edge_lens[1];
        for (int e = 0; e < 2; ++e) {
            int64_t elen = e == 0 ? W : R;
            for (int64_t pos = 0; pos < elen; ++pos) {
                int64_t k = idx4(o, 0, 0, e, pos);
                if (!o->valid_mask[k]) continue;
                int64_t sr = o->edge_start_r[k], sc = o->edge_start_c[k];
                int64_t lr = e == 0 ? R - 1 : pos, lc = e == 0 ? pos : W - 1;
                if (sr == 0 || sc == 0) {
                    D[k] = o->edge_Df[k];
                    Lr[k] = (double)(llabs(lr - sr) + llabs(lc - sc));
                }
            }
        }
    }
    /* first row */
    for (int64_t j = 1; j < n2; ++j) {
        int64_t W = o->edge_lens[(0 * n2 + j) * 2 + 0];
        int64_t R = o->edge_lens[(0 * n2 + j) * 2 + 1];
        int64_t pW = o->edge_lens[(0 * n2 + j - 1) * 2 + 0];
        D[idx4(o, 0, j, 0, 0)] = D[idx4(o, 0, j - 1, 0, pW - 1)];
        Lr[idx4(o, 0, j, 0, 0)] = Lr[idx4(o, 0, j - 1, 0, pW - 1)];
        for (int e = 0; e < 2; ++e) {
            int64_t elen = e == 0 ? W : R;
            for (int64_t pos = 1; pos < elen; ++pos) {
                int64_t k = idx4(o, 0, j, e, pos);
                if (!o->valid_mask[k]) continue;
                int64_t sr = o->edge_start_r[k], sc = o->edge_start_c[k];
                int64_t lr = e == 0 ? R - 1 : pos, lc = e == 0 ? pos : W - 1;
                if (sr == 0) {
                    D[k] = o->edge_Df[k];
                    Lr[k] = (double)(llabs(lr - sr) + llabs(lc - sc));
                } else if (sc == 0) {
                    int64_t s1, e1, s2, e2, pe, pp;
                    tile_bounds(o, 0, j, &s1, &e1, &s2, &e2);
                    if (prev_edge_slot(o, 0, j - 1, s1 + sr, s2, &pe, &pp)) continue;
                    double prev = D[idx4(o, 0, j - 1, pe, pp)];
                    if (!isfinite(prev)) continue;
                    D[k] = o->edge_Df[k] + prev - o->edge_Cf_olap[k];
                    Lr[k] = Lr[idx4(o, 0, j - 1, pe, pp)] +
                            (double)(llabs(lr - sr) + llabs(lc - sc));
                }
            }
        }
    }
    /* first column */
    for (int64_t i = 1; i < n1; ++i) {
        int64_t W = o->edge_lens[(i * n2 + 0) * 2 + 0];
        int64_t R = o->edge_lens[(i * n2 + 0) * 2 + 1];
        int64_t pR = o->edge_lens[((i - 1) * n2 + 0) * 2 + 1];
        D[idx4(o, i, 0, 1, 0)] = D[idx4(o, i - 1, 0, 1, pR - 1)];
        Lr[idx4(o, i, 0, 1, 0)] = Lr[idx4(o, i - 1, 0, 1, pR - 1)];
        for (int e = 0; e < 2; ++e) {
            int64_t elen = e == 0 ? W : R;
            for (int64_t pos = 1; pos < elen; ++pos) {
                int64_t k = idx4(o, i, 0, e, pos);
                if (!o->valid_mask[k]) continue;
                int64_t sr = o->edge_start_r[k], sc = o->edge_start_c[k];
                int64_t lr = e == 0 ? R - 1 : pos, lc = e == 0 ? pos : W - 1;
                if (sc == 0) {
                    D[k] = o->edge_Df[k];
                    Lr[k] = (double)(llabs(lr - sr) + llabs(lc - sc));
                } else if (sr == 0) {
                    int64_t s1, e1, s2, e2, pe, pp;
                    tile_bounds(o, i, 0, &s1, &e1, &s2, &e2);
                    if (prev_edge_slot(o, i - 1, 0, s1, s2 + sc, &pe, &pp)) continue;
                    double prev = D[idx4(o, i - 1, 0, pe, pp)];
                    if (!isfinite(prev)) continue;
                    D[k] = o->edge_Df[k] + prev - o->edge_Cf_olap[k];
                    Lr[k] = Lr[idx4(o, i - 1, 0, pe, pp)] +
                            (double)(llabs(lr - sr) + llabs(lc - sc));
                }
            }
        }
    }
    /* interior, row-major */
    for (int64_t i = 1; i < n1; ++i) {
        for (int64_t j = 1; j < n2; ++j) {
            int64_t W = o->edge_lens[(i * n2 + j) * 2 + 0];
            int64_t R = o->edge_lens[(i * n2 + j) * 2 + 1];
            for (int e = 0; e < 2; ++e) {
                int64_t elen = e == 0 ? W : R;
                for (int64_t pos = 0; pos < elen; ++pos) {
                    int64_t k = idx4(o, i, j, e, pos);
                    if (!o->valid_mask[k]) continue;
                    if (pos == 0) {
                        int64_t q;
                        if (e == 0) {
                            int64_t pW = o->edge_lens[(i * n2 + j - 1) * 2 + 0];
                            q = idx4(o, i, j - 1, 0, pW - 1);
                        } else {
                            int64_t pR = o->edge_lens[((i - 1) * n2 + j) * 2 + 1];
                            q = idx4(o, i - 1, j, 1, pR - 1);
                        }
                        if (isfinite(D[q])) { D[k] = D[q]; Lr[k] = Lr[q]; }
                        continue;
                    }
                    int64_t lr = e == 0 ? R - 1 : pos, lc = e == 0 ? pos : W - 1;
                    int64_t sr = o->edge_start_r[k], sc = o->edge_start_c[k];
                    int64_t pi, pj;
                    if (sr == 0) { pi = i - 1; pj = j; }
                    else if (sc == 0) { pi = i; pj = j - 1; }
                    else {
                        D[k] = o->edge_Df[k];
                        Lr[k] = (double)(llabs(lr - sr) + llabs(lc - sc));
                        continue;
                    }
                    int64_t s1, e1, s2, e2, pe, pp;
                    tile_bounds(o, i, j, &s1, &e1, &s2, &e2);
                    if (prev_edge_slot(o, pi, pj, s1 + sr, s2 + sc, &pe, &pp)) continue;
                    double prev = D[idx4(o, pi, pj, pe, pp)];
                    double plen = Lr[idx4(o, pi, pj, pe, pp)];
                    if (!isfinite(prev)) continue;
                    D[k] = prev + o->edge_Df[k] - o->edge_Cf_olap[k];
                    Lr[k] = plen + (double)(llabs(lr - sr) + llabs(lc - sc));
                }
            }
        }
    }
}

/* sync_tile_overlap_edges (Parflex.py:920-969), in place on D_arr/L_arr. */
static void sync_edges(oracle_result *o)
{
    const int64_t n1 = o->n1, n2 = o->n2;
    double *D = o->D_arr, *Lr = o->L_arr;
    for (int64_t i = 0; i < n1; ++i)
        for (int64_t j = 0; j + 1 < n2; ++j) {
            int64_t el = o->edge_lens[(i * n2 + j) * 2 + 0];
            if (el == 0) continue;
            int64_t a = idx4(o, i, j, 0, el - 1), b = idx4(o, i, j + 1, 0, 0);
            if (isfinite(D[a]) && !isfinite(D[b])) { D[b] = D[a]; Lr[b] = Lr[a]; }
            else if (!isfinite(D[a]) && isfinite(D[b])) { D[a] = D[b]; Lr[a] = Lr[b]; }
        }
    for (int64_t i = 0; i + 1 < n1; ++i)
        for (int64_t j = 0; j < n2; ++j) {
            int64_t el = o->edge_lens[(i * n2 + j) * 2 + 1];
            if (el == 0) continue;
            int64_t a = idx4(o, i, j, 1, el - 1), b = idx4(o, i + 1, j, 1, 0);
            if (isfinite(D[a]) && !isfinite(D[b])) { D[b] = D[a]; Lr[b] = Lr[a]; }
            else if (!isfinite(D[a]) && isfinite(D[b])) { D[a] = D[b]; Lr[a] = Lr[b]; }
        }
    for (int64_t i = 0; i < n1; ++i)
        for (int64_t j = 0; j < n2; ++j) {
            int64_t et = o->edge_lens[(i * n2 + j) * 2 + 0];
            int64_t er = o->edge_lens[(i * n2 + j) * 2 + 1];
            if (et == 0 || er == 0) continue;
            int64_t t = idx4(o, i, j, 0, et - 1), r = idx4(o, i, j, 1, er - 1);
            if (isfinite(D[t]) && !isfinite(D[r])) { D[r] = D[t]; Lr[r] = Lr[t]; }
            else if (!isfinite(D[t]) && isfinite(D[r])) { D[t] = D[r]; Lr[t] = Lr[r]; }
            else if (isfinite(D[t]) && isfinite(D[r]) && fabs(D[t] - D[r]) > 1e-10) {
                D[r] = D[t]; Lr[r] = Lr[t];
            }
        }
}

/* _nb_backtrace_within_chunk (Parflex.py:977-1012): writes global points
 * from the end cell back to the start cell, returns the count. */
int64_t oracle_backtrace_segment(const int8_t *B, int64_t nrows, int64_t ncols,
                                 const int64_t *steps, int S, int64_t start_r,
                                 int64_t start_c, int64_t end_r, int64_t end_c,
                                 int64_t gro, int64_t gco, int64_t *out)
{
    int64_t max_iters = nrows + ncols, k = 0, r = end_r, c = end_c;
    int64_t it;
    for (it = 0; it < max_iters; ++it) {
        out[2 * k] = r + gro; out[2 * k + 1] = c + gco; ++k;
        if (r == start_r && c == start_c) return k;
        int s = B[r * ncols + c];
        if (s < 0 || s >= S) {
            if (r != start_r || c != start_c) {
                out[2 * k] = start_r + gro; out[2 * k + 1] = start_c + gco; ++k;
            }
            return k;
        }
        int64_t pr = r - steps[2 * s], pc = c - steps[2 * s + 1];
        if (pr < 0 || pc < 0 || pr >= nrows || pc >= ncols) {
            if (r != start_r || c != start_c) {
                out[2 * k] = start_r + gro; out[2 * k + 1] = start_c + gco; ++k;
            }
            return k;
        }
        r = pr; c = pc;
    }
    if (r != start_r || c != start_c) {
        out[2 * k] = start_r + gro; out[2 * k + 1] = start_c + gco; ++k;
    }
    return k;
}

/* backtrace_and_stitch (Parflex.py:1032-1103).  Returns the number of
 * points written to out (K x 2, start-first order).  tiles_out (optional)
 * receives the visited (i, j, edge, idx) tuples. */
int64_t oracle_stitch(const oracle_result *o, const int64_t *steps, int S,
                      int64_t ci, int64_t cj, int64_t ce, int64_t cx,
                      int64_t *out, int64_t *tiles_out, int64_t *n_tiles)
{
    int64_t n = 0, nt = 0;
    int64_t vis[101][4];
    int64_t *seg = (int64_t *)malloc(sizeof(int64_t) * (size_t)(2 * (2 * o->L + 8)));
    for (int iter = 0; iter < 101; ++iter) {
        int dup = 0;
        for (int64_t v = 0; v < nt; ++v)
            if (vis[v][0] == ci && vis[v][1] == cj && vis[v][2] == ce && vis[v][3] == cx) dup = 1;
        if (dup) break;
        vis[nt][0] = ci; vis[nt][1] = cj; vis[nt][2] = ce; vis[nt][3] = cx; ++nt;
        if (ci < 0 || cj < 0 || ci >= o->n1 || cj >= o->n2) break;
        int64_t s1, e1, s2, e2;
        tile_bounds(o, ci, cj, &s1, &e1, &s2, &e2);
        int64_t rows = e1 - s1, cols = e2 - s2;
        int64_t er = ce == 0 ? rows - 1 : cx, ec = ce == 0 ? cx : cols - 1;
        /* S at an edge cell is the stage-1 edge start encoding */
        int32_t sv;
        if (er == rows - 1 && ce == 0) sv = o->edge_S[idx4(o, ci, cj, 0, ec)];
        else if (ec == cols - 1 && ce == 1) sv = o->edge_S[idx4(o, ci, cj, 1, er)];
        else sv = 0; /* unreachable: edge slots always address edge cells */
        int64_t sr = sv >= 0 ? 0 : -(int64_t)sv, sc = sv >= 0 ? sv : 0;
        int64_t k = oracle_backtrace_segment(o->tile_B[ci * o->n2 + cj], rows,
                                             cols, steps, S, sr, sc, er, ec,
                                             s1, s2, seg);
        for (int64_t q = 0; q < k; ++q) {
            if (n == 0 || out[2 * (n - 1)] != seg[2 * q] ||
                out[2 * (n - 1) + 1] != seg[2 * q + 1]) {
                out[2 * n] = seg[2 * q]; out[2 * n + 1] = seg[2 * q + 1]; ++n;
            }
        }
        int64_t gsr = s1 + sr, gsc = s2 + sc;
        if (gsr == 0 || gsc == 0) break;
        int corner = (sr == 0 && sc == 0);
        int64_t pi, pj, pe;
        if (corner) { pi = ci - 1; pj = cj - 1; pe = 0; }
        else if (sv >= 0) { pi = ci - 1; pj = cj; pe = 0; }
        else { pi = ci; pj = cj - 1; pe = 1; }
        if (pi < 0 || pj < 0 || pi >= o->n1 || pj >= o->n2) break;
        int64_t ps1, pe1, ps2, pe2;
        tile_bounds(o, pi, pj, &ps1, &pe1, &ps2, &pe2);
        int64_t prows = pe1 - ps1, pcols = pe2 - ps2, pidx, pmax;
        if (corner) { pidx = pcols - 1; pmax = pcols; }
        else {
            int64_t plr = gsr - ps1, plc = gsc - ps2;
            pidx = pe == 0 ? plc : plr;
            pmax = pe == 0 ? pcols : prows;
        }
        if (pidx < 0 || pidx >= pmax) break;
        ci = pi; cj = pj; ce = pe; cx = pidx;
    }
    free(seg);
    /* reverse */
    for (int64_t a = 0, b = n - 1; a < b; ++a, --b) {
        int64_t t0 = out[2 * a], t1 = out[2 * a + 1];
        out[2 * a] = out[2 * b]; out[2 * a + 1] = out[2 * b + 1];
        out[2 * b] = t0; out[2 * b + 1] = t1;
    }
    if (tiles_out) memcpy(tiles_out, vis, sizeof(int64_t) * 4 * (size_t)nt);
    if (n_tiles) *n_tiles = nt;
    return n;
}

/* _build_edge_lookups + _nb_scan_edges (Parflex.py:1110-1222). */
static void scan_edges(oracle_result *o, int64_t buf)
{
    const int64_t N = o->N, M = o->M, n1 = o->n1, n2 = o->n2, Lb = o->L;
    const double LARGE = 1e9;
    int64_t *top = (int64_t *)malloc(sizeof(int64_t) * 4 * (size_t)M);
    int64_t *right = (int64_t *)malloc(sizeof(int64_t) * 4 * (size_t)N);
    for (int64_t g = 0; g < M; ++g) top[4 * g] = -1;
    for (int64_t g = 0; g < N; ++g) right[4 * g] = -1;
    for (int64_t bi = 0; bi < n1; ++bi)
        for (int64_t bj = 0; bj < n2; ++bj) {
            int64_t s1, e1, s2, e2;
            tile_bounds(o, bi, bj, &s1, &e1, &s2, &e2);
            int64_t rows = e1 - s1, cols = e2 - s2;
            if (s1 <= N - 1 && N - 1 < e1) {
                int64_t lr = N - 1 - s1;
                for (int64_t g = s2; g < e2; ++g) {
                    if (top[4 * g] >= 0) continue;
                    int64_t lc = g - s2;
                    if (lr == rows - 1) {
                        top[4 * g] = bi; top[4 * g + 1] = bj; top[4 * g + 2] = 0; top[4 * g + 3] = lc;
                    } else if (lc == cols - 1) {
                        top[4 * g] = bi; top[4 * g + 1] = bj; top[4 * g + 2] = 1; top[4 * g + 3] = lr;
                    }
                }
            }
            if (s2 <= M - 1 && M - 1 < e2) {
                int64_t lc = M - 1 - s2;
                for (int64_t g = s1; g < e1; ++g) {
                    if (right[4 * g] >= 0) continue;
                    int64_t lr = g - s1;
                    if (lc == cols - 1) {
                        right[4 * g] = bi; right[4 * g + 1] = bj; right[4 * g + 2] = 1; right[4 * g + 3] = lr;
                    } else if (lr == rows - 1) {
                        right[4 * g] = bi; right[4 * g + 1] = bj; right[4 * g + 2] = 0; right[4 * g + 3] = lc;
                    }
                }
            }
        }
    for (int64_t g = 0; g < M; ++g) { o->top_D[g] = NAN; o->top_L[g] = 0.0; }
    for (int64_t g = 0; g < N; ++g) { o->right_D[g] = NAN; o->right_L[g] = 0.0; }
    int64_t ms = o->max_segs;
    for (int64_t q = 0; q < 2 * ms; ++q) {
        o->seg_best_norm[q] = INFINITY;
        for (int f = 0; f < 6; ++f) o->seg_best_meta[q * 6 + f] = -1;
    }
    double best = LARGE;
    o->found = 0;
    for (int f = 0; f < 6; ++f) o->best_end[f] = -1;
    for (int pass = 0; pass < 2; ++pass) {
        int64_t G = pass == 0 ? M : N;
        int64_t *lk = pass == 0 ? top : right;
        for (int64_t g = 0; g < G; ++g) {
            if (buf > 0 && g < buf) continue;
            int64_t ci = lk[4 * g], cj = lk[4 * g + 1], et = lk[4 * g + 2], ix = lk[4 * g + 3];
            if (ci < 0) continue;
            int64_t pel = o->edge_lens[(ci * n2 + cj) * 2 + et];
            if (ix < 0 || ix >= pel) continue;
            double Dv = o->D_arr[idx4(o, ci, cj, et, ix)];
            double Lv = o->L_arr[idx4(o, ci, cj, et, ix)];
            if (!isfinite(Dv) || Lv <= 0.0) continue;
            if (pass == 0 && Dv >= LARGE) continue;
            double norm = Dv / Lv;
            if (pass == 0) { o->top_D[g] = Dv; o->top_L[g] = Lv; }
            else { o->right_D[g] = Dv; o->right_L[g] = Lv; }
            int64_t grow = pass == 0 ? N - 1 : g, gcol = pass == 0 ? g : M - 1;
            if (norm < best) {
                best = norm;
                o->best_end[0] = grow; o->best_end[1] = gcol;
                o->best_end[2] = ci; o->best_end[3] = cj;
                o->best_end[4] = et; o->best_end[5] = ix;
                o->found = 1;
            }
            int64_t si = g / Lb;
            if (si < ms && norm < o->seg_best_norm[pass * ms + si]) {
                int64_t *m = &o->seg_best_meta[(pass * ms + si) * 6];
                o->seg_best_norm[pass * ms + si] = norm;
                m[0] = ci; m[1] = cj; m[2] = et; m[3] = ix; m[4] = grow; m[5] = gcol;
            }
        }
    }
    o->best_cost = best;
    free(top);
    free(right);
}

/* Full ParFlex on a host cost matrix (Parflex.py:1510-1547), keeping every
 * intermediate for the tests.  Returns 0, or -1 on allocation failure, or
 * -2 when stage 2 finds no endpoint (the reference raises ValueError). */
int oracle_parflex2(const double *C, int64_t N, int64_t M, int64_t ldc,
                    const int64_t *steps, const double *weights, int S,
                    double beta, int64_t L, int threads, int want_tile_wp,
                    int fp32, oracle_result *o)
{
    memset(o, 0, sizeof(*o));
    if (N < 2 || M < 2 || L < 2 || S < 1 || S > ORACLE_MAX_STEPS) return -3;
    o->N = N; o->M = M; o->L = L; o->hop = L - 1;
    o->n1 = (N - 1 + o->hop - 1) / o->hop;
    o->n2 = (M - 1 + o->hop - 1) / o->hop;
    const int64_t nt = o->n1 * o->n2, n4 = nt * 2 * L;
    o->edge_Df = (double *)malloc(sizeof(double) * (size_t)n4);
    o->edge_S = (int32_t *)calloc((size_t)n4, sizeof(int32_t));
    o->edge_start_r = (int64_t *)calloc((size_t)n4, sizeof(int64_t));
    o->edge_start_c = (int64_t *)calloc((size_t)n4, sizeof(int64_t));
    o->edge_Cf_olap = (double *)calloc((size_t)n4, sizeof(double));
    o->edge_lens = (int64_t *)calloc((size_t)(nt * 2), sizeof(int64_t));
    o->valid_mask = (uint8_t *)calloc((size_t)n4, 1);
    o->tile_B = (int8_t **)calloc((size_t)nt, sizeof(int8_t *));
    o->tile_best = (double *)calloc((size_t)nt, sizeof(double));
    o->tile_wp_len = (int64_t *)calloc((size_t)nt, sizeof(int64_t));
    o->D_prop = (double *)malloc(sizeof(double) * (size_t)n4);
    o->L_prop = (double *)malloc(sizeof(double) * (size_t)n4);
    o->D_arr = (double *)malloc(sizeof(double) * (size_t)n4);
    o->L_arr = (double *)malloc(sizeof(double) * (size_t)n4);
    o->top_D = (double *)malloc(sizeof(double) * (size_t)M);
    o->top_L = (double *)malloc(sizeof(double) * (size_t)M);
    o->right_D = (double *)malloc(sizeof(double) * (size_t)N);
    o->right_L = (double *)malloc(sizeof(double) * (size_t)N);
    int64_t nst = (M + L - 1) / L, nsr = (N + L - 1) / L;
    o->max_segs = nst > nsr ? nst : nsr;
    if (o->max_segs < 1) o->max_segs = 1;
    o->seg_best_norm = (double *)malloc(sizeof(double) * (size_t)(2 * o->max_segs));
    o->seg_best_meta = (int64_t *)malloc(sizeof(int64_t) * (size_t)(12 * o->max_segs));
    if (!o->edge_Df || !o->edge_S || !o->edge_start_r || !o->edge_start_c ||
        !o->edge_Cf_olap || !o->edge_lens || !o->valid_mask || !o->tile_B ||
        !o->tile_best || !o->tile_wp_len || !o->D_prop || !o->L_prop ||
        !o->D_arr || !o->L_arr || !o->top_D || !o->top_L || !o->right_D ||
        !o->right_L || !o->seg_best_norm || !o->seg_best_meta)
        return -1;
    for (int64_t q = 0; q < n4; ++q) {
        o->edge_Df[q] = INFINITY;
        o->D_prop[q] = INFINITY;
        o->L_prop[q] = INFINITY;
    }
    if (stage1(o, C, ldc, steps, weights, S, threads, want_tile_wp, fp32)) return -1;
    build_valid_mask(o);
    propagate(o);
    memcpy(o->D_arr, o->D_prop, sizeof(double) * (size_t)n4);
    memcpy(o->L_arr, o->L_prop, sizeof(double) * (size_t)n4);
    sync_edges(o);
    double mn = (double)(N < M ? N : M), mx = (double)(N < M ? M : N);
    double buffer_global = mn * (1 - (1 - beta) * mn / mx);
    scan_edges(o, (int64_t)buffer_global);
    if (!o->found) return -2;
    o->wp = (int64_t *)malloc(sizeof(int64_t) * 2 * (size_t)(101 * (2 * L + 8)));
    o->tile_order = (int64_t *)malloc(sizeof(int64_t) * 4 * 101);
    if (!o->wp || !o->tile_order) return -1;
    o->wp_len = oracle_stitch(o, steps, S, o->best_end[2], o->best_end[3],
                              o->best_end[4], o->best_end[5], o->wp,
                              o->tile_order, &o->n_stitch);
    return 0;
}

int oracle_parflex(const double *C, int64_t N, int64_t M, int64_t ldc,
                   const int64_t *steps, const double *weights, int S,
                   double beta, int64_t L, int threads, int want_tile_wp,
                   oracle_result *o)
{
    return oracle_parflex2(C, N, M, ldc, steps, weights, S, beta, L, threads,
                           want_tile_wp, 0, o);
}

/* Size of oracle_result, so the Python side can check its struct layout. */
int64_t oracle_result_size(void) { return (int64_t)sizeof(oracle_result); }

/* The cosine cost as a fixed-order chain of fused multiply-adds, the
 * definition of the device's FMA cost mode (PFX_BATCH_COST_FMA; the reference
 * forms C = 1 - F1^T F2 with a BLAS product, FlexDTW.py:213-216,
 * Parflex.py:1470, whose rounding order is the library's): for L2-normalised
 * A (d x N) and B (d x M), row-major by feature,
 *   acc = A[0][i] * B[0][j];  acc = fma(A[f][i], B[f][j], acc), f = 1..d-1;
 *   C[i][j] = 1 - acc.
 * fma() is correctly rounded (C99); nothing else is contracted
 * (-ffp-contract=off). */
void oracle_cost_fma(const double *A, const double *B, int d, int64_t N, int64_t M, double *C)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) {
        for (int64_t j = 0; j < M; ++j) {
            double acc = A[i] * B[j];
            for (int f = 1; f < d; ++f) acc = fma(A[(int64_t)f * N + i], B[(int64_t)f * M + j], acc);
            C[i * M + j] = 1.0 - acc;
        }
    }
}
