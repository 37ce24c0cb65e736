// Stage 1 (plan path): FlexDTW on every tile, FP64, two rows per lane, cost
// read from the tile-skewed layout, warps synchronised pairwise.
//
// Recurrence and tie-breaking: FlexDTW.py:326-370 (see stage1_f64.cu).
//
// Mapping.  A strip is 64 tile rows; lane i owns rows 64k+2i (A) and
// 64k+2i+1 (B) and at local step tau computes A = (64k+2i, tau-2i) and
// B = (64k+2i+1, tau-2i-1): row rho = r mod 64 sits at column tau - rho, and
// r + c = 64k + tau is the same for every cell of a warp-step.  The
// predecessors of A are lane i-1's B two steps ago ((1,1)), lane i-1's B
// three steps ago ((1,2), relayed: what this lane received one step earlier)
// and lane i-1's A three steps ago ((2,1)); those of B are this lane's own A
// two and three steps ago and again lane i-1's B three steps ago.  Two
// shuffles of (D, P) per step feed both cells, which are independent of each
// other.  mdist = (r + c) - |P| is formed in FP64 (exact: both integers).
//
// Lane 0 takes rows 64k-2 and 64k-1 (the previous strip's lane 31) from a
// per-warp shared-memory ring indexed by (strip start + column) mod RB.
// Strips start `lag` (>= 80) steps apart.  Inside a tile warps do not use CTA
// barriers: each publishes the global step it has completed (release store by
// lane 31, the ring writer) and, before a block, waits (acquire, bounded)
// until its producer has written everything the block reads and its consumer
// has read every slot the block overwrites.  A wait that runs out sets the
// status word and the CTA's abort flag; every warp then leaves the tile at its
// next wait and the CTA stops claiming tiles.
//
// Work queue.  The kernel is persistent: each CTA claims tile descriptors
// (cost slab, output addresses, shape) from a device queue with one atomic
// per tile, so the tiles of one alignment or of a whole batch of alignments
// of uneven sizes run in one launch.  Queues are ordered largest tile first.
// A CTA barrier separates consecutive tiles of a CTA (rings and progress
// words are reset there).
//
// Selection.  Every cell first takes a branch-free, division-free comparison
// of the three candidates (cross products with a 2^-48 relative margin, see
// qless_exact); cells too close to call, cells with a predecessor on row 0 /
// column 0 or outside the tile, and non-finite values go -- one uniform
// branch per warp-step -- to the exact per-lane routine, which falls back to
// IEEE division.  Only blocks touching a tile boundary ("edge" blocks) pay
// for the bounds tests and the edge-row stores.  The cost queue runs two
// steps ahead.
#include <algorithm>
#include <cooperative_groups.h>
#include <cuda/atomic>

#include "common.cuh"

#include <math_constants.h>

namespace pfx {

constexpr int kSpinLimit = 1 << 22;

// Pulls the cost of a strip's next block of steps (kBlk steps x 32 lanes,
// contiguous in the skewed slab) into L2 with one bulk prefetch, so that the
// DP's own loads, two steps ahead, hit L2 instead of HBM.  Issued by one lane;
// the range must lie inside the strip (the caller checks).
template <typename V2>
__device__ __forceinline__ void prefetch_next_block(const V2* strip, int tau_next) {
    const V2* p = strip + (int64_t)tau_next * 32;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p),
                 "r"((uint32_t)(kBlk * 32 * sizeof(V2)))
                 : "memory");
}

// IEEE arithmetic of the DP's value type (FP64 plain form, FP32 chosen form),
// rounded to nearest, never contracted.
__device__ __forceinline__ double addr(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float addr(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double mulr(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mulr(float a, float b) { return __fmul_rn(a, b); }
template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// Exact RN(b/nd) < RN(a/md) (nd, md positive integers), per lane, no warp
// collectives.  Division only when the cross products cannot decide.
__device__ __forceinline__ bool qless_exact(double b, double nd, double a, double md) {
    const double U = __dmul_rn(b, md);
    const double V = __dmul_rn(a, nd);
    const double diff = __dadd_rn(V, -U);
    const double mag = __dadd_rn(fabs(U), fabs(V));
    const double tau = __dmul_rn(mag, 0x1p-48);
    if (mag >= 0x1p-950) {
        if (diff > tau) return true;
        if (-diff > tau) return false;
    }
    return __ddiv_rn(b, nd) < __ddiv_rn(a, md);
}

// FP32 form: RN32(b/nd) < RN32(a/md).  The cross products of two FP32 values
// and two integers below 2^24 are exact in FP64, so their difference has the
// sign of the exact comparison: <= 0 decides "not less"; a relative margin of
// 2^-21 (two FP32 roundings are at most 2^-24 each) decides "less"; in
// between the two IEEE divisions decide.
__device__ __forceinline__ bool qless_exact(float b, float nd, float a, float md) {
    const double U = __dmul_rn((double)b, (double)md);
    const double V = __dmul_rn((double)a, (double)nd);
    const double diff = __dadd_rn(V, -U);
    if (diff <= 0.0) return false;
    if (diff > __dmul_rn(__dadd_rn(fabs(U), fabs(V)), 0x1p-21)) return true;
    return __fdiv_rn(b, nd) < __fdiv_rn(a, md);
}

// Exact selection of one cell with r, c >= 1 (generic steps, any position).
template <bool STD, bool ALLIN, typename T>
__device__ __forceinline__ void select_exact(const Geo& g, T w_last, int r, int c, T rc, T cval,
                                          T x1D, int x1P, T x2D, int x2P, T x3D, int x3P, T& oD,
                                          int& oP, int& code) {
    int bs = -1, bk = 0, bP = 0;
    T bA = 0, bM = 1;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        if (!STD && s >= g.S) continue;
        const int kd = STD ? s : g.kind[s];
        const bool inb = ALLIN || kd == 0 || (kd == 1 ? c >= 2 : r >= 2);
        if (!inb) continue;
        const T pD = kd == 0 ? x1D : (kd == 1 ? x2D : x3D);
        const int pP = kd == 0 ? x1P : (kd == 1 ? x2P : x3P);
        const T a = addr(pD, mulr(cval, (T)g.w[s]));
        const T md = addr(rc, -fabs((T)pP));
        const bool take = bs < 0 ? a < (T)CUDART_INF : qless_exact(a, md, bA, bM);
        if (take) {
            bs = s;
            bk = kd;
            bA = a;
            bM = md;
            bP = pP;
        }
    }
    if (bs < 0) {
        // reference: D[-1,-1] (still 0) + C * w[-1], P[-1,-1] (0), B = -1
        oD = addr((T)0, mulr(cval, w_last));
        oP = 0;
        code = 3;
    } else {
        oD = bA;
        code = bs;
        const int pr = r - (bk == 2 ? 2 : 1);
        const int pcn = c - (bk == 1 ? 2 : 1);
        oP = pr == 0 ? pcn : (pcn == 0 ? -pr : bP);
    }
}

// Steps (1,1), (1,2), (2,1): branch-free selection of one cell with r, c >= 1.
// Returns false when a comparison is too close to call or a value is not
// finite; the caller then recomputes the cell with select_exact.  EDGE adds
// the in-bounds tests of (1,2) (c >= 2) and (2,1) (r >= 2) and the start
// encoding of a predecessor on row 0 / column 0 (FlexDTW.py:365-370).
template <bool EDGE>
__device__ __forceinline__ bool select_fast_std(const Geo& g, int r, int c, double rc,
                                                double cval, double x1D, int x1P, double x2D,
                                                int x2P, double x3D, int x3P, double& oD,
                                                int& oP, int& code) {
    const double a0 = __dadd_rn(x1D, __dmul_rn(cval, g.w[0]));
    const double a1 = __dadd_rn(x2D, __dmul_rn(cval, g.w[1]));
    const double a2 = __dadd_rn(x3D, __dmul_rn(cval, g.w[2]));
    const double m0 = __dadd_rn(rc, -fabs((double)x1P));
    const double m1 = __dadd_rn(rc, -fabs((double)x2P));
    const double m2 = __dadd_rn(rc, -fabs((double)x3P));
    const bool in1 = !EDGE || c >= 2, in2 = !EDGE || r >= 2;
    const double U1 = __dmul_rn(a1, m0), V1 = __dmul_rn(a0, m1);
    const double d1 = __dadd_rn(V1, -U1);
    const double g1 = __dadd_rn(fabs(U1), fabs(V1));
    const double t1 = __dmul_rn(g1, 0x1p-48);
    const bool win1 = in1 && d1 > t1;
    const bool ok1 = !in1 || (g1 >= 0x1p-950 && (d1 > t1 || -d1 > t1));
    const double bA = win1 ? a1 : a0, bM = win1 ? m1 : m0;
    const double U2 = __dmul_rn(a2, bM), V2 = __dmul_rn(bA, m2);
    const double d2 = __dadd_rn(V2, -U2);
    const double g2 = __dadd_rn(fabs(U2), fabs(V2));
    const double t2 = __dmul_rn(g2, 0x1p-48);
    const bool win2 = in2 && d2 > t2;
    const bool ok2 = !in2 || (g2 >= 0x1p-950 && (d2 > t2 || -d2 > t2));
    oD = win2 ? a2 : bA;
    const int inh = win2 ? x3P : (win1 ? x2P : x1P);
    code = win2 ? 2 : (win1 ? 1 : 0);
    if (EDGE) {
        const int pr = r - (win2 ? 2 : 1);
        const int pcn = c - (win1 && !win2 ? 2 : 1);
        oP = pr == 0 ? pcn : (pcn == 0 ? -pr : inh);
    } else {
        oP = inh;
    }
    return a0 < CUDART_INF && ok1 && ok2;
}

// FP32 form of select_fast_std: FP32 path costs, exact FP64 cross products
// (see the FP32 qless_exact) for the two comparisons.
template <bool EDGE>
__device__ __forceinline__ bool select_fast_std(const Geo& g, int r, int c, float rc, float cval,
                                                float x1D, int x1P, float x2D, int x2P,
                                                float x3D, int x3P, float& oD, int& oP,
                                                int& code) {
    const float a0 = __fadd_rn(x1D, __fmul_rn(cval, (float)g.w[0]));
    const float a1 = __fadd_rn(x2D, __fmul_rn(cval, (float)g.w[1]));
    const float a2 = __fadd_rn(x3D, __fmul_rn(cval, (float)g.w[2]));
    const float m0 = __fadd_rn(rc, -fabsf((float)x1P));
    const float m1 = __fadd_rn(rc, -fabsf((float)x2P));
    const float m2 = __fadd_rn(rc, -fabsf((float)x3P));
    const bool in1 = !EDGE || c >= 2, in2 = !EDGE || r >= 2;
    const double U1 = __dmul_rn((double)a1, (double)m0), V1 = __dmul_rn((double)a0, (double)m1);
    const double d1 = __dadd_rn(V1, -U1);
    const double t1 = __dmul_rn(__dadd_rn(fabs(U1), fabs(V1)), 0x1p-21);
    const bool win1 = in1 && d1 > t1;
    const bool ok1 = !in1 || d1 > t1 || d1 <= 0.0;
    const float bA = win1 ? a1 : a0, bM = win1 ? m1 : m0;
    const double U2 = __dmul_rn((double)a2, (double)bM), V2 = __dmul_rn((double)bA, (double)m2);
    const double d2 = __dadd_rn(V2, -U2);
    const double t2 = __dmul_rn(__dadd_rn(fabs(U2), fabs(V2)), 0x1p-21);
    const bool win2 = in2 && d2 > t2;
    const bool ok2 = !in2 || d2 > t2 || d2 <= 0.0;
    oD = win2 ? a2 : bA;
    const int inh = win2 ? x3P : (win1 ? x2P : x1P);
    code = win2 ? 2 : (win1 ? 1 : 0);
    if (EDGE) {
        const int pr = r - (win2 ? 2 : 1);
        const int pcn = c - (win1 && !win2 ? 2 : 1);
        oP = pr == 0 ? pcn : (pcn == 0 ? -pr : inh);
    } else {
        oP = inh;
    }
    return a0 < CUDART_INF_F && a1 < CUDART_INF_F && a2 < CUDART_INF_F && ok1 && ok2;
}

template <typename T>
struct Wave {
    T aD1, aD2, aD3, bD1, bD2, xpD;  // own A outputs 1..3 steps ago, own B 1..2 ago,
    int aP1, aP2, aP3, bP1, bP2, xpP;  // lane i-1's B received one step ago
    typename Vec2<T>::type q[2];     // cost queue, step tau in slot tau & 1
};

// Per-warp rings of a strip's last two rows, [NW][RB] slots.  Slot s of a
// ring holds row 64k+63 ("B") at the strip's local step s+63 and row 64k+62
// ("A") at step s+62, the pair the next strip's lane 0 reads at once: D as
// one {B, A} vector and the start encodings as one {B, A} int2, so a read is
// two shared-memory loads and a write two stores (lane 31 writes A one step
// late, together with B).
template <typename T>
struct Rings {
    typename Vec2<T>::type* D;  // {D of row 64k+63, D of row 64k+62}
    int2* P;                    // {P of row 64k+63, P of row 64k+62}
};
template <typename T>
__host__ __device__ constexpr int ring_slot_bytes() {
    return (int)(sizeof(typename Vec2<T>::type) + sizeof(int2));
}

// rg: the CTA's rings.  A warp reads its producer's ring at rbase and
// writes its own at wbase, both with rg's layout: rg.D itself, or in a
// cluster the generic address of the other CTA's rings.  A slot is accessed
// at base + its byte offset in rg, so that the address derives from the base
// alone.  bw (when non-null) receives the block's backpointer word instead of
// the store to td.Bw.
template <typename X, typename T>
__device__ __forceinline__ X ring_at(const char* rbase, const Rings<T>& rg, const X* p) {
    return *reinterpret_cast<const X*>(
        rbase + (reinterpret_cast<const char*>(p) - reinterpret_cast<const char*>(rg.D)));
}
template <typename X, typename T>
__device__ __forceinline__ void ring_put(char* wbase, const Rings<T>& rg, const X* p, X v) {
    *reinterpret_cast<X*>(wbase + (reinterpret_cast<const char*>(p) -
                                   reinterpret_cast<const char*>(rg.D))) = v;
}
template <typename T>
__device__ __forceinline__ typename Vec2<T>::type make_v2(T x, T y) {
    typename Vec2<T>::type v;
    v.x = x;
    v.y = y;
    return v;
}

// PUSH: the ring is written at wbase (generic address, a cluster peer's
// shared memory possibly); otherwise straight into this CTA's rings.
template <bool EDGE, bool STD, bool PUSH, typename T>
__device__ __forceinline__ void run_block(const Geo& g, Wave<T>& st, const Rings<T>& rg,
                                          const char* rbase, char* wbase,
                                          const typename Vec2<T>::type* __restrict__ Cs,
                                          int span, int tau0, int k, int R, int W, int lane,
                                          int prev_base, int mine_base, int rmask, int Tb,
                                          int lag, const TileDesc& td, int nP,
                                          uint2* bw = nullptr) {
    using V2 = typename Vec2<T>::type;
    const unsigned F = 0xffffffffu;
    const T w_last = (T)(g.S == 1 ? g.w[0] : (g.S == 2 ? g.w[1] : g.w[2]));
    const int rA = 64 * k + 2 * lane, rB = rA + 1;
    uint32_t bitsA = 0, bitsB = 0;
    const T rc0 = (T)(64 * k + tau0);
#pragma unroll 1
    for (int tq = 0; tq < kBlk; tq += 2) {
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int t = tq + u;
            const int tau = tau0 + t;
            const T rc = addr(rc0, (T)t);
            const V2 cc = st.q[u & 1];
            if (tau + 2 < span) st.q[u & 1] = __ldcs(Cs + (int64_t)(tau + 2) * 32);
            T x1D = __shfl_up_sync(F, st.bD2, 1);
            int x1P = __shfl_up_sync(F, st.bP2, 1);
            T x3D = __shfl_up_sync(F, st.aD3, 1);
            int x3P = __shfl_up_sync(F, st.aP3, 1);
            {
                // every lane reads the same slot (a broadcast); lane 0 keeps it
                const int rs = prev_base + ((Tb + t - lag - 1) & rmask);
                const V2 rD = ring_at(rbase, rg, rg.D + rs);
                const int2 rP = ring_at(rbase, rg, rg.P + rs);
                if (lane == 0) {
                    x1D = rD.x;
                    x1P = rP.x;
                    x3D = rD.y;
                    x3P = rP.y;
                }
            }
            const T x2D = st.xpD;
            const int x2P = st.xpP;
            const int cA = tau - 2 * lane, cB = cA - 1;
            T oAD, oBD;
            int oAP, oBP, codeA, codeB;
            bool actA = true, actB = true;
            bool okA, okB;
            if (STD) {
                okA = select_fast_std<EDGE>(g, rA, cA, rc, cc.x, x1D, x1P, x2D, x2P, x3D, x3P, oAD,
                                            oAP, codeA);
                okB = select_fast_std<EDGE>(g, rB, cB, rc, cc.y, st.aD2, st.aP2, st.aD3, st.aP3,
                                            x2D, x2P, oBD, oBP, codeB);
            } else {
                okA = okB = false;
            }
            if (EDGE) {
                actA = rA < R && cA >= 0 && cA < W;
                actB = rB < R && cB >= 0 && cB < W;
                // boundary cells are set below; absent cells are zeroed
                okA = !actA || rA == 0 || cA == 0 || okA;
                okB = !actB || cB == 0 || okB;
            }
            if (__any_sync(F, !(okA && okB))) {
                if (!okA) {
                    if (rA == 0 || cA == 0) {
                        oAD = cc.x; oAP = 0; codeA = 0;
                    } else {
                        select_exact<STD, !EDGE>(g, w_last, rA, cA, rc, cc.x, x1D, x1P, x2D, x2P,
                                                 x3D, x3P, oAD, oAP, codeA);
                    }
                }
                if (!okB) {
                    if (cB == 0) {
                        oBD = cc.y; oBP = 0; codeB = 0;
                    } else {
                        select_exact<STD, !EDGE>(g, w_last, rB, cB, rc, cc.y, st.aD2, st.aP2,
                                                 st.aD3, st.aP3, x2D, x2P, oBD, oBP, codeB);
                    }
                }
            }
            if (EDGE) {
                double* eD = td.eD;
                int32_t* eP = td.eP;
                if (actA && (rA == 0 || cA == 0)) { oAD = cc.x; oAP = 0; codeA = 0; }
                if (actB && cB == 0) { oBD = cc.y; oBP = 0; codeB = 0; }
                if (!actA) { oAD = 0; oAP = 0; codeA = 0; }
                if (!actB) { oBD = 0; oBP = 0; codeB = 0; }
                // edges are FP64 for stage 2 (exact widening in the FP32 form)
                if (actA && rA == R - 1) { eD[cA] = (double)oAD; eP[cA] = oAP; }
                if (actB && rB == R - 1) { eD[cB] = (double)oBD; eP[cB] = oBP; }
                if (actA && cA == W - 1) { eD[td.L + rA] = (double)oAD; eP[td.L + rA] = oAP; }
                if (actB && cB == W - 1) { eD[td.L + rB] = (double)oBD; eP[td.L + rB] = oBP; }
            }
            if (lane == 31 && actB) {
                // B of this step and A of the previous one (the same column,
                // active whenever B is): slot (step - 63)
                const int ws = mine_base + ((Tb + t - 63) & rmask);
                if (PUSH) {
                    ring_put(wbase, rg, rg.D + ws, make_v2<T>(oBD, st.aD1));
                    ring_put(wbase, rg, rg.P + ws, make_int2(oBP, st.aP1));
                } else {
                    rg.D[ws] = make_v2<T>(oBD, st.aD1);
                    rg.P[ws] = make_int2(oBP, st.aP1);
                }
            }
            bitsA |= (uint32_t)codeA << (2 * t);
            bitsB |= (uint32_t)codeB << (2 * t);
            st.aD3 = st.aD2; st.aP3 = st.aP2;
            st.aD2 = st.aD1; st.aP2 = st.aP1;
            st.aD1 = oAD;    st.aP1 = oAP;
            st.bD2 = st.bD1; st.bP2 = st.bP1;
            st.bD1 = oBD;    st.bP1 = oBP;
            st.xpD = x1D;    st.xpP = x1P;
        }
    }
    if (bw) {
        *bw = make_uint2(bitsA, bitsB);
    } else if (rA < R) {
        uint2* Bt = reinterpret_cast<uint2*>(td.Bw);
        Bt[((int64_t)k * nP + (tau0 >> 4)) * 32 + lane] = make_uint2(bitsA, bitsB);
    }
}

// Division-free decision of "the new candidate's quotient is strictly below
// the incumbent's", RN(a_new / m_new) < RN(a_inc / m_inc) with positive
// integer-valued m, for the FP64 form.  Returns whether the cross products
// decide it (else the caller divides); `win` is the answer when they do.
//   U = RN(a_new * m_inc), V = RN(a_inc * m_new), d = RN(V - U) and the
//   threshold t = RN(|U| * 2^-46 + 2^-900) (one FMA).  d's error is below
//   2^-52 (|U| + |V|) (plus 2^-1073 where a product is subnormal).
//   * |V| <= 3 |U|: t >= 2^-48 (|U| + |V|) + 2^-900 exceeds that error by a
//     factor of 16, so |d| > t fixes the sign of the exact a_inc m_new -
//     a_new m_inc and leaves a relative gap > 2^-49 between the exact
//     quotients: their roundings cannot meet.
//   * |V| > 3 |U|: the exact difference has V's sign and |V| / 2 or more of
//     magnitude, the same conclusion.
//   |d| > t needs max(|U|, |V|) > 2^-901: no quotient is subnormal.  A NaN
//   or infinite product never decides (every comparison with it is false or
//   t is infinite).
__device__ __forceinline__ bool decide_quot(double a_new, double m_new, double a_inc,
                                            double m_inc, bool& win) {
    const double U = __dmul_rn(a_new, m_inc);
    const double V = __dmul_rn(a_inc, m_new);
    const double d = __dadd_rn(V, -U);
    const double t = __fma_rn(fabs(U), 0x1p-46, 0x1p-900);
    win = d > t;
    return win || -d > t;
}
// FP32 form: the cross products of FP32 values and integers below 2^24 are
// exact in FP64 (see the FP32 qless_exact): d <= 0 decides "not below", a
// relative margin of 2^-21 decides "below".
__device__ __forceinline__ bool decide_quot(float a_new, float m_new, float a_inc, float m_inc,
                                            bool& win) {
    const double U = __dmul_rn((double)a_new, (double)m_inc);
    const double V = __dmul_rn((double)a_inc, (double)m_new);
    const double d = __dadd_rn(V, -U);
    win = d > __dmul_rn(__dadd_rn(fabs(U), fabs(V)), 0x1p-21);
    return win || d <= 0.0;
}
__device__ __forceinline__ bool finite_first(double a0, double, double) { return a0 < CUDART_INF; }
__device__ __forceinline__ bool finite_first(float a0, float a1, float a2) {
    return a0 < CUDART_INF_F && a1 < CUDART_INF_F && a2 < CUDART_INF_F;
}

// Steps (1,1), (1,2), (2,1) at a cell with every predecessor inside the tile
// and r, c >= 2, mdists given: the selection of select_fast_std<false>.
template <typename T>
__device__ __forceinline__ bool select_std_m(T cval, T w0, T w1, T w2, T x1D, int x1P, T m0,
                                             T x2D, int x2P, T m1, T x3D, int x3P, T m2, T& oD,
                                             int& oP, int& code) {
    const T a0 = addr(x1D, mulr(cval, w0));
    const T a1 = addr(x2D, mulr(cval, w1));
    const T a2 = addr(x3D, mulr(cval, w2));
    bool win1, win2;
    const bool ok1 = decide_quot(a1, m1, a0, m0, win1);
    const T bA = win1 ? a1 : a0, bM = win1 ? m1 : m0;
    const bool ok2 = decide_quot(a2, m2, bA, bM, win2);
    oD = win2 ? a2 : bA;
    oP = win2 ? x3P : (win1 ? x2P : x1P);
    code = win2 ? 2 : (win1 ? 1 : 0);
    return finite_first(a0, a1, a2) && ok1 && ok2;
}

// Exact selection of the fast block's undecided cells (rare), by value.
template <typename T>
struct SelOut {
    T d;
    int p, code;
};
template <typename T>
__device__ __forceinline__ SelOut<T> select_exact_std_call(T w0, T w1, T w2, int r, int c, T rc,
                                                        T cval, T x1D, int x1P, T x2D, int x2P,
                                                        T x3D, int x3P) {
    Geo g;
    g.S = 3;
    g.kind[0] = 0;
    g.kind[1] = 1;
    g.kind[2] = 2;
    g.w[0] = (double)w0;
    g.w[1] = (double)w1;
    g.w[2] = (double)w2;
    SelOut<T> o;
    select_exact<true, true>(g, w2, r, c, rc, cval, x1D, x1P, x2D, x2P, x3D, x3P, o.d, o.p,
                             o.code);
    return o;
}

// A block of 16 steps of the standard step set in which every cell of the
// strip is inside the tile with r, c >= 2 and off the tile's last row and
// column (the caller's "interior" test).  Same results as
// run_block<false, true, PUSH, T>, with fewer instructions per step:
//  * no bounds tests, no edge stores, and no guard on the cost loads (the
//    block ends at least 17 steps before the strip's span);
//  * mdist of a predecessor that the previous step also used is that step's
//    mdist + 1 (r + c grows by one per step), and B's (2,1) predecessor is
//    A's (1,2) one, so a step converts three start encodings, not six;
//  * ring slots are read and written as {B, A} pairs (two shared-memory
//    loads per step, two stores by lane 31);
//  * the FP64 decision margin is one FMA (decide_quot).
// The loop is unrolled two steps deep only: steps t and t+1 are independent
// (each reads outputs of two steps back), and a small loop body stays in the
// instruction cache (a 16-step unroll, or a second copy of the body, each
// measured slower).
//
// MASK (a run-time flag, so that one copy of the loop body serves both: a
// second inlined copy measured slower): the same path for a block of strip
// k >= 1 at tau0 >= 80 (every cell at r >= 64, c >= 18, so every
// predecessor of a cell inside the tile is inside too) that reaches the
// tile's last column or its last row, or lies partly outside the tile (the
// right end of a strip, the last strip): cells outside the tile (r >= R or
// c >= W) are set to 0 and never call for the exact routine, cells on the
// last row / column store their edge values, and the cost loads stop at the
// strip's span.  Same results as run_block<true, true, PUSH, T>.
template <bool PUSH, typename T>
__device__ __forceinline__ void run_block_std(const Geo& g, Wave<T>& st, const Rings<T>& rg,
                                              char* wbase,
                                              const typename Vec2<T>::type* __restrict__ Cs,
                                              int tau0, int k, int lane, int prev_base,
                                              int mine_base, int rmask, int Tb, int lag,
                                              const TileDesc& td, int nP, uint2* bw,
                                              const bool MASK, int R, int W, int span) {
    using V2 = typename Vec2<T>::type;
    const unsigned F = 0xffffffffu;
    const T w0 = (T)g.w[0], w1 = (T)g.w[1], w2 = (T)g.w[2];
    const int rA = 64 * k + 2 * lane, rB = rA + 1;
    const T rc0 = (T)(64 * k + tau0);
    // mdist of A's and B's (1,2) predecessors at the next step
    T m1A_next = addr(rc0, -fabs((T)st.xpP));
    T m1B_next = addr(rc0, -fabs((T)st.aP3));
    uint32_t bitsA = 0, bitsB = 0;
    const V2* cp = Cs + (int64_t)(tau0 + 2) * 32;  // the cost two steps ahead
    const V2* rD = rg.D + prev_base;
    const int2* rP = rg.P + prev_base;
    const int rs0 = Tb - lag - 1;
#pragma unroll 1
    for (int tq = 0; tq < kBlk; tq += 2) {
        const T rcq = addr(rc0, (T)tq);
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int t = tq + u;
            const T rc = addr(rcq, (T)u);
            const V2 cc = st.q[u & 1];
            if (!MASK || tau0 + t + 2 < span) st.q[u & 1] = __ldcs(cp + (int64_t)t * 32);
            const int rs = (rs0 + t) & rmask;
            const V2 ringD = rD[rs];  // every lane reads the same slot; lane 0 keeps it
            const int2 ringP = rP[rs];
            T x1D = __shfl_up_sync(F, st.bD2, 1);
            int x1P = __shfl_up_sync(F, st.bP2, 1);
            T x3D = __shfl_up_sync(F, st.aD3, 1);
            int x3P = __shfl_up_sync(F, st.aP3, 1);
            x1D = lane == 0 ? ringD.x : x1D;
            x1P = lane == 0 ? ringP.x : x1P;
            x3D = lane == 0 ? ringD.y : x3D;
            x3P = lane == 0 ? ringP.y : x3P;
            const T x2D = st.xpD;
            const int x2P = st.xpP;
            const T m0A = addr(rc, -fabs((T)x1P));
            const T m1A = m1A_next;
            const T m2A = addr(rc, -fabs((T)x3P));
            const T m0B = addr(rc, -fabs((T)st.aP2));
            const T m1B = m1B_next;
            m1A_next = addr(m0A, (T)1);
            m1B_next = addr(m0B, (T)1);
            T oAD, oBD;
            int oAP, oBP, codeA, codeB;
            bool okA = select_std_m<T>(cc.x, w0, w1, w2, x1D, x1P, m0A, x2D, x2P, m1A, x3D,
                                       x3P, m2A, oAD, oAP, codeA);
            bool okB = select_std_m<T>(cc.y, w0, w1, w2, st.aD2, st.aP2, m0B, st.aD3, st.aP3,
                                       m1B, x2D, x2P, m1A, oBD, oBP, codeB);
            bool actA = true, actB = true;
            if (MASK) {
                const int cA = tau0 + t - 2 * lane;
                actA = rA < R && cA < W;
                actB = rB < R && cA - 1 < W;
                okA = okA || !actA;
                okB = okB || !actB;
            }
            if (__any_sync(F, !(okA && okB))) {
                const int cA = tau0 + t - 2 * lane;
                if (!okA) {
                    const SelOut<T> o = select_exact_std_call<T>(w0, w1, w2, rA, cA, rc, cc.x,
                                                                 x1D, x1P, x2D, x2P, x3D, x3P);
                    oAD = o.d;
                    oAP = o.p;
                    codeA = o.code;
                }
                if (!okB) {
                    const SelOut<T> o = select_exact_std_call<T>(w0, w1, w2, rB, cA - 1, rc,
                                                                 cc.y, st.aD2, st.aP2, st.aD3,
                                                                 st.aP3, x2D, x2P);
                    oBD = o.d;
                    oBP = o.p;
                    codeB = o.code;
                }
            }
            if (MASK) {
                const int cA = tau0 + t - 2 * lane, cB = cA - 1;
                if (!actA) { oAD = 0; oAP = 0; codeA = 0; }
                if (!actB) { oBD = 0; oBP = 0; codeB = 0; }
                // edges are FP64 for stage 2 (exact widening in the FP32 form)
                double* eD = td.eD;
                int32_t* eP = td.eP;
                if (actA && rA == R - 1) { eD[cA] = (double)oAD; eP[cA] = oAP; }
                if (actB && rB == R - 1) { eD[cB] = (double)oBD; eP[cB] = oBP; }
                if (actA && cA == W - 1) { eD[td.L + rA] = (double)oAD; eP[td.L + rA] = oAP; }
                if (actB && cB == W - 1) { eD[td.L + rB] = (double)oBD; eP[td.L + rB] = oBP; }
            }
            if (lane == 31 && actB) {
                // B of this step and A of the previous one: slot (step - 63)
                const int ws = mine_base + ((Tb + t - 63) & rmask);
                if (PUSH) {
                    ring_put(wbase, rg, rg.D + ws, make_v2<T>(oBD, st.aD1));
                    ring_put(wbase, rg, rg.P + ws, make_int2(oBP, st.aP1));
                } else {
                    rg.D[ws] = make_v2<T>(oBD, st.aD1);
                    rg.P[ws] = make_int2(oBP, st.aP1);
                }
            }
            bitsA |= (uint32_t)codeA << (2 * t);
            bitsB |= (uint32_t)codeB << (2 * t);
            st.aD3 = st.aD2; st.aP3 = st.aP2;
            st.aD2 = st.aD1; st.aP2 = st.aP1;
            st.aD1 = oAD;    st.aP1 = oAP;
            st.bD2 = st.bD1; st.bP2 = st.bP1;
            st.bD1 = oBD;    st.bP1 = oBP;
            st.xpD = x1D;    st.xpP = x1P;
        }
    }
    if (bw) {
        *bw = make_uint2(bitsA, bitsB);
    } else if (!MASK || rA < R) {
        uint2* Bt = reinterpret_cast<uint2*>(td.Bw);
        Bt[((int64_t)k * nP + (tau0 >> 4)) * 32 + lane] = make_uint2(bitsA, bitsB);
    }
}

// Bounded wait until progress word *p reaches target; gives up early when
// another warp of the CTA has already given up (*abort set).
__device__ __forceinline__ bool wait_progress(int* p, int target, const volatile int* abort) {
    cuda::atomic_ref<int, cuda::thread_scope_block> a(*p);
    for (int it = 0; it < kSpinLimit; ++it) {
        if (a.load(cuda::memory_order_acquire) >= target) return true;
        if (*abort) return false;
        __nanosleep(32);
    }
    return false;
}

// Ring length: the largest power of two whose rings fit the shared-memory
// limit, capped at the first power of two >= lag + 64 (enough slack that the
// pairwise waits rarely block); at least lag - 29 (one block of slack).
// `vbytes` is the size of a DP value (8 for FP64, 4 for FP32).
__host__ __device__ inline int ring_len(int lag, int nw, int smem_limit, int vbytes) {
    int cap = 16;
    while (cap * 2 <= lag + 64) cap *= 2;
    if (cap < lag + 64) cap *= 2;
    int fit = 16;
    const int per = nw * (2 * vbytes + (int)sizeof(int2));
    while ((fit * 2) * per + nw * (int)sizeof(int) <= smem_limit) fit *= 2;
    const int rb = cap < fit ? cap : fit;
    return rb >= lag - 29 ? rb : 0;
}

// ---------------------------------------------------------------------------
// In-kernel cost (CostGen).  The CTA that claimed a tile first writes the
// tile's tile-skewed FP64 cost into its own slot, then runs the DP on it, so
// a batch needs one slot per resident CTA instead of a slab per tile, and
// CTAs in their cost phase (FP64-pipe bound) share the SMs with CTAs in their
// DP phase (issue and latency bound).  Mapping and summation order are those
// of k_cost_skew (layout.cu): units of two strips x (NW * 32) steps; the
// unit's column features are staged in shared memory split by column parity
// and the two strips' row features as one (A, B) pair per lane; each warp
// computes 32 steps of both strips in passes of 8 steps, in which 9 column
// vectors serve 32 cells of a lane.  Cells outside the tile are 0, as in the
// slabs.  The staging reuses the rings' shared memory, which holds nothing
// between tiles.
constexpr int kGenCV = 4;

__host__ __device__ constexpr int gen_window(int nw) { return nw * 32 + 66; }
__host__ __device__ inline size_t gen_smem_bytes(int nw, int d) {
    return (size_t)d * (gen_window(nw) + 128) * sizeof(double);
}

template <int NW, int DMAX>
__device__ __forceinline__ void gen_tile_cost(const double* __restrict__ fa, int lda,
                                           const double* __restrict__ fb, int ldb, int R, int W,
                                           int d, double* __restrict__ slab) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int U = NW * 32;
    constexpr int CX = gen_window(NW), CH = CX / 2;
    double* sB = reinterpret_cast<double*>(smem_raw);  // [d][2][CH]
    double* sA = sB + d * CX;                          // [d][2 strips][64 rows]
    const double2* sA2 = reinterpret_cast<const double2*>(sA);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int span = ceil_div32(W + kStripRows - 1, kBlk) * kBlk;
    const int nS = ceil_div32(R, kStripRows);
    const int nchunk = ceil_div32(span, U);
    for (int kk = 0; 2 * kk < nS; ++kk) {
        const bool two = 2 * kk + 1 < nS;
        const int rA0 = 128 * kk + 2 * lane, rB0 = rA0 + 1, rA1 = rA0 + 64, rB1 = rA1 + 1;
        double2* out0 = reinterpret_cast<double2*>(slab) + (int64_t)(2 * kk) * span * 32 + lane;
        double2* out1 = out0 + (int64_t)span * 32;
        for (int ch = 0; ch < nchunk; ++ch) {
            const int ts = ch * U;
            __syncthreads();  // every warp is done with the previous unit's features
            // the unit's features, as asynchronous copies all in flight at once
            // (zero-filled outside the tile)
            for (int q = threadIdx.x; q < d * CX; q += NW * 32) {
                const int f = q / CX, x = q - f * CX;
                const int c = ts - 64 + x;
                const bool in = c >= 0 && c < W;
                cp_async8(sB + (f * 2 + (x & 1)) * CH + (x >> 1),
                          in ? fb + (int64_t)f * ldb + c : fb, in);
            }
            if (ch == 0)
                for (int q = threadIdx.x; q < d * 128; q += NW * 32) {
                    const int f = q >> 7, r = 128 * kk + (q & 127);
                    cp_async8(sA + q, r < R ? fa + (int64_t)f * lda + r : fa, r < R);
                }
            cp_async_wait_all();
            __syncthreads();
#pragma unroll 1
            for (int blk = 0; blk < 32 / kGenCV; ++blk) {
                const int t0 = ts + 32 * warp + kGenCV * blk;  // warp-uniform
                if (t0 >= span) break;
                // b[j] holds window column x = xA0 - 1 + j, xA0 = t0 - ts + 64 - 2 lane
                const int h0 = ((t0 - ts + 64) >> 1) - lane;
                double accA0[kGenCV], accB0[kGenCV], accA1[kGenCV], accB1[kGenCV];
#pragma unroll
                for (int f = 0; f < DMAX; ++f) {
                    if (f >= d) break;
                    const double* se = sB + (f * 2) * CH;  // even x
                    const double* so = se + CH;             // odd x
                    double b[kGenCV + 1];
#pragma unroll
                    for (int j = 0; j <= kGenCV; ++j)
                        b[j] = (j & 1) ? se[h0 + (j >> 1)] : so[h0 - 1 + (j >> 1)];
                    const double2 a0 = sA2[(f * 2) * 32 + lane], a1 = sA2[(f * 2 + 1) * 32 + lane];
#pragma unroll
                    for (int v = 0; v < kGenCV; ++v) {
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
#pragma unroll
                for (int v = 0; v < kGenCV; ++v) {
                    const int tau = t0 + v;
                    if (tau < span) {
                        const int cA = tau - 2 * lane, cB = cA - 1;
                        const bool inA = cA >= 0 && cA < W, inB = cB >= 0 && cB < W;
                        out0[(int64_t)tau * 32] =
                            make_double2((rA0 < R && inA) ? __dsub_rn(1.0, accA0[v]) : 0.0,
                                         (rB0 < R && inB) ? __dsub_rn(1.0, accB0[v]) : 0.0);
                        if (two)
                            out1[(int64_t)tau * 32] =
                                make_double2((rA1 < R && inA) ? __dsub_rn(1.0, accA1[v]) : 0.0,
                                             (rB1 < R && inB) ? __dsub_rn(1.0, accB1[v]) : 0.0);
                    }
                }
            }
        }
    }
    __syncthreads();  // the slot holds the whole tile before any warp's DP reads it
}

template <int NW, bool STD, typename T, bool GEN = false>
__global__ void __launch_bounds__(NW * 32, 16 / NW)
    k_stage1_v3(const TileDesc* __restrict__ descs, const int ntiles_max,
                const int* __restrict__ ntiles_dev, int* __restrict__ head, const Geo g,
                int32_t* __restrict__ status, const int RB, const CostGen gen) {
    using V2 = typename Vec2<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Rings<T> rg;
    rg.D = reinterpret_cast<V2*>(smem_raw);
    rg.P = reinterpret_cast<int2*>(rg.D + NW * RB);
    int* prog = reinterpret_cast<int*>(rg.P + NW * RB);
    __shared__ TileDesc td;
    __shared__ Sched2 s_sc;  // schedule of the current tile (read from smem, not held in registers)
    __shared__ int s_item, s_abort, s_ttot;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int prevw = (warp + NW - 1) % NW, nextw = (warp + 1) % NW;
    const int ntiles = ntiles_dev ? min(*ntiles_dev, ntiles_max) : ntiles_max;
    if (GEN && (int)blockIdx.x >= gen.nslots) return;  // no cost slot (the launch prevents it)
    if (threadIdx.x == 0) s_abort = 0;
    cuda::atomic_ref<int, cuda::thread_scope_block> my_prog(prog[warp]);
    for (;;) {
        if (threadIdx.x == 0) {
            const int it = atomicAdd(head, 1);
            s_item = it;
            if (it < ntiles) {
                td = descs[it];
                s_sc = make_sched2(td.R, td.W, NW);
                s_ttot = (s_sc.nS - 1) * s_sc.lag + s_sc.span;
            }
        }
        if (!GEN && threadIdx.x < NW) prog[threadIdx.x] = 0;
        __syncthreads();
        if (s_item >= ntiles || s_abort) return;
        if constexpr (GEN) {
            // the tile's cost into this CTA's slot (through the rings' shared
            // memory, so the progress words are reset afterwards)
            double* slot = gen.slots + (int64_t)blockIdx.x * gen.stride;
            if (gen.d <= 12)
                gen_tile_cost<NW, 12>(td.fa, td.lda, td.fb, td.ldb, td.R, td.W, gen.d, slot);
            else
                gen_tile_cost<NW, kGenMaxD>(td.fa, td.lda, td.fb, td.ldb, td.R, td.W, gen.d,
                                            slot);
            if (threadIdx.x < NW) prog[threadIdx.x] = 0;
        }
        {
            // edge rows past the tile's extent stay +inf / 0 (the DP writes the rest)
            double* eD = td.eD;
            int32_t* eP = td.eP;
            for (int i = threadIdx.x; i < 2 * td.L; i += NW * 32) {
                eD[i] = CUDART_INF;
                eP[i] = 0;
            }
        }
        __syncthreads();
        const int32_t R = td.R, W = td.W;
        const Sched2& sc = s_sc;
        const int lag = sc.lag;
        const int Ttot = s_ttot;
        const V2* Ct =
            GEN ? reinterpret_cast<const V2*>(gen.slots + (int64_t)blockIdx.x * gen.stride)
                : reinterpret_cast<const V2*>(td.Csk);

        Wave<T> st;
        st.aD1 = st.aD2 = st.aD3 = st.bD1 = st.bD2 = st.xpD = 0;
        st.aP1 = st.aP2 = st.aP3 = st.bP1 = st.bP2 = st.xpP = 0;
#pragma unroll
        for (int q = 0; q < 2; ++q) st.q[q].x = st.q[q].y = 0;

        for (int Tb = 0; Tb < Ttot; Tb += kBlk) {
            int k = -1;
            if (Tb >= warp * lag) {
                const int j = (Tb - warp * lag) / (NW * lag);
                const int kk = warp + j * NW;
                if (kk < sc.nS && Tb < kk * lag + sc.span) k = kk;
            }
            if (k >= 0) {
                int failed = 0;
                if (lane == 0) {
                    // producer (strip k-1) has written every ring slot this block reads
                    if (k >= 1 && !wait_progress(prog + prevw, Tb - lag + 78, &s_abort)) failed = 1;
                    // consumer (strip k+1) has read every slot this block overwrites
                    if (!failed && k + 1 < sc.nS &&
                        !wait_progress(prog + nextw, Tb + lag - RB - 45, &s_abort))
                        failed = 1;
                    if (failed) {
                        if (status) atomicExch(status, kStatusWaitTimeout);
                        s_abort = 1;
                    }
                }
                if (__shfl_sync(0xffffffffu, failed, 0)) break;  // to the tile barrier
                const int tau0 = Tb - k * lag;
                const V2* Cs = Ct + (int64_t)k * sc.span * 32 + lane;
                if (lane == 0 && tau0 + 2 * kBlk <= sc.span)
                    prefetch_next_block(Ct + (int64_t)k * sc.span * 32, tau0 + kBlk);
                if (tau0 == 0) {
#pragma unroll
                    for (int q = 0; q < 2; ++q) st.q[q] = __ldcs(Cs + q * 32);
                }
                const bool lean = k >= 1 && tau0 >= 80;
                const bool interior = lean && k <= sc.nS - 2 && tau0 + 17 <= W;
                if (STD && lean) {
                    run_block_std<false, T>(g, st, rg, reinterpret_cast<char*>(rg.D), Cs, tau0,
                                            k, lane, prevw * RB, warp * RB, RB - 1, Tb, lag, td,
                                            sc.nP, nullptr, !interior, R, W, sc.span);
                } else if (!STD && interior) {
                    run_block<false, STD, false>(g, st, rg, reinterpret_cast<const char*>(rg.D),
                                                 reinterpret_cast<char*>(rg.D), Cs, sc.span, tau0,
                                                 k, R, W, lane, prevw * RB, warp * RB, RB - 1, Tb,
                                                 lag, td, sc.nP);
                } else
                    run_block<true, STD, false>(g, st, rg, reinterpret_cast<const char*>(rg.D),
                                         reinterpret_cast<char*>(rg.D), Cs,
                                         sc.span, tau0, k, R, W, lane,
                                         prevw * RB, warp * RB, RB - 1, Tb, lag, td, sc.nP);
            }
            __syncwarp();
            if (lane == 31) my_prog.store(Tb + kBlk, cuda::memory_order_release);
        }
        __syncthreads();  // every warp is done with this tile's rings and descriptor
    }
}

// ---------------------------------------------------------------------------
// One tile on a cluster of two CTAs (16 warps each): 32 warps share the strip
// pipeline of a tile, so a tile takes about (nS - 1 + 32) / 32 strip times
// instead of (nS - 1 + 16) / 16.  For alignments with fewer tiles than SMs.
// Virtual warp v = 16 * rank + warp takes strips v, v + 32, ...; strip k + 1
// reads strip k's last rows from a ring in its own CTA's shared memory.
// Where producer and consumer sit in different CTAs (v = 15 -> 16 or
// 31 -> 0) the producer writes that ring into the consumer's CTA
// (distributed shared memory, posted stores off the dependency chain), and
// the pairwise progress words are read and written at cluster scope.
// Rank 0 claims the tiles; three cluster barriers per tile (claim, set-up,
// end), which every thread of both CTAs reaches on every path: waits are
// bounded and a warp that gives up goes on to the tile's end barrier.
constexpr int kClW = 16;   // warps per CTA
constexpr int kClN = 2;    // CTAs per cluster

__device__ __forceinline__ int ld_acquire_cluster(const int* p) {
    int v;
    asm volatile("ld.acquire.cluster.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_cluster(int* p, int v) {
    asm volatile("st.release.cluster.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ bool wait_progress_cl(const int* p, int target,
                                                 const volatile int* abort) {
    for (int it = 0; it < kSpinLimit; ++it) {
        if (ld_acquire_cluster(p) >= target) return true;
        if (*abort) return false;
        __nanosleep(32);
    }
    return false;
}

template <bool STD, typename T>
__global__ void __launch_bounds__(kClW * 32, 1)
    k_stage1_cl(const TileDesc* __restrict__ descs, const int ntiles, int* __restrict__ head,
                const Geo g, int32_t* __restrict__ status, const int RB) {
    using V2 = typename Vec2<T>::type;
    constexpr int NWT = kClW * kClN;
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Rings<T> rg;  // this CTA's rings
    rg.D = reinterpret_cast<V2*>(smem_raw);
    rg.P = reinterpret_cast<int2*>(rg.D + kClW * RB);
    // progress words: [w] warp w's; [kClW] the other CTA's last warp's (this
    // CTA's warp 0 waits on it); [kClW + 1] the other CTA's warp 0's (this
    // CTA's last warp waits on it) -- written by the other CTA, polled here
    int* prog = reinterpret_cast<int*>(rg.P + kClW * RB);
    __shared__ TileDesc td;
    __shared__ Sched2 s_sc;
    __shared__ int s_item, s_abort, s_ttot;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int vw = rank * kClW + warp;
    const int pv = (vw + NWT - 1) % NWT, nv = (vw + 1) % NWT;
    // the producer's rings (generic address, this CTA's or the peer's)
    // a warp writes its ring into its consumer's CTA (posted stores, off the
    // dependency chain) and reads its producer's ring from its own CTA: ring
    // region w of a CTA is written by warp w of the CTA that feeds it (its own
    // warp w, or for w = kClW - 1 the other CTA's last warp)
    const char* rbase = reinterpret_cast<const char*>(rg.D);
    char* wbase = reinterpret_cast<char*>(cl.map_shared_rank(rg.D, nv / kClW));
    // cluster scope only where the neighbour is in the other CTA
    const bool prev_remote = pv / kClW != rank, next_remote = nv / kClW != rank;
    const bool read_remotely = warp == 0 || warp == kClW - 1;  // my progress word
    int* rprog = cl.map_shared_rank(prog, 1 - rank);  // the other CTA's words
    if (threadIdx.x == 0) s_abort = 0;
    cl.sync();  // both CTAs run before any access to the other's shared memory
    for (;;) {
        if (rank == 0 && threadIdx.x == 0) {
            const int* peer_abort = cl.map_shared_rank(&s_abort, 1);
            const int it = (s_abort || *peer_abort) ? ntiles : atomicAdd(head, 1);
            s_item = it;
            *cl.map_shared_rank(&s_item, 1) = it;
        }
        cl.sync();  // the claimed tile reaches both CTAs
        if (s_item >= ntiles) return;  // both CTAs, nothing remote after the barrier
        if (threadIdx.x == 0) {
            td = descs[s_item];
            s_sc = make_sched2(td.R, td.W, NWT);
            s_ttot = (s_sc.nS - 1) * s_sc.lag + s_sc.span;
        }
        if (threadIdx.x < kClW + 2) prog[threadIdx.x] = 0;
        __syncthreads();
        if (rank == 0) {
            // edge rows past the tile's extent stay +inf / 0 (the DP writes the rest)
            double* eD = td.eD;
            int32_t* eP = td.eP;
            for (int i = threadIdx.x; i < 2 * td.L; i += kClW * 32) {
                eD[i] = CUDART_INF;
                eP[i] = 0;
            }
        }
        cl.sync();  // progress words reset and edges filled in both CTAs
        const int32_t R = td.R, W = td.W;
        const Sched2& sc = s_sc;
        const int lag = sc.lag;
        const int Ttot = s_ttot;
        const V2* Ct = reinterpret_cast<const V2*>(td.Csk);

        Wave<T> st;
        st.aD1 = st.aD2 = st.aD3 = st.bD1 = st.bD2 = st.xpD = 0;
        st.aP1 = st.aP2 = st.aP3 = st.bP1 = st.bP2 = st.xpP = 0;
#pragma unroll
        for (int q = 0; q < 2; ++q) st.q[q].x = st.q[q].y = 0;

        for (int Tb = 0; Tb < Ttot; Tb += kBlk) {
            int k = -1;
            uint2 bw = make_uint2(0u, 0u);
            if (Tb >= vw * lag) {
                const int j = (Tb - vw * lag) / (NWT * lag);
                const int kk = vw + j * NWT;
                if (kk < sc.nS && Tb < kk * lag + sc.span) k = kk;
            }
            if (k >= 0) {
                int failed = 0;
                if (lane == 0) {
                    // producer (strip k-1) has written every ring slot this block reads
                    if (k >= 1 &&
                        !(prev_remote
                              ? wait_progress_cl(prog + kClW, Tb - lag + 78, &s_abort)
                              : wait_progress(prog + pv % kClW, Tb - lag + 78, &s_abort)))
                        failed = 1;
                    // consumer (strip k+1) has read every slot this block overwrites
                    if (!failed && k + 1 < sc.nS &&
                        !(next_remote
                              ? wait_progress_cl(prog + kClW + 1, Tb + lag - RB - 45, &s_abort)
                              : wait_progress(prog + nv % kClW, Tb + lag - RB - 45, &s_abort)))
                        failed = 1;
                    if (failed) {
                        if (status) atomicExch(status, kStatusWaitTimeout);
                        s_abort = 1;
                    }
                }
                if (__shfl_sync(0xffffffffu, failed, 0)) break;  // to the tile's end barrier
                const int tau0 = Tb - k * lag;
                const V2* Cs = Ct + (int64_t)k * sc.span * 32 + lane;
                if (lane == 0 && tau0 + 2 * kBlk <= sc.span)
                    prefetch_next_block(Ct + (int64_t)k * sc.span * 32, tau0 + kBlk);
                if (tau0 == 0) {
#pragma unroll
                    for (int q = 0; q < 2; ++q) st.q[q] = __ldcs(Cs + q * 32);
                }
                const bool lean = k >= 1 && tau0 >= 80;
                const bool interior = lean && k <= sc.nS - 2 && tau0 + 17 <= W;
                if (STD && lean)
                    run_block_std<true, T>(g, st, rg, wbase, Cs, tau0, k, lane,
                                           (pv % kClW) * RB, warp * RB, RB - 1, Tb, lag, td,
                                           sc.nP, &bw, !interior, R, W, sc.span);
                else if (!STD && interior)
                    run_block<false, STD, true>(g, st, rg, rbase, wbase, Cs, sc.span, tau0, k, R,
                                                W, lane, (pv % kClW) * RB, warp * RB, RB - 1, Tb,
                                                lag, td, sc.nP, &bw);
                else
                    run_block<true, STD, true>(g, st, rg, rbase, wbase, Cs, sc.span, tau0, k, R, W,
                                         lane,
                                         (pv % kClW) * RB, warp * RB, RB - 1, Tb, lag, td,
                                         sc.nP, &bw);
            }
            __syncwarp();
            // publish first: the backpointer store below is nobody's dependency
            if (lane == 31) {
                if (read_remotely) {
                    // also into the other CTA's copy, so that its reader polls locally
                    st_release_cluster(prog + warp, Tb + kBlk);
                    st_release_cluster(rprog + (warp == 0 ? kClW + 1 : kClW), Tb + kBlk);
                } else {
                    cuda::atomic_ref<int, cuda::thread_scope_block> a(prog[warp]);
                    a.store(Tb + kBlk, cuda::memory_order_release);
                }
            }
            if (k >= 0 && 64 * k + 2 * lane < R) {
                uint2* Bt = reinterpret_cast<uint2*>(td.Bw);
                Bt[((int64_t)k * sc.nP + ((Tb - k * lag) >> 4)) * 32 + lane] = bw;
            }
        }
        cl.sync();  // every warp of both CTAs is done with this tile's rings
    }
}

static int smem_optin() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v;
}

static int smem_per_sm() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    return v;
}

// Shared memory budget per CTA when 16/NW CTAs share an SM.
static int cta_budget(int nw) {
    const int per_cta = smem_per_sm() / (16 / nw) - 2048;  // static smem and reserve
    const int optin = smem_optin();
    return per_cta < optin ? per_cta : optin;
}

static size_t smem_bytes(int32_t L, int nw, int smem_limit, int vbytes) {
    const Sched2 s = make_sched2(L, L, nw);
    const int rb = ring_len(s.lag, nw, smem_limit, vbytes);
    if (rb == 0) return (size_t)1 << 30;  // does not fit
    return (size_t)nw * rb * (2 * vbytes + sizeof(int2)) + nw * sizeof(int);
}

int stage1_queue_warps(int ntiles, int32_t L, int num_sms) {
    // fewer warps per tile fill the strip pipeline better (utilisation ~
    // strips / (strips - 1 + warps)) but need several tiles per SM; the
    // FP64 rings are the larger, so they decide what fits
    if ((int64_t)ntiles >= 4LL * num_sms && smem_bytes(L, 4, cta_budget(4), 8) < (1u << 30))
        return 4;
    if ((int64_t)ntiles >= 2LL * num_sms && smem_bytes(L, 8, cta_budget(8), 8) < (1u << 30))
        return 8;
    return smem_bytes(L, 16, cta_budget(16), 8) < (1u << 30) ? 16 : 0;
}

// Dynamic shared memory of the queue kernel: the rings, or the in-kernel
// cost's staging (gen_d > 0) where that is larger.
static size_t queue_smem(int32_t L, int nw, int vbytes, int gen_d) {
    const size_t ring = smem_bytes(L, nw, cta_budget(nw), vbytes);
    const size_t gen = gen_d > 0 ? gen_smem_bytes(nw, gen_d) : 0;
    return ring > gen ? ring : gen;
}

// CTAs of the queue kernel resident at once on this device (its grid size
// for a long queue), or 0 when it does not fit.
template <int NW, bool STD, typename T, bool GEN>
static int queue_resident(const Geo& g, int gen_d, size_t* smem_out) {
    const size_t smem = queue_smem(g.L, NW, (int)sizeof(T), gen_d);
    if (smem >= ((size_t)1 << 30) || smem > (size_t)cta_budget(NW)) return 0;
    auto kern = k_stage1_v3<NW, STD, T, GEN>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return 0;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NW * 32, smem) !=
        cudaSuccess)
        return 0;
    if (smem_out) *smem_out = smem;
    return sms * (per_sm < 1 ? 1 : per_sm);
}

template <int NW, bool STD, typename T, bool GEN>
static cudaError_t launch_q_t(const TileDesc* descs, int ntiles, const int* ntiles_dev, int* head,
                              const Geo& g, int32_t* status, cudaStream_t st,
                              const CostGen& gen) {
    const int limit = cta_budget(NW);
    const Sched2 s = make_sched2(g.L, g.L, NW);
    const int rb = ring_len(s.lag, NW, limit, (int)sizeof(T));
    if (rb == 0) return cudaErrorInvalidValue;
    size_t smem = 0;
    const int resident = queue_resident<NW, STD, T, GEN>(g, GEN ? gen.d : 0, &smem);
    if (resident <= 0) return cudaErrorInvalidValue;
    // with the in-kernel cost every CTA needs a cost slot of its own
    if (GEN && gen.nslots < std::min(resident, ntiles)) return cudaErrorInvalidValue;
    const int grid = std::min(resident, ntiles);
    if (grid <= 0) return cudaSuccess;
    k_stage1_v3<NW, STD, T, GEN>
        <<<grid, NW * 32, smem, st>>>(descs, ntiles, ntiles_dev, head, g, status, rb, gen);
    count_launches(1);
    return cudaGetLastError();
}

template <bool STD, typename T>
static cudaError_t launch_cl_t(const TileDesc* descs, int ntiles, int* head, const Geo& g,
                               int32_t* status, cudaStream_t st) {
    const int limit = cta_budget(kClW);
    const Sched2 s = make_sched2(g.L, g.L, kClW * kClN);
    const int rb = ring_len(s.lag, kClW, limit, (int)sizeof(T));
    if (rb == 0) return cudaErrorInvalidValue;
    const size_t smem =
        (size_t)kClW * rb * ring_slot_bytes<T>() + (kClW + 2) * sizeof(int);
    auto kern = k_stage1_cl<STD, T>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClN;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(kClW * 32);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(kClN * (unsigned)ntiles);
    int maxc = 0;
    e = cudaOccupancyMaxActiveClusters(&maxc, kern, &cfg);
    if (e != cudaSuccess) return e;
    if (maxc < 1) return cudaErrorInvalidConfiguration;
    const int nc = ntiles < maxc ? ntiles : maxc;
    if (nc <= 0) return cudaSuccess;
    cfg.gridDim = dim3(kClN * (unsigned)nc);
    e = cudaLaunchKernelEx(&cfg, kern, descs, ntiles, head, g, status, rb);
    count_launches(1);
    return e;
}

template <bool STD, typename T>
static int cl_max_t(const Geo& g) {
    const int limit = cta_budget(kClW);
    const Sched2 s = make_sched2(g.L, g.L, kClW * kClN);
    const int rb = ring_len(s.lag, kClW, limit, (int)sizeof(T));
    if (rb == 0) return 0;
    const size_t smem =
        (size_t)kClW * rb * ring_slot_bytes<T>() + (kClW + 2) * sizeof(int);
    auto kern = k_stage1_cl<STD, T>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return 0;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClN;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(kClW * 32);
    cfg.dynamicSmemBytes = smem;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(kClN);
    int maxc = 0;
    if (cudaOccupancyMaxActiveClusters(&maxc, kern, &cfg) != cudaSuccess) return 0;
    return maxc;
}

int stage1_cluster_max(const Geo& g, bool fp32) {
    const bool std_steps = g.S == 3 && g.kind[0] == 0 && g.kind[1] == 1 && g.kind[2] == 2;
    if (fp32) return std_steps ? cl_max_t<true, float>(g) : cl_max_t<false, float>(g);
    return std_steps ? cl_max_t<true, double>(g) : cl_max_t<false, double>(g);
}

cudaError_t launch_stage1_cluster(const TileDesc* descs, int ntiles, int* head, const Geo& g,
                                  int32_t* status, bool fp32, cudaStream_t st) {
    const bool std_steps = g.S == 3 && g.kind[0] == 0 && g.kind[1] == 1 && g.kind[2] == 2;
    if (fp32)
        return std_steps ? launch_cl_t<true, float>(descs, ntiles, head, g, status, st)
                         : launch_cl_t<false, float>(descs, ntiles, head, g, status, st);
    return std_steps ? launch_cl_t<true, double>(descs, ntiles, head, g, status, st)
                     : launch_cl_t<false, double>(descs, ntiles, head, g, status, st);
}

template <typename T, bool GEN>
static cudaError_t launch_q_type(const TileDesc* descs, int ntiles, const int* nd, int* head,
                                 const Geo& g, int32_t* status, int nw, cudaStream_t st,
                                 const CostGen& gen) {
    const bool std_steps = g.S == 3 && g.kind[0] == 0 && g.kind[1] == 1 && g.kind[2] == 2;
    switch (nw) {
        case 4:
            return std_steps
                       ? launch_q_t<4, true, T, GEN>(descs, ntiles, nd, head, g, status, st, gen)
                       : launch_q_t<4, false, T, GEN>(descs, ntiles, nd, head, g, status, st, gen);
        case 8:
            return std_steps
                       ? launch_q_t<8, true, T, GEN>(descs, ntiles, nd, head, g, status, st, gen)
                       : launch_q_t<8, false, T, GEN>(descs, ntiles, nd, head, g, status, st, gen);
        default:
            return std_steps
                       ? launch_q_t<16, true, T, GEN>(descs, ntiles, nd, head, g, status, st, gen)
                       : launch_q_t<16, false, T, GEN>(descs, ntiles, nd, head, g, status, st,
                                                       gen);
    }
}

cudaError_t launch_stage1_queue(const TileDesc* descs, int ntiles, const int* ntiles_dev,
                                int* head, const Geo& g, int32_t* status, int nw, bool fp32,
                                cudaStream_t st, const CostGen* gen) {
    const CostGen off{nullptr, 0, 0, 0};
    if (gen && gen->d > 0) {
        if (fp32 || gen->d > kGenMaxD || !gen->slots) return cudaErrorInvalidValue;
        return launch_q_type<double, true>(descs, ntiles, ntiles_dev, head, g, status, nw, st,
                                           *gen);
    }
    return fp32 ? launch_q_type<float, false>(descs, ntiles, ntiles_dev, head, g, status, nw, st,
                                              off)
                : launch_q_type<double, false>(descs, ntiles, ntiles_dev, head, g, status, nw,
                                               st, off);
}

int stage1_gen_slots(const Geo& g, int nw, int d) {
    if (d < 1 || d > kGenMaxD) return 0;
    const bool std_steps = g.S == 3 && g.kind[0] == 0 && g.kind[1] == 1 && g.kind[2] == 2;
    switch (nw) {
        case 4:
            return std_steps ? queue_resident<4, true, double, true>(g, d, nullptr)
                             : queue_resident<4, false, double, true>(g, d, nullptr);
        case 8:
            return std_steps ? queue_resident<8, true, double, true>(g, d, nullptr)
                             : queue_resident<8, false, double, true>(g, d, nullptr);
        case 16:
            return std_steps ? queue_resident<16, true, double, true>(g, d, nullptr)
                             : queue_resident<16, false, double, true>(g, d, nullptr);
        default:
            return 0;
    }
}

// Order-preserving compaction of a tile queue by a tile mask (one CTA: a
// block-wide prefix count per chunk of 1024 descriptors).
__global__ void __launch_bounds__(1024) k_compact_descs(const TileDesc* __restrict__ in, int n,
                                                        const uint8_t* __restrict__ mask,
                                                        TileDesc* __restrict__ out,
                                                        int* __restrict__ count) {
    __shared__ int warp_sums[32];
    __shared__ int base;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c0 = 0; c0 < n; c0 += 1024) {
        const int i = c0 + (int)threadIdx.x;
        const bool keep = i < n && mask[in[i].tile];
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        const int before = __popc(bal & ((1u << lane) - 1u));
        if (lane == 0) warp_sums[warp] = __popc(bal);
        __syncthreads();
        int off = 0;
        for (int w = 0; w < warp; ++w) off += warp_sums[w];
        if (keep) out[base + off + before] = in[i];
        __syncthreads();
        if (threadIdx.x == 0) {
            int tot = 0;
            for (int w = 0; w < 32; ++w) tot += warp_sums[w];
            base += tot;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = base;
}

__global__ void k_mask_slots(const uint8_t* __restrict__ mask, int n, int32_t* __restrict__ slot) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) slot[t] = mask[t] ? t : -1;
}

cudaError_t launch_mask_slots(const uint8_t* mask, int n, int32_t* slot, cudaStream_t st) {
    k_mask_slots<<<(n + 255) / 256, 256, 0, st>>>(mask, n, slot);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_compact_descs(const TileDesc* in, int n, const uint8_t* mask, TileDesc* out,
                                 int* count, cudaStream_t st) {
    k_compact_descs<<<1, 1024, 0, st>>>(in, n, mask, out, count);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace pfx
