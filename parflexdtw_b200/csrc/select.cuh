// Exact FlexDTW step selection shared by the stage-1 kernels.
#pragma once
#include <math_constants.h>

#include "common.cuh"

namespace pfx {

// Exact test of RN(b / nd) < RN(a / md) for positive integer-valued nd, md
// (the reference compares the rounded quotients pathcost / mdist with a
// strict <).  Common case without division: the cross products
// U = RN(b*md) and V = RN(a*nd) each carry a relative error below 2^-53, so
// when they differ by more than 2^-48 (|U| + |V|) the exact quotients differ
// by more than 16 ulps in the same direction and their roundings cannot
// coincide.  Everything else -- near ties, zeros and tiny values, infinities
// and NaN -- takes the two IEEE divisions, so the outcome always equals the
// reference's.
__device__ __forceinline__ bool quot_less(double b, double nd, double a, double md) {
    const double U = __dmul_rn(b, md);
    const double V = __dmul_rn(a, nd);
    const double diff = __dadd_rn(V, -U);
    const double mag = __dadd_rn(fabs(U), fabs(V));
    const double tau = __dmul_rn(mag, 0x1p-48);
    if (mag >= 0x1p-950) {  // false for NaN
        if (diff > tau) return true;
        if (-diff > tau) return false;
    }
    return __ddiv_rn(b, nd) < __ddiv_rn(a, md);
}

// Step selection of one interior cell (r, c >= 1), FlexDTW.py:338-370.
// Candidates in the caller's step order; the first in-bounds candidate whose
// quotient is below +inf becomes the incumbent (the reference starts from
// mincost = inf), later ones replace it only on a strictly smaller quotient.
// STD: the steps are (1,1), (1,2), (2,1) in that order (compile-time kinds).
// ALLIN: the caller guarantees r >= 2 and c >= 2 (every predecessor exists).
template <bool STD, bool ALLIN>
__device__ __forceinline__ void select_step(const Geo& g, double w_last, int r, int c, double cval,
                                            double x1D, int x1P, double x2D, int x2P, double x3D,
                                            int x3P, double& oD, int& oP, int& code) {
    const int rc = r + c;
    int bs = -1, bk = 0, bPP = 0;
    double bA = 0.0, bM = 1.0;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        if (!STD && s >= g.S) continue;
        const int kd = STD ? s : g.kind[s];
        const bool inb = ALLIN || kd == 0 || (kd == 1 ? c >= 2 : r >= 2);
        if (!inb) continue;
        const double pD = kd == 0 ? x1D : (kd == 1 ? x2D : x3D);
        const int pP = kd == 0 ? x1P : (kd == 1 ? x2P : x3P);
        const double a = __dadd_rn(pD, __dmul_rn(cval, g.w[s]));
        const double md = (double)(rc - abs(pP));
        const bool take = bs < 0 ? (a < CUDART_INF) : quot_less(a, md, bA, bM);
        if (take) {
            bs = s;
            bk = kd;
            bA = a;
            bM = md;
            bPP = pP;
        }
    }
    if (bs < 0) {
        // reference: D[-1,-1] (still 0) + C * w[-1], P[-1,-1] (0), B = -1
        oD = __dadd_rn(0.0, __dmul_rn(cval, w_last));
        oP = 0;
        code = 3;
    } else {
        oD = bA;
        code = bs;
        const int pr = r - (bk == 2 ? 2 : 1);
        const int pcn = c - (bk == 1 ? 2 : 1);
        oP = pr == 0 ? pcn : (pcn == 0 ? -pr : bPP);
    }
}

}  // namespace pfx
