/* sg_line.cuh -- one SOGRAND component decode per warp.
 *
 * Restates SOGRAND_bitSO + sogrand_main_logic
 * (SOGRAND_C/cubic_decoder_final.c:521-746) for n = 16, k = 8, even = 0,
 * as warp-cooperative code:
 *   - lanes 0..15 own the 16 positions of the line for the set-up (hard
 *     decision, |LLR|, JacLog terms, sort, IC, per-position PM increments and
 *     syndrome columns) and for the soft output;
 *   - the guess loop runs 32 consecutive patterns of the enumeration order
 *     at once, one per lane: each lane forms its pattern's path metric and
 *     syndrome and evaluates exp(-PM); a ballot finds the codewords; the
 *     running P_notGuess is then advanced in enumeration order, and the list
 *     is updated at each codeword in that order, so the guess count T and
 *     every floating-point sum match the sequential reference exactly.
 * All floating-point operations that the reference performs are issued as
 * separately rounded IEEE operations (the file is built with -fmad=false);
 * exp/log are sg_exp/sg_log.
 */
#pragma once
#include <stdint.h>
#include "sg_enum.h"
#include "sg_math.h"

#define SG_FULL 0xffffffffu

struct SgLineParams {
    int32_t L;
    uint32_t tmax;     /* Tmax clamped to 2^32-1 (T never exceeds 65536) */
    double thres;
};

/* Per-warp shared scratch of one line decode. */
struct SgWarpScratch {
    double delta[16];   /* JacLog(|L|) - JacLog(-|L|) per sorted position */
    double qa[16];      /* values for the tie-exact sort */
    double elist[8];    /* exp(-PM) of the listed codewords */
    uint32_t cmask[8];  /* listed codewords, bit i = position i */
    int32_t perm[16];   /* sorted rank -> position */
    uint32_t hs[16];    /* syndrome column of each sorted position */
};

__constant__ uint8_t c_hcol[16];
__constant__ uint8_t c_prow[8];
__constant__ uint8_t c_ptab[256];

/* (int32_t) of a double as x86-64 cvttsd2si computes it: NaN and values
 * outside int32 give INT32_MIN (the reference casts round(...) at :621). */
__device__ __forceinline__ int32_t sg_cvt_i32(double v)
{
    if (!(v > -2147483649.0 && v < 2147483648.0))
        return INT32_MIN;
    return (int32_t)v;
}

/* Exact restatement of the reference's recursive quicksort (:763) on 16
 * values with an explicit stack.  The two partitions are disjoint, so the
 * processing order of the stack does not change the result.  Run by one
 * lane, only when the line has tied reliabilities (a rank sort orders ties
 * differently). */
__device__ __noinline__ void sg_quicksort16(double* a, int32_t* perm)
{
    int32_t st_off[32], st_n[32];
    int sp = 0;
    st_off[sp] = 0;
    st_n[sp] = 16;
    sp++;
    while (sp > 0) {
        sp--;
        int32_t off = st_off[sp], n = st_n[sp];
        if (n < 2)
            continue;
        double* x = a + off;
        int32_t* pm = perm + off;
        double p = x[n / 2];
        int32_t i = 0, j = n - 1;
        while (i <= j) {
            while (x[i] < p)
                i++;
            while (x[j] > p)
                j--;
            if (i <= j) {
                double t = x[i];
                x[i] = x[j];
                x[j] = t;
                int32_t tt = pm[i];
                pm[i] = pm[j];
                pm[j] = tt;
                i++;
                j--;
            }
        }
        if (j > 0 && sp < 32) {
            st_off[sp] = off;
            st_n[sp] = j + 1;
            sp++;
        }
        if (i < n && sp < 32) {
            st_off[sp] = off + i;
            st_n[sp] = n - i;
            sp++;
        }
    }
}

struct SgLineResult {
    double lapp;      /* lanes 0..15 */
    double le;        /* lanes 0..15 */
    uint32_t hdword;  /* bit i = hard decision of L_APP at position i (all lanes) */
    uint32_t T;       /* guesses (all lanes) */
    int32_t ncw;      /* codewords found (all lanes) */
};

/* Decode one line.  llr: this lane's input LLR (lanes 0..15; others
 * ignored).  enum_tabs: SG_ENUM_NTAB tables of SG_ENUM_LEN entries.
 * etab/ltab: shared-memory copies of the exp/log tables. */
__device__ __forceinline__ SgLineResult sg_decode_line(double llr, const SgLineParams& lp,
                                                        const uint32_t* __restrict__ enum_tabs,
                                                        const double* etab, const double* ltab,
                                                        SgWarpScratch* ws)
{
    const int lane = threadIdx.x & 31;
    const bool act = lane < 16;
    if (!act)
        llr = 1.0;
    const double a = fabs(llr);
    /* HardDec (:758): 1 unless llr > 0 */
    const uint32_t hdm = __ballot_sync(SG_FULL, act && !(llr > 0.0)) & 0xffffu;
    /* JacLog(-|L_i|) for getPM_HD (:617, :764) */
    const double jn = act ? sg_jaclog(-a, etab, ltab) : 0.0;
    double pmhd = 0.0;
#pragma unroll
    for (int i = 0; i < 16; i++)
        pmhd = __dadd_rn(pmhd, __shfl_sync(SG_FULL, jn, i));

    /* QuickSort of |L| ascending (:618) */
    int lt = 0, eq = 0;
#pragma unroll
    for (int j = 0; j < 16; j++) {
        const double aj = __shfl_sync(SG_FULL, a, j);
        lt += (aj < a);
        eq += (aj == a) && (j != lane);
    }
    /* ties (and NaN, which no comparison orders) take the exact quicksort */
    if (!__any_sync(SG_FULL, act && (eq > 0 || a != a))) {
        if (act)
            ws->perm[lt] = lane;
    } else {
        if (act) {
            ws->qa[lane] = a;
            ws->perm[lane] = lane;
        }
        __syncwarp();
        if (lane == 0)
            sg_quicksort16(ws->qa, ws->perm);
    }
    __syncwarp();
    const int src = act ? ws->perm[lane] : 0;
    const double as = __shfl_sync(SG_FULL, a, src);

    /* IC (:619-622): beta = (|L|_(7) - |L|_(0)) / 7, IC = max(round(.), 0) */
    const double a0 = __shfl_sync(SG_FULL, as, 0);
    const double a7 = __shfl_sync(SG_FULL, as, 7);
    const double beta = __ddiv_rn(__dsub_rn(a7, a0), 7.0);
    int32_t ic = sg_cvt_i32(round(__dsub_rn(__ddiv_rn(a0, beta), 1.0)));
    if (ic < 0)
        ic = 0;
    const int itab = ic < SG_ENUM_IC_CANON ? ic : SG_ENUM_IC_CANON;

    /* PM increment of each sorted position (getPM, :765) and its syndrome */
    const double jn_src = __shfl_sync(SG_FULL, jn, src);
    if (act) {
        ws->delta[lane] = __dsub_rn(sg_jaclog(as, etab, ltab), jn_src);
        ws->hs[lane] = c_hcol[src];
    }
    uint32_t s0 = 0;
#pragma unroll
    for (int i = 0; i < 16; i++)
        if ((hdm >> i) & 1u)
            s0 ^= c_hcol[i];
    __syncwarp();

    /* Guess loop (:624-744) */
    const uint32_t* tab = enum_tabs + (size_t)itab * SG_ENUM_LEN;
    double P = 1.0;   /* P_notGuess */
    double pnl = 0.0; /* pNL of the last getLConf */
    int32_t curl = 0;
    uint32_t T = 0;
    bool done = false;
    for (uint32_t base = 0; !done; base += 32) {
        const uint32_t t = base + lane;
        const bool valid = t < SG_ENUM_LEN;
        const uint32_t ent = valid ? __ldg(tab + t) : 0u;
        /* T < Tmax is checked before each new logistic weight (:652) */
        const uint32_t cut = __ballot_sync(SG_FULL, valid && (ent & SG_ENUM_GS) && t > 0 && t >= lp.tmax);
        uint32_t lim = __ballot_sync(SG_FULL, valid);
        if (cut)
            lim &= (1u << (__ffs(cut) - 1)) - 1u;
        const int nv = __popc(lim);
        uint32_t m = ent & 0xffffu;
        double pm = pmhd;
        uint32_t syn = s0;
        while (m) {
            const int r = __ffs(m) - 1;
            pm = __dadd_rn(pm, ws->delta[r]);
            syn ^= ws->hs[r];
            m &= m - 1u;
        }
        const double e = sg_exp(-pm, etab);
        const uint32_t hits = __ballot_sync(SG_FULL, syn == 0u) & lim;
        for (int j = 0; j < nv; j++) {
            const double ej = __shfl_sync(SG_FULL, e, j);
            P = __dsub_rn(P, ej);
            if ((hits >> j) & 1u) {
                /* list insertion and getLConf (:674-686, :767-774) */
                const uint32_t mj = __shfl_sync(SG_FULL, ent, j) & 0xffffu;
                uint32_t cm = hdm;
                for (uint32_t mm = mj; mm; mm &= mm - 1u)
                    cm ^= 1u << ws->perm[__ffs(mm) - 1];
                __syncwarp();
                if (lane == 0) {
                    ws->elist[curl] = ej;
                    ws->cmask[curl] = cm;
                }
                __syncwarp();
                double ppos = 0.0;
                for (int i = 0; i <= curl; i++)
                    ppos = __dadd_rn(ppos, ws->elist[i]);
                const double pneg = __dmul_rn(0x1p-8, P); /* 2^-(n-k) * P_notGuess */
                pnl = pneg;
                const double den = __dadd_rn(ppos, pneg);
                const double conf = (den > 1e-40) ? __ddiv_rn(ppos, den) : 1.0;
                curl++;
                if (conf > lp.thres || curl == lp.L) {
                    T = base + (uint32_t)j + 1u;
                    done = true;
                    break;
                }
            }
        }
        if (!done) {
            T = base + (uint32_t)nv;
            if (nv < 32)
                done = true;
        }
    }

    /* Soft output (:536-577) */
    SgLineResult res;
    res.T = T;
    res.ncw = curl;
    double lapp, le;
    if (curl == 0) {
        lapp = llr;
        le = 0.0;
    } else {
        const double pnlc = fmax(pnl, 1e-40);
        double pp1 = __ddiv_rn(1.0, __dadd_rn(1.0, sg_exp(llr, etab)));
        double pp0 = __dsub_rn(1.0, pp1);
        pp1 = fmin(fmax(pp1, 1e-40), 1.0);
        pp0 = fmin(fmax(pp0, 1e-40), 1.0);
        double p1 = 0.0, p0 = 0.0;
        for (int j = 0; j < curl; j++) {
            const double c = (double)((ws->cmask[j] >> lane) & 1u);
            const double pj = ws->elist[j];
            p1 = __dadd_rn(p1, __dmul_rn(c, pj));
            p0 = __dadd_rn(p0, __dmul_rn(__dsub_rn(1.0, c), pj));
        }
        p0 = __dadd_rn(p0, __dmul_rn(pnlc, pp0));
        p1 = __dadd_rn(p1, __dmul_rn(pnlc, pp1));
        lapp = __dsub_rn(sg_log(fmax(p0, 1e-40), ltab), sg_log(fmax(p1, 1e-40), ltab));
        le = __dsub_rn(lapp, llr);
    }
    res.lapp = lapp;
    res.le = le;
    res.hdword = __ballot_sync(SG_FULL, act && !(lapp > 0.0)) & 0xffffu;
    __syncwarp();
    return res;
}
