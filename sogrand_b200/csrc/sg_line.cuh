/* sg_line.cuh -- one SOGRAND component decode per warp.
 *
 * Restates SOGRAND_bitSO + sogrand_main_logic
 * (SOGRAND_C/cubic_decoder_final.c:521-746) for n = 16, k = 8, even = 0,
 * as warp-cooperative code with results bit-identical to the sequential
 * reference (given the same exp/log):
 *
 *  set-up   lanes 0..15 own the 16 positions: hard decision, |LLR|,
 *           JacLog terms, the sort (rank sort, or the reference's exact
 *           quicksort when magnitudes tie), IC, the PM increment and
 *           syndrome column of each sorted position.  From these the warp
 *           builds per-line tables:
 *             A[lo]     PM_HD + the increments of the bits of lo, added in
 *                       ascending order -- exactly the prefix of getPM's
 *                       sequential sum (:765) over the 8 least reliable
 *                       positions;
 *             synlo/hi  syndrome of each byte of a pattern (ParityCheck,
 *                       :748-755, is linear), the hard decision's own
 *                       syndrome folded into synlo.
 *  guesses  32*G consecutive patterns of the order table per step, G per
 *           lane: PM = A[lo] + increments of the high bits (ascending),
 *           syndrome = synlo[lo] ^ synhi[hi], e = exp(-PM).
 *  P_notGuess  the reference subtracts e of every guess in order (:626,
 *           :672, :712).  Within one binade [2^E, 2^(E+1)) every difference
 *           rounds to the grid u = 2^(E-52), so fl(P - e) = u*round(M - e/u)
 *           with M = P/u an integer: when a step holds no codeword and no
 *           lane's term is large, ties, or leaves the binade, the running
 *           value after the step is M minus the warp's exact integer sum
 *           (two 32-bit warp reductions of the terms' 26-bit halves).
 *           Every other step replays the reference's sequence itself: the
 *           32 terms are staged in shared memory and every lane performs the
 *           32 IEEE subtractions in order.  The result equals the sequential
 *           loop bit for bit.
 *  list     codewords are taken in lane order; getLConf (:767-774) uses the
 *           running P_notGuess at each, so T and the list match exactly.
 *  output   soft output of :536-577 on lanes 0..15.
 * The file is built with -fmad=false: every floating-point operation the
 * reference performs is a separately rounded IEEE operation here.
 */
#pragma once
#include <stddef.h>
#include <stdint.h>
#include "sg_crmath.h"
#include "sg_enum.h"
#include "sg_math.h"

/* The decoder's exp and log, chosen per instantiation by the template
 * parameter CR of sg_decode_line: false (the default decoder) -- the
 * table-driven routines of sg_math.h, within 0.51 ulp; true (the
 * reference-exact mode) -- the correctly rounded routines of sg_crmath.h,
 * with which every result equals the reference's under a correctly rounded
 * libm, at about 2x the cost per exp. */
template <bool CR>
__device__ __forceinline__ double sg_dec_exp(double x, const double* tab)
{
    return CR ? sg_exp_cr(x, tab) : sg_exp(x, tab);
}
template <bool CR>
__device__ __forceinline__ double sg_dec_exp_neg(double x, const double* tab)
{
    return CR ? sg_exp_cr_neg(x, tab) : sg_exp_neg(x, tab);
}
template <bool CR>
__device__ __forceinline__ double sg_dec_log(double x, const double* tab)
{
    return CR ? sg_log_cr(x, tab) : sg_log(x, tab);
}

#define SG_FULL 0xffffffffu

template <bool B>
struct SgBoolTag {
    static constexpr bool value = B;
};

struct SgLineParams {
    int32_t L;
    uint32_t tmax;     /* Tmax clamped to 2^32-1 (T never exceeds 65536) */
    double thres;
};

/* Per-warp shared scratch of one line decode. */
#define SG_LIST_MAX 8 /* SG_MAX_L of the C ABI; the entry points reject larger L */

struct alignas(16) SgWarpScratch { /* A is read as double2 */
    double A[256];      /* PM prefix over the low byte of a pattern, entry lo
                           stored at sg_swz(lo) */
    double dz[16];      /* dz[0] = 0, dz[1 + j] = PM increment of sorted
                           position 8 + j (j < 8), the rest 0; indexed by the
                           byte offsets of an order-table entry */
    double qa[16];      /* values for the tie-exact sort, then the input LLRs */
    double ex[16];      /* exp(input LLR) of each position, for the soft output */
    double es[32];      /* general case: exp(-PM) of the 32 patterns of a half */
    double ps[32];      /* general case: P_notGuess after each of them */
    int32_t perm[16];   /* sorted rank -> position */
    int32_t rank[16];   /* position -> sorted rank */
    uint8_t synlo[256]; /* syndrome of the low byte (and of the hard decision),
                           entry lo stored at sg_swz(lo) */
    uint8_t synhi[256]; /* syndrome of the high byte */
    /* the list (touched only at codewords and in the soft output, so it
     * lives here rather than in registers): entry k = exp(-PM) of the k-th
     * codeword found and its bits (bit i = position i) */
    double lst_e[SG_LIST_MAX];
    uint32_t lst_cm[SG_LIST_MAX];
    double pnl;         /* pNL of the last getLConf */
    int32_t curl;       /* codewords listed */
    uint32_t hdm;       /* hard decision, bit i = position i */
};
static_assert(offsetof(SgWarpScratch, synlo) % 8 == 0 && offsetof(SgWarpScratch, synhi) % 8 == 0,
              "syndrome tables are written 8 bytes at a time");

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

/* A codeword found at pattern mask `mj` (sorted positions) whose guess left
 * P_notGuess = P and contributed ej = exp(-PM): list insertion and getLConf
 * (:674-686, :767-774).  Returns true when the line decode stops. */
__device__ __forceinline__ bool sg_list_hit(SgWarpScratch* ws, const SgLineParams& lp, uint32_t mj, double P,
                                            double ej, int lane)
{
    /* AddTEP (:761): position i flips when its sorted rank is in the pattern */
    const int myrank = lane < 16 ? ws->rank[lane] : 0;
    const uint32_t cm = ws->hdm ^ (__ballot_sync(SG_FULL, lane < 16 && ((mj >> myrank) & 1u)) & 0xffffu);
    const int curl = ws->curl;
    double ppos = 0.0;
    for (int i = 0; i < curl; i++)
        ppos = __dadd_rn(ppos, ws->lst_e[i]);
    ppos = __dadd_rn(ppos, ej);
    const double pneg = __dmul_rn(0x1p-8, P); /* 2^-(n-k) * P_notGuess */
    __syncwarp();
    if (lane == 0) {
        ws->lst_e[curl] = ej;
        ws->lst_cm[curl] = cm;
        ws->pnl = pneg;
        ws->curl = curl + 1;
    }
    __syncwarp();
    const double den = __dadd_rn(ppos, pneg);
    const double conf = (den > 1e-40) ? __ddiv_rn(ppos, den) : 1.0;
    return conf > lp.thres || curl + 1 == lp.L;
}

/* General case of one 32-pattern half (first pattern index bh, nv valid
 * patterns): the reference's own sequence P -= e (:626, :672, :712), one
 * IEEE subtraction per pattern in order, evaluated redundantly by every lane
 * from the terms staged in shared memory.  Exact whatever the step holds
 * (codewords, binade crossings, ties, large or tiny terms).  Terms of lanes
 * >= nv are finite and subtracted too: nv < 32 only when the line decode
 * ends in this half, after which P is not read.  With codewords in the half
 * P is recorded after every term, then the codewords are listed in order
 * with the P that followed each.  Sets T and done when the decode stops. */
__device__ __forceinline__ void sg_seq_half(double e, uint32_t ent, uint32_t hits, uint32_t bh, double& P,
                                            SgWarpScratch* ws, uint32_t& T, bool& done, const SgLineParams& lp,
                                            int lane)
{
    ws->es[lane] = e;
    __syncwarp();
    const double2* e2 = reinterpret_cast<const double2*>(ws->es);
    double p = P;
    if (!hits) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const double2 v = e2[k];
            p = __dsub_rn(p, v.x);
            p = __dsub_rn(p, v.y);
        }
        P = p;
    } else {
        double2* p2 = reinterpret_cast<double2*>(ws->ps);
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const double2 v = e2[k];
            const double p0 = __dsub_rn(p, v.x);
            p = __dsub_rn(p0, v.y);
            if (lane == 0)
                p2[k] = make_double2(p0, p);
        }
        P = p;
        __syncwarp();
        uint32_t hm = hits;
        while (hm) {
            const int j = __ffs(hm) - 1;
            const uint32_t mj = sg_ent_pattern(__shfl_sync(SG_FULL, ent, j));
            if (sg_list_hit(ws, lp, mj, ws->ps[j], ws->es[j], lane)) {
                T = bh + (uint32_t)j + 1u;
                done = true;
                break;
            }
            hm &= hm - 1u;
        }
    }
    __syncwarp();
}

/* Extra results of a line decode run for the adjoint (ADJ = true): the
 * sums over the counted guesses that P_notGuess depends on, and the list.
 * Valid for decodes that stop at a list insertion (Tmax >= 65536). */
struct SgAdjOut {
    double etot;    /* uniform: sum of exp(-PM) over the counted guesses */
    double esort;   /* lane r < 16: the same sum over guesses whose pattern holds sorted position r */
    double pnl;     /* uniform: pNL of the last list insertion (before the 1e-40 clamp) */
    double my_e;    /* lane k < curl: exp(-PM) of list entry k */
    uint32_t my_cm; /* lane k < curl: bits of list entry k */
    uint32_t hdm;   /* hard decision, bit i = position i */
    int32_t curl;
    int32_t myrank; /* lane i < 16: sorted rank of position i */
};

/* Decode one line.  llr: this lane's input LLR (lanes 0..15; others
 * ignored).  enum_tabs: SG_ENUM_NTAB tables of SG_ENUM_LEN entries.
 * etab/ltab: shared-memory copies of the exp/log tables. */
template <int G, bool ADJ = false, bool CR = false>
__device__ __forceinline__ SgLineResult sg_decode_line(double llr, const SgLineParams& lp,
                                                        const uint32_t* __restrict__ enum_tabs,
                                                        const double* etab, const double* ltab,
                                                        SgWarpScratch* ws, SgAdjOut* adj = nullptr)
{
    const int lane = threadIdx.x & 31;
    const bool act = lane < 16;
    if (!act)
        llr = 1.0;
    const double a = fabs(llr);
    /* HardDec (:758): 1 unless llr > 0 */
    const uint32_t hdm = __ballot_sync(SG_FULL, act && !(llr > 0.0)) & 0xffffu;
    /* JacLog(-|L_i|) for getPM_HD (:617, :764) */
    /* lanes 0..15: JacLog(-|L_i|); lanes 16..31: JacLog(+|L_(lane-16)|), used
     * for the sorted PM increments below */
    const double a_all = __shfl_sync(SG_FULL, a, lane & 15);
    const double xj = act ? -a_all : a_all;
    const double ex = sg_dec_exp<CR>(xj, etab);
    /* JacLog(xj) = xj if xj > 50, 0 if xj < -50, else log(1 + e^xj) (:762),
     * with its exp kept */
    const double jl = xj > 50 ? xj : (xj < -50 ? 0.0 : sg_dec_log<CR>(1.0 + ex, ltab));
    const double jn = act ? jl : 0.0;
    {
        /* the soft output's exp(LLR) of position p is this exp of lane p + 16
         * when the LLR is positive, of lane p otherwise (a NaN LLR is its own
         * exp) */
        const double lp_ = __shfl_sync(SG_FULL, llr, lane & 15);
        if (act ? !(lp_ > 0.0) : (lp_ > 0.0))
            ws->ex[lane & 15] = lp_ == lp_ ? ex : lp_;
    }

    /* QuickSort of |L| ascending (:618): rank of each position.  Lane p and
     * lane p + 16 count for position p the smaller (and equal) magnitudes
     * among positions 0..7 and 8..15 respectively, then add.  The
     * magnitudes are non-negative, so their high 32 bits order them unless
     * two are equal there; only then are the full values compared. */
    int lt = 0, eq = 0;
    {
        const int p = lane & 15, j0 = lane & 16 ? 8 : 0;
        const uint32_t ah = (uint32_t)(sg_bits(a) >> 32), mine = (uint32_t)(sg_bits(a_all) >> 32);
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const uint32_t hj = __shfl_sync(SG_FULL, ah, j0 + k);
            lt += (hj < mine);
            eq += (hj == mine);
        }
        eq += __shfl_xor_sync(SG_FULL, eq, 16) - 1; /* less the position itself */
        if (__any_sync(SG_FULL, act && eq > 0)) {
            lt = 0;
            eq = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const double aj = __shfl_sync(SG_FULL, a, j0 + k);
                lt += (aj < a_all);
                eq += (aj == a_all) && (j0 + k != p);
            }
            eq += __shfl_xor_sync(SG_FULL, eq, 16);
        }
        lt += __shfl_xor_sync(SG_FULL, lt, 16);
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
    /* getPM_HD: the JacLog terms summed in position order; A[0..15] is free
     * until the tables below are built */
    if (act)
        ws->A[lane] = jn;
    __syncwarp();
    double pmhd = 0.0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const double2 v = reinterpret_cast<const double2*>(ws->A)[i];
        pmhd = __dadd_rn(pmhd, v.x);
        pmhd = __dadd_rn(pmhd, v.y);
    }
    __syncwarp();
    const int src = act ? ws->perm[lane] : 0;
    if (act)
        ws->rank[src] = lane;
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
    const double jp_src = __shfl_sync(SG_FULL, jl, 16 + src); /* JacLog(|L|) of the same position */
    const double dl = act ? __dsub_rn(jp_src, jn_src) : 0.0;
    const uint32_t hs = act ? c_hcol[src] : 0u;
    /* syndrome of the hard decision */
    const uint32_t s0 = __reduce_xor_sync(SG_FULL, (act && ((hdm >> lane) & 1u)) ? (uint32_t)c_hcol[lane] : 0u);

    /* per-line tables; lane j fills A entries j + 32*i, i = 0..7, and
     * syndrome entries 8*j + k, k = 0..7 */
    {
        /* the increments by sorted rank, through es (free until the guess
         * loop) */
        if (act)
            ws->es[lane] = dl;
        __syncwarp();
        double d[8];
        uint32_t hl[8], hh[8];
#pragma unroll
        for (int b = 0; b < 8; b += 2) {
            const double2 v = reinterpret_cast<const double2*>(ws->es)[b / 2];
            d[b] = v.x;
            d[b + 1] = v.y;
        }
#pragma unroll
        for (int b = 0; b < 8; b++) {
            hl[b] = __shfl_sync(SG_FULL, hs, b);
            hh[b] = __shfl_sync(SG_FULL, hs, 8 + b);
        }
        double v0 = pmhd;
        uint32_t sl = s0, sh = 0;
#pragma unroll
        for (int b = 0; b < 5; b++)
            if ((lane >> b) & 1) {
                v0 = __dadd_rn(v0, d[b]);
                sl ^= hl[3 + b];
                sh ^= hh[3 + b];
            }
        const double v1 = __dadd_rn(v0, d[5]);
        const double v2 = __dadd_rn(v0, d[6]);
        const double v3 = __dadd_rn(v1, d[6]);
        /* entry i is stored at sg_swz(i) */
        ws->A[sg_swz(lane)] = v0;
        ws->A[sg_swz(lane + 32)] = v1;
        ws->A[sg_swz(lane + 64)] = v2;
        ws->A[sg_swz(lane + 96)] = v3;
        ws->A[sg_swz(lane + 128)] = __dadd_rn(v0, d[7]);
        ws->A[sg_swz(lane + 160)] = __dadd_rn(v1, d[7]);
        ws->A[sg_swz(lane + 192)] = __dadd_rn(v2, d[7]);
        ws->A[sg_swz(lane + 224)] = __dadd_rn(v3, d[7]);
        /* byte k of the 8 entries 8*lane + k: the lane's syndrome (positions
         * 3..7) XOR those of positions 0..2 selected by k, built in place
         * in two 32-bit words (every value is below 256) */
        const uint32_t lo0 = sl * 0x01010101u ^ hl[0] * 0x01000100u ^ hl[1] * 0x01010000u;
        const uint32_t hi0 = sh * 0x01010101u ^ hh[0] * 0x01000100u ^ hh[1] * 0x01010000u;
        {
            /* stored at sg_swz(8*lane + k) = 8*lane' + (k ^ c): group lane' =
             * lane ^ (g >> 3), bytes permuted by c = g & 7, g the XOR value
             * of the group's bits 5..7 */
            const uint32_t g = (0x14AFEB50u >> (4 * (lane >> 2))) & 15u;
            const uint32_t lo1 = lo0 ^ hl[2] * 0x01010101u;
            const uint32_t sel = 0x3210u ^ ((g & 3u) * 0x1111u);
            const uint32_t w0 = __byte_perm(lo0, 0u, sel), w1 = __byte_perm(lo1, 0u, sel);
            reinterpret_cast<uint2*>(ws->synlo)[lane ^ (g >> 3)] = (g & 4u) ? make_uint2(w1, w0) : make_uint2(w0, w1);
        }
        reinterpret_cast<uint2*>(ws->synhi)[lane] = make_uint2(hi0, hi0 ^ hh[2] * 0x01010101u);
        if (lane < 16)
            ws->dz[lane] = (lane >= 1 && lane <= 8) ? ws->es[lane + 7] : 0.0;
    }
    /* the sort is done with qa: it keeps the input LLRs for the soft output */
    if (act)
        ws->qa[lane] = llr;
    if (lane == 0) {
        ws->curl = 0;
        ws->pnl = 0.0;
        ws->hdm = hdm;
    }
    __syncwarp();

    /* Guess loop (:624-744) */
    const uint32_t* tab = enum_tabs + (size_t)itab * SG_ENUM_LEN;
    const bool has_tmax = lp.tmax < SG_ENUM_LEN;
    double P = 1.0; /* P_notGuess */

    uint32_t T = 0;
    bool done = false;
    double adj_tot = 0.0, adj_r[ADJ ? 16 : 1];
#pragma unroll
    for (int r = 0; r < (ADJ ? 16 : 1); r++)
        adj_r[r] = 0.0;
    /* The loop is instantiated twice.  Without a Tmax cut (TM false) every
     * step holds 32 * G valid patterns: SG_ENUM_LEN is a multiple of 32 * G,
     * so a step either lies inside the order table or starts at its end,
     * where the line decode ends with T = SG_ENUM_LEN. */
    auto guess_loop = [&](auto tm_tag) {
    constexpr bool TM = decltype(tm_tag)::value;
    static_assert(SG_ENUM_LEN % (32u * G) == 0, "steps tile the order table");
    for (uint32_t base = 0; !done; base += 32u * G) {
        if (!TM && base >= SG_ENUM_LEN) {
            T = SG_ENUM_LEN;
            break;
        }
        /* G patterns per lane: lane j of half h tests pattern base + 32h + j */
        uint32_t ent[G];
        double e[G];
        uint32_t hits[G];
        int nv[G];
        int nvt = 0; /* valid patterns of the step, in order */
#pragma unroll
        for (int h = 0; h < G; h++) {
            const uint32_t bh = base + 32u * h;
            const uint32_t t = bh + lane;
            if (TM) {
                ent[h] = __ldg(tab + (t < SG_ENUM_LEN ? t : SG_ENUM_LEN - 1u));
                nv[h] = bh >= SG_ENUM_LEN ? 0 : (bh + 32u <= SG_ENUM_LEN ? 32 : (int)(SG_ENUM_LEN - bh));
            } else {
                ent[h] = __ldg(tab + t);
                nv[h] = 32;
            }
        }
        if (TM) {
            /* T < Tmax is checked before each new logistic weight (:652); a cut
             * in one half ends the step there */
            bool cut_seen = false;
#pragma unroll
            for (int h = 0; h < G; h++) {
                const uint32_t t = base + 32u * h + lane;
                const uint32_t cut =
                    __ballot_sync(SG_FULL, lane < nv[h] && (ent[h] & SG_ENUM_GS) && t > 0 && t >= lp.tmax);
                if (cut_seen)
                    nv[h] = 0;
                else if (cut) {
                    nv[h] = __ffs(cut) - 1;
                    cut_seen = true;
                }
            }
        }
#pragma unroll
        for (int h = 0; h < G; h++) {
            const uint32_t lo = ent[h] & 0xffu; /* already the storage index sg_swz(low byte) */
            const uint32_t hi = (ent[h] >> 8) & 0xffu;
            double pm = ws->A[lo];
            const uint32_t syn = (uint32_t)ws->synlo[lo] ^ (uint32_t)ws->synhi[hi];
            /* high positions in ascending order: the first two from the
             * entry's offsets (offset 0 reads dz[0] = 0, and pm + 0 = pm
             * since pm >= +0), any further ones in a loop few steps enter */
            const char* dzb = reinterpret_cast<const char*>(ws->dz);
            pm = __dadd_rn(pm, *reinterpret_cast<const double*>(dzb + ((ent[h] >> 17) & 0x7fu)));
            pm = __dadd_rn(pm, *reinterpret_cast<const double*>(dzb + ((ent[h] >> 24) & 0x7fu)));
            if (__any_sync(SG_FULL, (ent[h] & SG_ENUM_HI3) != 0u)) {
                uint32_t rest = hi & (hi - 1u);
                rest &= rest - 1u;
                while (rest) {
                    pm = __dadd_rn(pm, ws->dz[__ffs(rest)]);
                    rest &= rest - 1u;
                }
            }
            e[h] = sg_dec_exp_neg<CR>(-pm, etab);
            hits[h] = __ballot_sync(SG_FULL, syn == 0u) & (nv[h] >= 32 ? SG_FULL : ((1u << nv[h]) - 1u));
            nvt += nv[h];
        }

        /* common case: no codeword, no large term, no tie and no binade
         * crossing in the step -- P_notGuess moves by the exact integer sum */
        bool any_hit = false, stepped = false;
#pragma unroll
        for (int h = 0; h < G; h++)
            any_hit |= hits[h] != 0u;
        if (!any_hit && P >= 0x1p-970) {
            const int E = (int)((sg_bits(P) >> 52) & 0x7ffu) - 1023;
            const double iu = sg_from_bits((uint64_t)(52 - E + 1023) << 52);
            /* d = round(q) < 2^52 is the mantissa of q + 2^52; its two 26-bit
             * halves are summed over the warp in 32-bit integers (at most
             * 32 * G terms below 2^26 each) */
            static_assert(G <= 2, "32-bit sums of 26-bit halves hold 64 terms");
            uint32_t slo = 0u, shi = 0u;
            bool bad = false;
#pragma unroll
            for (int h = 0; h < G; h++) {
                const double q = lane < nv[h] ? __dmul_rn(e[h], iu) : 0.0;
                const double t = __dadd_rn(q, 0x1p52);
                const double d = __dsub_rn(t, 0x1p52);
                bad |= !(q < 0x1p52) || fabs(__dsub_rn(q, d)) == 0.5;
                const uint64_t tb = sg_bits(t);
                slo += (uint32_t)tb & 0x3ffffffu;
                shi += (uint32_t)(tb >> 26) & 0x3ffffffu;
            }
            if (!__any_sync(SG_FULL, bad)) {
                const uint32_t tlo = __reduce_add_sync(SG_FULL, slo);
                const uint32_t thi = __reduce_add_sync(SG_FULL, shi);
                /* exact below 2^53; a larger (rounded) total fails the test below */
                const double tot = __dadd_rn(__dmul_rn(__uint2double_rn(thi), 0x1p26), __uint2double_rn(tlo));
                const double M0 = __dmul_rn(P, iu);
                if (tot <= __dsub_rn(M0, 0x1p52 + 1.0)) {
                    P = __dmul_rn(__dsub_rn(M0, tot), sg_from_bits((uint64_t)(E - 52 + 1023) << 52));
                    T = base + (uint32_t)nvt;
                    if (nvt < 32 * G)
                        done = true;
                    stepped = true;
                }
            }
        }

        /* general case, one half after the other */
        if (!stepped) {
#pragma unroll
            for (int h = 0; h < G; h++) {
                if (done)
                    break;
                sg_seq_half(e[h], ent[h], hits[h], base + 32u * h, P, ws, T, done, lp, lane);
                if (!done && nv[h] < 32) {
                    T = base + 32u * h + (uint32_t)nv[h];
                    done = true;
                }
            }
            if (!done)
                T = base + 32u * G;
        }
        if (ADJ) {
            /* the guesses of this step that entered P_notGuess: [base, T) */
#pragma unroll
            for (int h = 0; h < G; h++) {
                if (base + 32u * h + (uint32_t)lane < T) {
                    adj_tot += e[h];
                    const uint32_t m = sg_ent_pattern(ent[h]);
#pragma unroll
                    for (int r = 0; r < (ADJ ? 16 : 1); r++)
                        if ((m >> r) & 1u)
                            adj_r[r] += e[h];
                }
            }
        }
    }
    };
    if (has_tmax)
        guess_loop(SgBoolTag<true>());
    else
        guess_loop(SgBoolTag<false>());
    if (ADJ) {
        /* sums over the warp; lane r keeps sorted position r */
        for (int off = 16; off > 0; off >>= 1)
            adj_tot += __shfl_xor_sync(SG_FULL, adj_tot, off);
        double mine_r = 0.0;
#pragma unroll
        for (int r = 0; r < (ADJ ? 16 : 1); r++) {
            double v = adj_r[r];
            for (int off = 16; off > 0; off >>= 1)
                v += __shfl_xor_sync(SG_FULL, v, off);
            if (lane == r)
                mine_r = v;
        }
        adj->etot = adj_tot;
        adj->esort = mine_r;
        const int curl = ws->curl;
        adj->pnl = ws->pnl;
        adj->my_e = lane < curl ? ws->lst_e[lane] : 0.0;
        adj->my_cm = lane < curl ? ws->lst_cm[lane] : 0u;
        adj->hdm = hdm;
        adj->curl = curl;
        adj->myrank = act ? ws->rank[lane] : 0;
    }

    /* Soft output (:536-577) */
    SgLineResult res;
    res.T = T;
    const int curl = ws->curl;
    res.ncw = curl;
    /* the input LLR of position lane & 15, kept in qa during the loop */
    const double x = ws->qa[lane & 15];
    double lapp, le;
    if (curl == 0) {
        lapp = x;
        le = 0.0;
    } else {
        /* every lane works on position lane & 15; lanes 0..15 then take
         * log(p0), lanes 16..31 log(p1) */
        const int pos = lane & 15;
        const double pnlc = fmax(ws->pnl, 1e-40);
        double pp1 = __ddiv_rn(1.0, __dadd_rn(1.0, ws->ex[pos]));
        double pp0 = __dsub_rn(1.0, pp1);
        pp1 = fmin(fmax(pp1, 1e-40), 1.0);
        pp0 = fmin(fmax(pp0, 1e-40), 1.0);
        double p1 = 0.0, p0 = 0.0;
        for (int j = 0; j < curl; j++) {
            const double c = (double)((ws->lst_cm[j] >> pos) & 1u);
            const double pj = ws->lst_e[j];
            p1 = __dadd_rn(p1, __dmul_rn(c, pj));
            p0 = __dadd_rn(p0, __dmul_rn(__dsub_rn(1.0, c), pj));
        }
        p0 = __dadd_rn(p0, __dmul_rn(pnlc, pp0));
        p1 = __dadd_rn(p1, __dmul_rn(pnlc, pp1));
        const double lg = sg_dec_log<CR>(fmax(act ? p0 : p1, 1e-40), ltab);
        lapp = __dsub_rn(lg, __shfl_sync(SG_FULL, lg, (lane & 15) + 16));
        le = __dsub_rn(lapp, x);
    }
    res.lapp = lapp;
    res.le = le;
    res.hdword = __ballot_sync(SG_FULL, act && !(lapp > 0.0)) & 0xffffu;
    __syncwarp();
    return res;
}
