/* sg_line16.cuh -- two SOGRAND component decodes per warp, 16 lanes each.
 *
 * The same restatement of SOGRAND_bitSO + sogrand_main_logic
 * (SOGRAND_C/cubic_decoder_final.c:521-746) as sg_decode_line, with the
 * same per-line tables, order tables, integer-sum fast path and sequential
 * replay, laid out for 16 lanes: lane p of a half-warp owns position p of
 * its line for the whole decode (both JacLog terms, a full rank count, 16
 * table entries), and a guess step tests 16 * G consecutive patterns of
 * each line, G per lane.  The two lines of a warp run in lockstep: every
 * warp collective is executed by all 32 lanes (16-lane shuffles, ballots
 * shifted to the half), the guess loop steps while either line is
 * undecided, and each half applies a step's results to its own line only.
 * Results are bit-identical to sg_decode_line's.  It is the lines-per-warp
 * = 2 / lane width = 16 point of the kernel configurations (variants
 * "w*-l2-*").
 */
#pragma once
#include "sg_line.cuh"

/* bit i = predicate of lane i of the half starting at lane hb */
__device__ __forceinline__ uint32_t sg_pballot(int hb, bool p)
{
    return (__ballot_sync(SG_FULL, p) >> hb) & 0xffffu;
}

/* sum / XOR over the 16 lanes of each half (all 32 lanes take part) */
__device__ __forceinline__ uint32_t sg_psum_u32(uint32_t v)
{
#pragma unroll
    for (int off = 8; off > 0; off >>= 1)
        v += __shfl_xor_sync(SG_FULL, v, off, 16);
    return v;
}

__device__ __forceinline__ uint32_t sg_pxor_u32(uint32_t v)
{
#pragma unroll
    for (int off = 8; off > 0; off >>= 1)
        v ^= __shfl_xor_sync(SG_FULL, v, off, 16);
    return v;
}

/* sg_list_hit for the line of a half-warp, executed by the whole warp: the
 * same list insertion and getLConf, the same floating-point operations in
 * the same order; only a half with `act` set changes its list.  Returns
 * true when that half's line decode stops. */
__device__ __forceinline__ bool sg_list_hit16(SgWarpScratch* ws, const SgLineParams& lp, uint32_t mj, double P,
                                              double ej, int sl, int hb, bool act)
{
    const int myrank = ws->rank[sl];
    const uint32_t cm = ws->hdm ^ sg_pballot(hb, (mj >> myrank) & 1u);
    const int curl = ws->curl;
    double ppos = 0.0;
    for (int i = 0; i < curl; i++)
        ppos = __dadd_rn(ppos, ws->lst_e[i]);
    ppos = __dadd_rn(ppos, ej);
    const double pneg = __dmul_rn(0x1p-8, P);
    __syncwarp();
    if (act && sl == 0) {
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

/* The reference's sequential P -= e over the 16 patterns of one sub-step
 * (first pattern index bh) for each half with `run` set, every lane of the
 * half evaluating its line's chain from the terms staged in shared memory;
 * codewords listed in order with the P that followed each.  Executed by the
 * whole warp (sg_seq_half for two 16-lane lines). */
__device__ __forceinline__ void sg_seq_sub16(double e, uint32_t ent, uint32_t hits, uint32_t bh, double& P,
                                             SgWarpScratch* ws, uint32_t& T, bool& done, bool run,
                                             const SgLineParams& lp, int sl, int hb)
{
    ws->es[sl] = e;
    __syncwarp();
    const double2* e2 = reinterpret_cast<const double2*>(ws->es);
    double2* p2 = reinterpret_cast<double2*>(ws->ps);
    const bool rec = __any_sync(SG_FULL, run && hits != 0u);
    double p = P;
    if (!rec) {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const double2 v = e2[k];
            p = __dsub_rn(p, v.x);
            p = __dsub_rn(p, v.y);
        }
    } else {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const double2 v = e2[k];
            const double p0 = __dsub_rn(p, v.x);
            p = __dsub_rn(p0, v.y);
            if (sl == 0)
                p2[k] = make_double2(p0, p);
        }
    }
    if (run)
        P = p;
    __syncwarp();
    uint32_t hm = run ? hits : 0u;
    while (__any_sync(SG_FULL, hm != 0u)) {
        const bool act = hm != 0u;
        const int j = act ? __ffs(hm) - 1 : 0;
        const uint32_t mj = sg_ent_pattern(__shfl_sync(SG_FULL, ent, j, 16));
        const bool stop = sg_list_hit16(ws, lp, mj, ws->ps[j], ws->es[j], sl, hb, act);
        if (act && stop) {
            T = bh + (uint32_t)j + 1u;
            done = true;
            hm = 0u;
        } else if (act) {
            hm &= hm - 1u;
        }
    }
    __syncwarp();
}

/* Decode two lines, one per half-warp, in lockstep.  Every lane of the warp
 * calls this together.  llr: the input LLR of this lane's position (lane
 * within its half); ws: the half's line scratch.  Returns, as
 * sg_decode_line, the soft output of this lane's position and its line's
 * hard-decision word, T and codewords listed. */
template <int G, bool CR>
__device__ __forceinline__ SgLineResult sg_decode_line16(double llr, const SgLineParams& lp,
                                                          const uint32_t* __restrict__ enum_tabs,
                                                          const double* etab, const double* ltab,
                                                          SgWarpScratch* ws)
{
    const int lane = threadIdx.x & 31;
    const int hb = lane & 16, sl = lane & 15;
    const double a = fabs(llr);
    /* HardDec (:758): 1 unless llr > 0 */
    const uint32_t hdm = sg_pballot(hb, !(llr > 0.0));
    /* JacLog(-|L|) for getPM_HD (:617, :764) and JacLog(+|L|) for the PM
     * increments, each with its exp kept */
    const double xn = -a, xq = a;
    const double exn = sg_dec_exp<CR>(xn, etab);
    const double exq = sg_dec_exp<CR>(xq, etab);
    const double jn = xn > 50 ? xn : (xn < -50 ? 0.0 : sg_dec_log<CR>(1.0 + exn, ltab));
    const double jq = xq > 50 ? xq : (xq < -50 ? 0.0 : sg_dec_log<CR>(1.0 + exq, ltab));
    /* the soft output's exp(LLR): exp(+|L|) for a positive LLR, exp(-|L|)
     * otherwise, a NaN LLR its own */
    ws->ex[sl] = llr > 0.0 ? exq : (llr == llr ? exn : llr);

    /* QuickSort of |L| ascending (:618): rank of each position, from the
     * magnitudes' high 32 bits unless two collide there (in either line:
     * the full comparison gives the same ranks) */
    int lt = 0, eq = 0;
    {
        const uint32_t ah = (uint32_t)(sg_bits(a) >> 32);
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const uint32_t hj = __shfl_sync(SG_FULL, ah, k, 16);
            lt += (hj < ah);
            eq += (hj == ah);
        }
        eq -= 1; /* less the position itself */
        if (__any_sync(SG_FULL, eq > 0)) {
            lt = 0;
            eq = 0;
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const double aj = __shfl_sync(SG_FULL, a, k, 16);
                lt += (aj < a);
                eq += (aj == a) && (k != sl);
            }
        }
    }
    /* ties (and NaN, which no comparison orders) take the exact quicksort */
    const bool qsort = sg_pballot(hb, eq > 0 || a != a) != 0u;
    if (!qsort) {
        ws->perm[lt] = sl;
    } else {
        ws->qa[sl] = a;
        ws->perm[sl] = sl;
    }
    __syncwarp();
    if (qsort && sl == 0)
        sg_quicksort16(ws->qa, ws->perm);
    /* getPM_HD: the JacLog terms summed in position order */
    ws->A[sl] = jn;
    __syncwarp();
    double pmhd = 0.0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const double2 v = reinterpret_cast<const double2*>(ws->A)[i];
        pmhd = __dadd_rn(pmhd, v.x);
        pmhd = __dadd_rn(pmhd, v.y);
    }
    __syncwarp();
    const int src = ws->perm[sl]; /* this lane now also speaks for sorted rank sl */
    ws->rank[src] = sl;
    const double as = __shfl_sync(SG_FULL, a, src, 16);

    /* IC (:619-622) */
    const double a0 = __shfl_sync(SG_FULL, as, 0, 16);
    const double a7 = __shfl_sync(SG_FULL, as, 7, 16);
    const double beta = __ddiv_rn(__dsub_rn(a7, a0), 7.0);
    int32_t ic = sg_cvt_i32(round(__dsub_rn(__ddiv_rn(a0, beta), 1.0)));
    if (ic < 0)
        ic = 0;
    const int itab = ic < SG_ENUM_IC_CANON ? ic : SG_ENUM_IC_CANON;

    /* PM increment of sorted position sl (getPM, :765) and its syndrome
     * column; the syndrome of the hard decision */
    const double dl = __dsub_rn(__shfl_sync(SG_FULL, jq, src, 16), __shfl_sync(SG_FULL, jn, src, 16));
    const uint32_t hs = c_hcol[src];
    const uint32_t s0 = sg_pxor_u32(((hdm >> sl) & 1u) ? (uint32_t)c_hcol[sl] : 0u);

    /* per-line tables: lane j fills A entries j + 16*i and the syndromes of
     * bytes 16*j + k, i, k = 0..15 */
    {
        ws->es[sl] = dl;
        __syncwarp();
        double d[8];
#pragma unroll
        for (int b = 0; b < 8; b += 2) {
            const double2 v = reinterpret_cast<const double2*>(ws->es)[b / 2];
            d[b] = v.x;
            d[b + 1] = v.y;
        }
        /* bits 0..3 of the entry from the lane, in ascending order */
        double w[16];
        w[0] = pmhd;
#pragma unroll
        for (int b = 0; b < 4; b++)
            if ((sl >> b) & 1)
                w[0] = __dadd_rn(w[0], d[b]);
        /* bits 4..7 from i, each added after the lower ones */
#pragma unroll
        for (int b = 0; b < 4; b++)
#pragma unroll
            for (int i = 0; i < (1 << b); i++)
                w[i + (1 << b)] = __dadd_rn(w[i], d[4 + b]);
#pragma unroll
        for (int i = 0; i < 16; i++)
            ws->A[sg_swz((uint32_t)(sl + 16 * i))] = w[i];
        /* syndromes: byte 16*sl + k is the XOR of the columns of its bits;
         * bits 4..7 from the lane, bits 0..3 from k (Gray order, one XOR per
         * entry) */
        uint32_t hl[8], hh[8];
#pragma unroll
        for (int b = 0; b < 8; b++) {
            hl[b] = __shfl_sync(SG_FULL, hs, b, 16);
            hh[b] = __shfl_sync(SG_FULL, hs, 8 + b, 16);
        }
        uint32_t bl = s0, bhi = 0u;
#pragma unroll
        for (int b = 0; b < 4; b++)
            if ((sl >> b) & 1) {
                bl ^= hl[4 + b];
                bhi ^= hh[4 + b];
            }
        uint32_t gl = 0u, gh = 0u;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            if (k) {
                const int b = __ffs(k) - 1; /* the bit in which Gray codes k-1 and k differ */
                gl ^= hl[b];
                gh ^= hh[b];
            }
            const uint32_t g = (uint32_t)(k ^ (k >> 1));
            const uint32_t byte = 16u * (uint32_t)sl + g;
            ws->synlo[sg_swz(byte)] = (uint8_t)(bl ^ gl);
            ws->synhi[byte] = (uint8_t)(bhi ^ gh);
        }
        ws->dz[sl] = (sl >= 1 && sl <= 8) ? ws->es[sl + 7] : 0.0;
    }
    /* the input LLRs for the soft output */
    ws->qa[sl] = llr;
    if (sl == 0) {
        ws->curl = 0;
        ws->pnl = 0.0;
        ws->hdm = hdm;
    }
    __syncwarp();

    /* Guess loop (:624-744), 16 * G patterns of each line per step, while
     * either line is undecided */
    const uint32_t* tab = enum_tabs + (size_t)itab * SG_ENUM_LEN;
    const bool has_tmax = lp.tmax < SG_ENUM_LEN;
    double P = 1.0; /* P_notGuess */
    uint32_t T = 0;
    bool done = false;
    auto guess_loop = [&](auto tm_tag) {
    constexpr bool TM = decltype(tm_tag)::value;
    static_assert(SG_ENUM_LEN % (16u * G) == 0, "steps tile the order table");
    for (uint32_t base = 0; __any_sync(SG_FULL, !done); base += 16u * G) {
        if (!TM && base >= SG_ENUM_LEN) {
            if (!done) {
                T = SG_ENUM_LEN;
                done = true;
            }
            break;
        }
        /* G patterns per lane: lane j of sub-step h tests pattern base + 16h + j */
        uint32_t ent[G];
        double e[G];
        uint32_t hits[G];
        int nv[G];
        int nvt = 0;
#pragma unroll
        for (int h = 0; h < G; h++) {
            const uint32_t bh = base + 16u * h;
            const uint32_t t = bh + (uint32_t)sl;
            if (TM) {
                ent[h] = __ldg(tab + (t < SG_ENUM_LEN ? t : SG_ENUM_LEN - 1u));
                nv[h] = bh >= SG_ENUM_LEN ? 0 : (bh + 16u <= SG_ENUM_LEN ? 16 : (int)(SG_ENUM_LEN - bh));
            } else {
                ent[h] = __ldg(tab + t);
                nv[h] = 16;
            }
        }
        if (TM) {
            /* T < Tmax is checked before each new logistic weight (:652) */
            bool cut_seen = false;
#pragma unroll
            for (int h = 0; h < G; h++) {
                const uint32_t t = base + 16u * h + (uint32_t)sl;
                const uint32_t cut = sg_pballot(hb, sl < nv[h] && (ent[h] & SG_ENUM_GS) && t > 0 && t >= lp.tmax);
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
            const uint32_t lo = ent[h] & 0xffu;
            const uint32_t hi = (ent[h] >> 8) & 0xffu;
            double pm = ws->A[lo];
            const uint32_t syn = (uint32_t)ws->synlo[lo] ^ (uint32_t)ws->synhi[hi];
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
            hits[h] = sg_pballot(hb, syn == 0u) & (nv[h] >= 16 ? 0xffffu : ((1u << nv[h]) - 1u));
            nvt += nv[h];
        }

        /* common case, per line: no codeword, no large term, no tie and no
         * binade crossing in the step -- P_notGuess moves by the exact
         * integer sum */
        bool any_hit = false, stepped = false;
#pragma unroll
        for (int h = 0; h < G; h++)
            any_hit |= hits[h] != 0u;
        const bool try_fast = !done && !any_hit && P >= 0x1p-970;
        if (__any_sync(SG_FULL, try_fast)) {
            const int E = (int)((sg_bits(P) >> 52) & 0x7ffu) - 1023;
            const double iu = sg_from_bits((uint64_t)(52 - E + 1023) << 52);
            static_assert(G <= 4, "32-bit sums of 26-bit halves hold 64 terms");
            uint32_t slo = 0u, shi = 0u;
            bool bad = false;
#pragma unroll
            for (int h = 0; h < G; h++) {
                const double q = sl < nv[h] ? __dmul_rn(e[h], iu) : 0.0;
                const double t = __dadd_rn(q, 0x1p52);
                const double d = __dsub_rn(t, 0x1p52);
                bad |= !(q < 0x1p52) || fabs(__dsub_rn(q, d)) == 0.5;
                const uint64_t tb = sg_bits(t);
                slo += (uint32_t)tb & 0x3ffffffu;
                shi += (uint32_t)(tb >> 26) & 0x3ffffffu;
            }
            const bool anybad = sg_pballot(hb, bad) != 0u;
            const uint32_t tlo = sg_psum_u32(slo);
            const uint32_t thi = sg_psum_u32(shi);
            const double tot = __dadd_rn(__dmul_rn(__uint2double_rn(thi), 0x1p26), __uint2double_rn(tlo));
            const double M0 = __dmul_rn(P, iu);
            if (try_fast && !anybad && tot <= __dsub_rn(M0, 0x1p52 + 1.0)) {
                P = __dmul_rn(__dsub_rn(M0, tot), sg_from_bits((uint64_t)(E - 52 + 1023) << 52));
                T = base + (uint32_t)nvt;
                if (nvt < 16 * G)
                    done = true;
                stepped = true;
            }
        }

        /* general case, one sub-step after the other, for the lines that
         * need it */
        const bool need = !done && !stepped;
        if (__any_sync(SG_FULL, need)) {
            bool run = need;
#pragma unroll
            for (int h = 0; h < G; h++) {
                sg_seq_sub16(e[h], ent[h], hits[h], base + 16u * h, P, ws, T, done, run, lp, sl, hb);
                if (run && !done && nv[h] < 16) {
                    T = base + 16u * h + (uint32_t)nv[h];
                    done = true;
                }
                run = run && !done;
            }
            if (run)
                T = base + 16u * G;
        }
    }
    };
    if (__any_sync(SG_FULL, has_tmax))
        guess_loop(SgBoolTag<true>());
    else
        guess_loop(SgBoolTag<false>());

    /* Soft output (:536-577) */
    SgLineResult res;
    res.T = T;
    const int curl = ws->curl;
    res.ncw = curl;
    const double x = ws->qa[sl];
    double lapp = x, le = 0.0;
    if (curl != 0) {
        const double pnlc = fmax(ws->pnl, 1e-40);
        double pp1 = __ddiv_rn(1.0, __dadd_rn(1.0, ws->ex[sl]));
        double pp0 = __dsub_rn(1.0, pp1);
        pp1 = fmin(fmax(pp1, 1e-40), 1.0);
        pp0 = fmin(fmax(pp0, 1e-40), 1.0);
        double p1 = 0.0, p0 = 0.0;
        for (int j = 0; j < curl; j++) {
            const double c = (double)((ws->lst_cm[j] >> sl) & 1u);
            const double pj = ws->lst_e[j];
            p1 = __dadd_rn(p1, __dmul_rn(c, pj));
            p0 = __dadd_rn(p0, __dmul_rn(__dsub_rn(1.0, c), pj));
        }
        p0 = __dadd_rn(p0, __dmul_rn(pnlc, pp0));
        p1 = __dadd_rn(p1, __dmul_rn(pnlc, pp1));
        const double lg0 = sg_dec_log<CR>(fmax(p0, 1e-40), ltab);
        const double lg1 = sg_dec_log<CR>(fmax(p1, 1e-40), ltab);
        lapp = __dsub_rn(lg0, lg1);
        le = __dsub_rn(lapp, x);
    }
    res.lapp = lapp;
    res.le = le;
    res.hdword = sg_pballot(hb, !(lapp > 0.0));
    __syncwarp();
    return res;
}
