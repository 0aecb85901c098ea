/* sg_persist.cuh -- batched persistent decoder.
 *
 * One CTA per SM stays resident for the whole batch.  It holds C codeword
 * slots (extrinsic cube, hard-decision words, counters) in shared memory.
 * Every warp repeatedly takes the next undecoded line of any slot whose
 * current phase still has lines to hand out, decodes it (sg_line.cuh), and
 * counts it done.  The warp that completes the 256th line of a phase
 * finishes that phase for the slot: early-termination test, statistics, and
 * either re-opening the slot for its next phase or retiring the codeword
 * (bits and statistics to global memory) and admitting the next codeword of
 * the batch from a device work queue (one atomic counter).  There is no
 * CTA-wide barrier: a slot whose phase is in its tail does not hold back the
 * warps, which move on to the other slots.  Per codeword, the phase
 * sequence and every line decode are those of sg_decode_kernel, so the
 * outputs are bit-identical to the plain decoder's.
 *
 * Waits are bounded: a warp that finds no line sleeps and retries; after
 * args.wait_limit consecutive idle rounds it records an error (SgQueue.err)
 * and exits.  The warps that hold lines are never the ones that give up, so
 * the batch still completes with the remaining warps.
 */
#pragma once

struct SgSlot {
    double le[SG_CUBE];
    uint16_t hdw[256];
    unsigned long long ng;
    unsigned long long ngp;
    unsigned int ngmax;
    int cw;    /* codeword decoded in the slot, -1 when empty */
    int phase; /* index of the phase being decoded */
    int next;  /* next line of the phase to hand out (>= 256: none) */
    int done;  /* lines of the phase finished */
};

template <int NW, int C>
struct SgPersistSmem {
    SgSlot slot[C];
    alignas(16) double etab[SG_EXP_TAB_LEN]; /* read as double2 by the exp routines */
    alignas(16) double ltab[SG_LOG_TAB_LEN];
    SgWarpScratch ws[NW];
};

struct SgQueue {
    unsigned long long head; /* next codeword of the batch to admit */
    unsigned int err;        /* bit 1: a warp gave up waiting */
    unsigned int pad;
};

__device__ __forceinline__ int sg_ld_volatile(const int* p) { return *(volatile const int*)p; }

/* Write the retired codeword's bits and statistics (the plain kernel's
 * output stage). */
__device__ __forceinline__ void sg_slot_retire(const SgSlot& sl, const SgDecodeArgs& args, int cw, int phases,
                                               bool conv, int lane)
{
    const int axis_last = (phases - 1) % 3;
    for (int t = lane; t < SG_INFO_BYTES; t += 32) {
        uint32_t byte = 0;
        for (int q = 0; q < 8; q++) {
            const int b = t * 8 + q;
            const int p = (b >> 6) * 256 + ((b >> 3) & 7) * 16 + (b & 7);
            int l, bit;
            if (axis_last == 0) {
                l = (p >> 8) * 16 + ((p >> 4) & 15);
                bit = p & 15;
            } else if (axis_last == 1) {
                l = (p >> 8) * 16 + (p & 15);
                bit = (p >> 4) & 15;
            } else {
                l = ((p >> 4) & 15) * 16 + (p & 15);
                bit = p >> 8;
            }
            byte = (byte << 1) | ((sl.hdw[l] >> bit) & 1u);
        }
        args.bits[(size_t)cw * SG_INFO_BYTES + t] = (uint8_t)byte;
    }
    if (lane == 0 && args.stats) {
        sg_cw_stats st;
        st.iterations = 0.5 * phases;
        st.ng = sl.ng;
        st.ng_p = sl.ngp;
        st.converged = conv ? 1 : 0;
        st.phases = phases;
        args.stats[cw] = st;
    }
}

/* Take the next codeword of the batch into slot `sl` (warp-wide), or mark
 * the slot empty when the batch is exhausted.  Codewords with non-finite
 * LLRs are reported (converged = -1) and skipped. */
__device__ __forceinline__ void sg_slot_admit(SgSlot& sl, const SgDecodeArgs& args, SgQueue* q, int lane)
{
    for (;;) {
        unsigned long long idx = 0;
        if (lane == 0)
            idx = atomicAdd(&q->head, 1ull);
        idx = __shfl_sync(SG_FULL, idx, 0);
        if (idx >= args.n_cw) {
            if (lane == 0)
                *(volatile int*)&sl.cw = -1;
            __syncwarp();
            return;
        }
        const double* g = args.llr + idx * SG_CUBE;
        bool bad = false;
        for (int i = lane; i < SG_CUBE; i += 32)
            bad |= !isfinite(__ldg(g + i));
        if (__any_sync(SG_FULL, bad)) {
            for (int t = lane; t < SG_INFO_BYTES; t += 32)
                args.bits[idx * SG_INFO_BYTES + t] = 0;
            if (lane == 0 && args.stats) {
                sg_cw_stats st;
                st.iterations = 0;
                st.ng = 0;
                st.ng_p = 0;
                st.converged = -1;
                st.phases = 0;
                args.stats[idx] = st;
            }
            continue;
        }
        for (int i = lane; i < SG_CUBE; i += 32)
            sl.le[i] = 0.0;
        if (lane == 0) {
            sl.ng = 0;
            sl.ngp = 0;
            sl.ngmax = 0;
            sl.phase = 0;
            sl.done = 0;
            *(volatile int*)&sl.cw = (int)idx;
        }
        __threadfence_block();
        __syncwarp();
        if (lane == 0)
            atomicExch(&sl.next, 0); /* open the first phase */
        __syncwarp();
        return;
    }
}

template <int NW, int C, int G, bool CR>
__global__ void __launch_bounds__(NW * 32, 1) sg_persist_kernel(const __grid_constant__ SgDecodeArgs args,
                                                                SgQueue* q)
{
    constexpr int NT = NW * 32;
    SgPersistSmem<NW, C>& S = *reinterpret_cast<SgPersistSmem<NW, C>*>(sg_smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < SG_EXP_TAB_LEN; i += NT)
        S.etab[i] = g_etab[i];
    for (int i = tid; i < SG_LOG_TAB_LEN; i += NT)
        S.ltab[i] = g_ltab[i];
    if (tid < C) {
        S.slot[tid].cw = -1;
        S.slot[tid].next = 256;
    }
    __syncthreads();
    if (warp < C)
        sg_slot_admit(S.slot[warp], args, q, lane);
    __syncthreads();

    SgLineParams lp;
    lp.L = args.L;
    lp.tmax = args.tmax;
    lp.thres = args.thres;
    const int nphase = 3 * args.imax;
    int idle = 0;
    for (;;) {
        /* find a line: slots in a warp-dependent order */
        int s = -1, l = 256;
        for (int k = 0; k < C; k++) {
            const int c = (warp + k) % C;
            int got = 256;
            if (lane == 0 && sg_ld_volatile(&S.slot[c].cw) >= 0 && sg_ld_volatile(&S.slot[c].next) < 256)
                got = atomicAdd(&S.slot[c].next, 1);
            got = __shfl_sync(SG_FULL, got, 0);
            if (got < 256) {
                s = c;
                l = got;
                break;
            }
        }
        if (s < 0) {
            bool live = false;
            for (int c = 0; c < C; c++)
                live |= sg_ld_volatile(&S.slot[c].cw) >= 0;
            if (!live)
                break;
            if (++idle > args.wait_limit) {
                if (lane == 0)
                    atomicOr(&q->err, 2u);
                break;
            }
            __nanosleep(256);
            continue;
        }
        idle = 0;
        __threadfence_block(); /* see the slot state published with the line */
        SgSlot& sl = S.slot[s];
        const int phase = sg_ld_volatile(&sl.phase);
        const int cw = sg_ld_volatile(&sl.cw);
        const int axis = phase % 3;
        const double alpha = args.alpha[phase];
        const double* g = args.llr + (size_t)cw * SG_CUBE;
        const int pos = sg_pos(axis, l, lane & 15);
        double v = 1.0;
        if (lane < 16) /* L_ch + (alpha*L_E) */
            v = __dadd_rn(__ldg(g + pos), __dmul_rn(alpha, sl.le[pos]));
        const SgLineResult r = sg_decode_line<G, false, CR>(v, lp, args.enum_tabs, S.etab, S.ltab, &S.ws[warp]);
        if (lane < 16) {
            sl.le[pos] = r.le;
            if (args.lapp)
                args.lapp[(size_t)cw * SG_CUBE + pos] = r.lapp;
        }
        if (lane == 0) {
            sl.hdw[l] = (uint16_t)r.hdword;
            atomicAdd(&sl.ng, (unsigned long long)r.T);
            atomicMax(&sl.ngmax, r.T);
        }
        __threadfence_block();
        __syncwarp();
        int d = 0;
        if (lane == 0)
            d = atomicAdd(&sl.done, 1);
        d = __shfl_sync(SG_FULL, d, 0);
        if (d != 255)
            continue;

        /* this warp finished the phase: every other line's writes are
         * visible after the fence that preceded its done increment */
        __threadfence_block();
        const int phases = phase + 1;
        const unsigned long long ngp = sl.ngp + (unsigned long long)(*(volatile unsigned int*)&sl.ngmax);
        const bool conv = sg_is_codeword(sl.hdw, lane);
        if (lane == 0)
            sl.ngp = ngp;
        __syncwarp();
        if (conv || phases == nphase) {
            sg_slot_retire(sl, args, cw, phases, conv, lane);
            __syncwarp();
            sg_slot_admit(sl, args, q, lane);
        } else {
            if (lane == 0) {
                sl.ngmax = 0;
                sl.done = 0;
                *(volatile int*)&sl.phase = phases;
            }
            __threadfence_block();
            __syncwarp();
            if (lane == 0)
                atomicExch(&sl.next, 0); /* open the next phase */
            __syncwarp();
        }
    }
}
