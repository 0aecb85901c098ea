/* sg_api.cu -- B200 SOGRAND cubic decoder: kernels and C ABI.
 *
 * Kernels
 *   sg_decode_kernel   the whole iterative decode of a codeword per CTA
 *                      (SOGRAND_C/cubic_decoder_final.c:119-289): the 32 KB
 *                      channel cube arrives in shared memory by one bulk
 *                      asynchronous copy (cp.async.bulk, completion on an
 *                      mbarrier) and stays there with the 32 KB extrinsic
 *                      cube for all iterations; 8 warps take the 256 lines
 *                      of a phase from a shared counter and decode one line
 *                      each (sg_line.cuh); after every phase one warp runs the
 *                      early-termination test on the 256 hard-decision words.
 *   sg_bitso_kernel    SOGRAND_bitSO on independent lines, one warp per line.
 *   sg_gen_kernel      seeded source + encoder + AWGN channel (sg_gen.h).
 *
 * Built with -fmad=false: no floating-point contraction anywhere, as in the
 * reference's plain gcc build; the exp/log routines use explicit FMAs.
 */
#include <cuda_runtime.h>

#include <errno.h>
#include <stddef.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sogrand_b200.h"
#include "sg_code.h"
#include "sg_enum.h"
#include "sg_gen.h"
#include "sg_line.cuh"
#include "sg_line16.cuh"
#include "sg_math.h"

#define SG_THREADS 256
#define SG_WARPS (SG_THREADS / 32)
/* Bounded device-side waits.  The limit of a wait that can give up (the
 * bulk-copy wait here, the persistent decoder's idle rounds) is a launch
 * argument, SG_WAIT_LIMIT_DEFAULT unless sg_set_wait_limit() changed it.
 * After a bulk-copy wait gave up, the copy may still be writing into the
 * CTA's shared memory: the CTA waits for it again, up to SG_DRAIN_LIMIT
 * polls, before it releases that memory. */
#define SG_WAIT_LIMIT_DEFAULT (1ll << 22)
#define SG_DRAIN_LIMIT (1ll << 26)

__device__ const double g_etab[SG_EXP_TAB_LEN] = SG_EXP_TAB_INIT;
__device__ const double g_ltab[SG_LOG_TAB_LEN] = SG_LOG_TAB_INIT;

/* ------------------------------------------------------------ device -- */

struct SgDecodeArgs {
    const double* llr;
    uint8_t* bits;
    double* lapp;
    sg_cw_stats* stats;
    const uint32_t* enum_tabs;
    unsigned int* err;
    double* ckpt; /* nullable: [n_cw][3*imax][4096], L_E entering each phase */
    unsigned long long n_cw;
    long long wait_limit; /* polls or idle rounds before a bounded wait gives up */
    int32_t L;
    int32_t imax;
    uint32_t tmax;
    int32_t use_bulk;
    double thres;
    double alpha[SG_MAX_PHASES];
};

/* Poll the mbarrier for phase `parity` at most `limit` times; 1 when it
 * completed. */
__device__ __forceinline__ uint32_t sg_mbar_wait(uint32_t mbar, uint32_t parity, long long limit)
{
    uint32_t ok = 0;
    for (long long it = 0; it < limit && !ok; it++) {
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(ok)
            : "r"(mbar), "r"(parity)
            : "memory");
    }
    return ok;
}

/* Outputs of a codeword that is not decoded: zero bits and statistics with
 * the given converged code (-1 non-finite input, -2 a wait gave up).
 * Called by the whole CTA. */
__device__ __forceinline__ void sg_cw_not_decoded(const SgDecodeArgs& args, unsigned long long cw, int code)
{
    if (threadIdx.x < SG_INFO_BYTES)
        args.bits[cw * SG_INFO_BYTES + threadIdx.x] = 0;
    if (threadIdx.x == 0 && args.stats) {
        sg_cw_stats st;
        st.iterations = 0;
        st.ng = 0;
        st.ng_p = 0;
        st.converged = code;
        st.phases = 0;
        args.stats[cw] = st;
    }
}

/* Shared memory of a decode CTA.  With LCH_SMEM the channel cube is staged
 * here by one bulk copy; otherwise each line reads its 16 channel LLRs from
 * global memory (L2-resident) once per phase. */
template <int NW, bool LCH_SMEM, int LPW = 1> /* LPW: lines decoded per warp at a time */
struct SgCwSmem {
    alignas(16) double lch[LCH_SMEM ? SG_CUBE : 2]; /* bulk-copy destination */
    double le[SG_CUBE];
    alignas(16) double etab[SG_EXP_TAB_LEN]; /* read as double2 by the exp routines */
    alignas(16) double ltab[SG_LOG_TAB_LEN];
    SgWarpScratch ws[NW * LPW];
    uint16_t hdw[256];
    unsigned long long mbar;
    unsigned long long ng;
    unsigned int ngmax;
    int line_next;
    int conv;
    int bad;
};

/* Cube index of bit `i` of line `l` in phase `axis` (lines of the reference's
 * column phase run along the stride-1 index, rows along stride 16, slices
 * along stride 256; cubic_decoder_final.c:157-247). */
__device__ __forceinline__ int sg_pos(int axis, int l, int i)
{
    const int a = l >> 4, b = l & 15;
    if (axis == 0)
        return a * 256 + b * 16 + i;
    if (axis == 1)
        return a * 256 + i * 16 + b;
    return i * 256 + a * 16 + b;
}

/* Early termination (cubic_decoder_final.c:317-391) on the 256 line words
 * of the phase just run: the hard decisions form a product codeword iff
 * every word is a component codeword and the words satisfy the component
 * parity equations along both other axes (bitwise).  Warp-wide. */
__device__ __forceinline__ bool sg_is_codeword(const uint16_t* hdw, int lane)
{
    bool bad = false;
    for (int q = lane; q < 256; q += 32) {
        const uint32_t x = hdw[q];
        bad |= ((x >> 8) & 0xffu) != c_ptab[x & 0xffu];
    }
    for (int q = lane; q < 128; q += 32) {
        const int a = q >> 3, j = q & 7;
        uint32_t acc = 0;
#pragma unroll
        for (int b = 0; b < 8; b++)
            if ((c_prow[b] >> j) & 1u)
                acc ^= hdw[a * 16 + b];
        bad |= acc != hdw[a * 16 + 8 + j];
    }
    for (int q = lane; q < 128; q += 32) {
        const int b = q >> 3, j = q & 7;
        uint32_t acc = 0;
#pragma unroll
        for (int a = 0; a < 8; a++)
            if ((c_prow[a] >> j) & 1u)
                acc ^= hdw[a * 16 + b];
        bad |= acc != hdw[(8 + j) * 16 + b];
    }
    return !__any_sync(SG_FULL, bad);
}

__device__ __forceinline__ uint32_t sg_smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

extern __shared__ __align__(128) unsigned char sg_smem_raw[];

template <int NW, bool LCH_SMEM, int MINB, int G, bool CR, int LPW = 1>
__global__ void __launch_bounds__(NW * 32, MINB) sg_decode_kernel(const __grid_constant__ SgDecodeArgs args)
{
    constexpr int NT = NW * 32;
    SgCwSmem<NW, LCH_SMEM, LPW>& S = *reinterpret_cast<SgCwSmem<NW, LCH_SMEM, LPW>*>(sg_smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool use_bulk = LCH_SMEM && args.use_bulk;
    for (int i = tid; i < SG_EXP_TAB_LEN; i += NT)
        S.etab[i] = g_etab[i];
    for (int i = tid; i < SG_LOG_TAB_LEN; i += NT)
        S.ltab[i] = g_ltab[i];
    const uint32_t mbar = sg_smem_u32(&S.mbar);
    if (tid == 0 && use_bulk) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t phase_bit = 0;
    SgLineParams lp;
    lp.L = args.L;
    lp.tmax = args.tmax;
    lp.thres = args.thres;

    for (unsigned long long cw = blockIdx.x; cw < args.n_cw; cw += gridDim.x) {
        const double* g = args.llr + cw * SG_CUBE;
        if (use_bulk) {
            if (tid == 0) {
                /* order earlier generic-proxy reads of lch before the async write */
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar),
                             "r"((uint32_t)(SG_CUBE * 8))
                             : "memory");
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                        sg_smem_u32(S.lch)),
                    "l"(g), "r"((uint32_t)(SG_CUBE * 8)), "r"(mbar)
                    : "memory");
            }
        } else if (LCH_SMEM) {
            for (int i = tid; i < SG_CUBE; i += NT)
                S.lch[i] = g[i];
        }
        for (int i = tid; i < SG_CUBE; i += NT)
            S.le[i] = 0.0;
        if (tid == 0) {
            S.ng = 0;
            S.conv = 0;
            S.bad = 0;
        }
        if (use_bulk && tid == 0) {
            if (!sg_mbar_wait(mbar, phase_bit, args.wait_limit)) {
                /* gave up: report it, then let the copy land before this
                 * CTA's shared memory is reused or released */
                atomicOr(args.err, 1u);
                if (!sg_mbar_wait(mbar, phase_bit, SG_DRAIN_LIMIT))
                    atomicOr(args.err, 2u);
                S.bad = 2;
            }
        }
        phase_bit ^= 1u;
        __syncthreads();
        if (S.bad == 2) {
            /* this codeword and the CTA's later ones are reported as not
             * decoded (converged = -2) */
            for (unsigned long long c = cw; c < args.n_cw; c += gridDim.x)
                sg_cw_not_decoded(args, c, -2);
            return;
        }
        bool nonfinite = false;
        for (int i = tid; i < SG_CUBE; i += NT)
            nonfinite |= !isfinite(LCH_SMEM ? S.lch[i] : __ldg(g + i));
        if (__syncthreads_or(nonfinite)) {
            sg_cw_not_decoded(args, cw, -1);
            __syncthreads();
            continue;
        }

        int phases = 0;
        unsigned long long ng_p = 0;
        int axis_last = 0;
        bool conv = false;
        for (int iter = 1; iter <= args.imax && !conv; iter++) {
            for (int axis = 0; axis < 3 && !conv; axis++) {
                const double alpha = args.alpha[3 * (iter - 1) + axis];
                if (tid == 0) {
                    S.line_next = 0;
                    S.ngmax = 0;
                }
                __syncthreads();
                if constexpr (LPW == 2) {
                    /* the warp takes two lines at a time, one per half, and
                     * decodes them in lockstep (sg_line16.cuh) */
                    const int hb = lane & 16, sl = lane & 15;
                    SgWarpScratch* wsl = &S.ws[2 * warp + (hb >> 4)];
                    for (;;) {
                        int l = 0;
                        if (lane == 0)
                            l = atomicAdd(&S.line_next, 2);
                        l = __shfl_sync(SG_FULL, l, 0) + (hb >> 4);
                        if (l >= 256) /* 256 lines: both halves leave together */
                            break;
                        const int pos = sg_pos(axis, l, sl);
                        const double le0 = S.le[pos];
                        const double v = __dadd_rn(LCH_SMEM ? S.lch[pos] : __ldg(g + pos), __dmul_rn(alpha, le0));
                        if (args.ckpt)
                            args.ckpt[(cw * (3ull * args.imax) + 3 * (iter - 1) + axis) * SG_CUBE + pos] = le0;
                        const SgLineResult r = sg_decode_line16<G, CR>(v, lp, args.enum_tabs, S.etab, S.ltab, wsl);
                        S.le[pos] = r.le;
                        if (args.lapp)
                            args.lapp[cw * SG_CUBE + pos] = r.lapp;
                        if (sl == 0) {
                            S.hdw[l] = (uint16_t)r.hdword;
                            atomicAdd(&S.ng, (unsigned long long)r.T);
                            atomicMax(&S.ngmax, r.T);
                        }
                    }
                } else {
                    for (;;) {
                        int l = 0;
                        if (lane == 0)
                            l = atomicAdd(&S.line_next, 1);
                        l = __shfl_sync(SG_FULL, l, 0);
                        if (l >= 256)
                            break;
                        const int pos = sg_pos(axis, l, lane & 15);
                        double v = 1.0;
                        if (lane < 16) { /* L_ch + (alpha*L_E) */
                            v = __dadd_rn(LCH_SMEM ? S.lch[pos] : __ldg(g + pos), __dmul_rn(alpha, S.le[pos]));
                            if (args.ckpt)
                                args.ckpt[(cw * (3ull * args.imax) + 3 * (iter - 1) + axis) * SG_CUBE + pos] = S.le[pos];
                        }
                        const SgLineResult r =
                            sg_decode_line<G, false, CR>(v, lp, args.enum_tabs, S.etab, S.ltab, &S.ws[warp]);
                        if (lane < 16) {
                            S.le[pos] = r.le;
                            if (args.lapp)
                                args.lapp[cw * SG_CUBE + pos] = r.lapp;
                        }
                        if (lane == 0) {
                            S.hdw[l] = (uint16_t)r.hdword;
                            atomicAdd(&S.ng, (unsigned long long)r.T);
                            atomicMax(&S.ngmax, r.T);
                        }
                    }
                }
                __syncthreads();
                phases++;
                axis_last = axis;
                ng_p += S.ngmax;
                if (warp == 0) {
                    const bool c = sg_is_codeword(S.hdw, lane);
                    if (lane == 0)
                        S.conv = c;
                }
                __syncthreads();
                conv = S.conv != 0;
            }
        }

        /* hard_decision (:393-415): info bit b = s*64 + r*8 + c is the sign of
         * L_APP at cube index s*256 + r*16 + c; packed MSB first (:272-280) */
        if (tid < SG_INFO_BYTES) {
            uint32_t byte = 0;
            for (int q = 0; q < 8; q++) {
                const int b = tid * 8 + q;
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
                byte = (byte << 1) | ((S.hdw[l] >> bit) & 1u);
            }
            args.bits[cw * SG_INFO_BYTES + tid] = (uint8_t)byte;
        }
        if (tid == 0 && args.stats) {
            sg_cw_stats st;
            st.iterations = 0.5 * phases;
            st.ng = S.ng;
            st.ng_p = ng_p;
            st.converged = conv ? 1 : 0;
            st.phases = phases;
            args.stats[cw] = st;
        }
        __syncthreads();
    }
}

#include "sg_persist.cuh"
#include "sg_adjoint.cuh"

struct SgLineSmem {
    alignas(16) double etab[SG_EXP_TAB_LEN];
    alignas(16) double ltab[SG_LOG_TAB_LEN];
    SgWarpScratch ws[SG_WARPS];
};

template <bool CR>
__global__ void __launch_bounds__(SG_THREADS) sg_bitso_kernel(const double* __restrict__ llr,
                                                               unsigned long long n_lines,
                                                               SgLineParams lp, double* lapp, double* le,
                                                               int32_t* nguess, int32_t* ncw,
                                                               const uint32_t* enum_tabs)
{
    __shared__ SgLineSmem S;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < SG_EXP_TAB_LEN; i += SG_THREADS)
        S.etab[i] = g_etab[i];
    for (int i = tid; i < SG_LOG_TAB_LEN; i += SG_THREADS)
        S.ltab[i] = g_ltab[i];
    __syncthreads();
    for (unsigned long long l = (unsigned long long)blockIdx.x * SG_WARPS + warp; l < n_lines;
         l += (unsigned long long)gridDim.x * SG_WARPS) {
        const double v = lane < 16 ? llr[l * 16 + lane] : 1.0;
        if (__any_sync(SG_FULL, !isfinite(v))) { /* not decoded: NaN out, N_guess -1 */
            if (lane < 16) {
                lapp[l * 16 + lane] = __longlong_as_double(0x7ff8000000000000ll);
                le[l * 16 + lane] = __longlong_as_double(0x7ff8000000000000ll);
            }
            if (lane == 0) {
                nguess[l] = -1;
                if (ncw)
                    ncw[l] = 0;
            }
            continue;
        }
        const SgLineResult r = sg_decode_line<1, false, CR>(v, lp, enum_tabs, S.etab, S.ltab, &S.ws[warp]);
        if (lane < 16) {
            lapp[l * 16 + lane] = r.lapp;
            le[l * 16 + lane] = r.le;
        }
        if (lane == 0) {
            nguess[l] = (int32_t)r.T;
            if (ncw)
                ncw[l] = r.ncw;
        }
    }
}

__global__ void __launch_bounds__(SG_THREADS) sg_gen_kernel(uint64_t seed, uint64_t cw0,
                                                             unsigned long long n_cw, double sigma,
                                                             double lo, double hi, uint8_t* info,
                                                             double* llr)
{
    __shared__ alignas(16) double etab[SG_EXP_TAB_LEN];
    __shared__ alignas(16) double ltab[SG_LOG_TAB_LEN];
    __shared__ uint16_t W[256];
    __shared__ alignas(16) double stage[SG_CUBE]; /* the codeword's LLRs, stored coalesced */
    __shared__ uint8_t ib[SG_INFO_BYTES];
    __shared__ uint8_t prow[8];
    __shared__ uint8_t ptab[256];
    const int tid = threadIdx.x;
    for (int i = tid; i < SG_EXP_TAB_LEN; i += SG_THREADS)
        etab[i] = g_etab[i];
    for (int i = tid; i < SG_LOG_TAB_LEN; i += SG_THREADS)
        ltab[i] = g_ltab[i];
    if (tid < 8)
        prow[tid] = c_prow[tid];
    ptab[tid] = c_ptab[tid];
    __syncthreads();
    for (unsigned long long c = blockIdx.x; c < n_cw; c += gridDim.x) {
        const uint64_t gc = cw0 + c;
        if (tid < 8) {
            const uint64_t r = sg_rand(seed, 0, gc * 8 + tid);
            for (int q = 0; q < 8; q++)
                ib[tid * 8 + q] = (uint8_t)(r >> (8 * q));
        }
        __syncthreads();
        /* sg_encode_words, each of its four stages spread over the block:
         * info words, parity columns of the first 8 slices, parity rows,
         * parity slices (the same words, every one written once) */
        if (tid < 64)
            W[(tid >> 3) * 16 + (tid & 7)] = (uint16_t)sg_brev8(ib[tid]);
        __syncthreads();
        if (tid < 64) {
            const int l = tid >> 3, jj = tid & 7;
            uint16_t acc = 0;
            for (int j = 0; j < 8; j++)
                if ((prow[j] >> jj) & 1)
                    acc ^= W[l * 16 + j];
            W[l * 16 + 8 + jj] = acc;
        }
        __syncthreads();
        if (tid < 128) {
            const uint16_t x = W[tid];
            W[tid] = (uint16_t)((x & 0xff) | (ptab[x & 0xff] << 8));
        }
        __syncthreads();
        if (tid < 128) {
            const int jj = tid >> 4, j = tid & 15;
            uint16_t acc = 0;
            for (int l = 0; l < 8; l++)
                if ((prow[l] >> jj) & 1)
                    acc ^= W[l * 16 + j];
            W[(8 + jj) * 16 + j] = acc;
        }
        if (info && tid < SG_INFO_BYTES)
            info[c * SG_INFO_BYTES + tid] = ib[tid];
        __syncthreads();
        const double s = sigma > 0.0 ? sigma : sg_sigma_draw(seed, gc, lo, hi, etab);
        /* sg_normal for this thread's 16 positions p = tid + 256k, taken as
         * one stream of polar attempts: every pass makes one attempt for every
         * lane and a lane moves to its next position when its pair is
         * accepted, so a warp no longer waits, position by position, for its
         * unluckiest lane.  Each position keeps its first accepted attempt
         * (after SG_POLAR_TRIES rejections, 0), as sg_normal does; the LLRs
         * are staged in shared memory and stored coalesced. */
        int k = 0;
        uint64_t att = 0;
        while (k < SG_CUBE / SG_THREADS) {
            const uint32_t p = (uint32_t)(tid + SG_THREADS * k);
            const uint64_t ctr = gc * 4096u + p;
            const double u = sg_sym_unit(sg_rand(seed, 1 + 2 * att, ctr));
            const double v = sg_sym_unit(sg_rand(seed, 2 + 2 * att, ctr));
            const double uu = u * u;
            const double vv = v * v;
            const double ss = uu + vv;
            const bool ok = ss > 0.0 && ss < 1.0;
            if (ok || att + 1 == SG_POLAR_TRIES) {
                double z = 0.0;
                if (ok) {
                    const double l = sg_log(ss, ltab);
                    const double m = -2.0 * l;
                    const double q = m / ss;
                    z = u * __dsqrt_rn(q);
                }
                const int bit = (W[p >> 4] >> (p & 15)) & 1;
                stage[p] = sg_llr_of(bit, s, z);
                k++;
                att = 0;
            } else {
                att++;
            }
        }
        __syncthreads();
        double* out = llr + c * SG_CUBE;
        if (((uintptr_t)llr & 15u) == 0) {
            for (int q = tid; q < SG_CUBE / 2; q += SG_THREADS)
                reinterpret_cast<double2*>(out)[q] = reinterpret_cast<const double2*>(stage)[q];
        } else {
            for (int q = tid; q < SG_CUBE; q += SG_THREADS)
                out[q] = stage[q];
        }
        __syncthreads();
    }
}

/* Reduction of per-codeword statistics and bit errors into one
 * sg_decode_summary (zeroed by the caller).  Iteration totals are sums of
 * multiples of 0.5 below 2^52, so the atomic double additions are exact and
 * the result does not depend on their order. */
__global__ void __launch_bounds__(256) sg_summary_kernel(const sg_cw_stats* __restrict__ stats,
                                                          const uint8_t* __restrict__ bits,
                                                          const uint8_t* __restrict__ ref,
                                                          unsigned long long n, const unsigned int* err,
                                                          sg_decode_summary* out)
{
    unsigned long long conv = 0, nonf = 0, tmo = 0, ng = 0, ngp = 0, be = 0, ble = 0;
    double it = 0.0;
    for (unsigned long long c = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (unsigned long long)gridDim.x * blockDim.x) {
        const sg_cw_stats st = stats[c];
        conv += st.converged == 1;
        nonf += st.converged == -1;
        tmo += st.converged == -2;
        ng += st.ng;
        ngp += st.ng_p;
        it += st.iterations;
        if (ref) {
            const uint4* a = reinterpret_cast<const uint4*>(bits + c * SG_INFO_BYTES);
            const uint4* b = reinterpret_cast<const uint4*>(ref + c * SG_INFO_BYTES);
            unsigned int e = 0;
            for (int q = 0; q < 4; q++) {
                const uint4 x = a[q], y = b[q];
                e += __popc(x.x ^ y.x) + __popc(x.y ^ y.y) + __popc(x.z ^ y.z) + __popc(x.w ^ y.w);
            }
            be += e;
            ble += e != 0;
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        conv += __shfl_xor_sync(SG_FULL, conv, off);
        nonf += __shfl_xor_sync(SG_FULL, nonf, off);
        tmo += __shfl_xor_sync(SG_FULL, tmo, off);
        ng += __shfl_xor_sync(SG_FULL, ng, off);
        ngp += __shfl_xor_sync(SG_FULL, ngp, off);
        be += __shfl_xor_sync(SG_FULL, be, off);
        ble += __shfl_xor_sync(SG_FULL, ble, off);
        it += __shfl_xor_sync(SG_FULL, it, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd((unsigned long long*)&out->converged, conv);
        atomicAdd((unsigned long long*)&out->nonfinite, nonf);
        atomicAdd((unsigned long long*)&out->timeouts, tmo);
        atomicAdd((unsigned long long*)&out->total_ng, ng);
        atomicAdd((unsigned long long*)&out->total_ng_p, ngp);
        atomicAdd((unsigned long long*)&out->bit_errors, be);
        atomicAdd((unsigned long long*)&out->block_errors, ble);
        atomicAdd(&out->total_iterations, it);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        atomicAdd((unsigned long long*)&out->blocks, n);
        if (err)
            out->device_error = *(volatile const unsigned int*)err;
        if (ref)
            atomicAdd((unsigned long long*)&out->bits_compared, n * (unsigned long long)SG_INFO_BITS);
    }
}

/* Decoder kernel configurations: warps per codeword CTA, channel cube in
 * shared memory (bulk copy) or read from global memory, minimum resident
 * CTAs per SM for the register budget, error patterns per lane per step,
 * and lines per warp (1: 32 lanes per line, sg_line.cuh; 2: 16 lanes per
 * line, sg_line16.cuh). */
struct SgVariant {
    const char* name;
    int nw;
    bool lch_smem;
    size_t smem;
    const void* fn;    /* table-driven exp/log */
    const void* fn_cr; /* correctly rounded exp/log (the reference-exact mode) */
};

#define SG_VARIANT(NW, L, M, G, NAME)                                                               \
    { NAME, NW, L, sizeof(SgCwSmem<NW, L>), (const void*)sg_decode_kernel<NW, L, M, G, false>, \
      (const void*)sg_decode_kernel<NW, L, M, G, true> }
#define SG_VARIANT_L2(NW, M, G, NAME)                                                                          \
    { NAME, NW, false, sizeof(SgCwSmem<NW, false, 2>), (const void*)sg_decode_kernel<NW, false, M, G, false, 2>, \
      (const void*)sg_decode_kernel<NW, false, M, G, true, 2> }
static const SgVariant g_variants[] = {
    SG_VARIANT(8, false, 3, 1, "w8-gmem"),
    SG_VARIANT(8, true, 2, 1, "w8-smem"),
    SG_VARIANT(12, true, 2, 1, "w12-smem"),
    SG_VARIANT(16, false, 2, 1, "w16-gmem"),
    SG_VARIANT(16, false, 2, 2, "w16-gmem-g2"),
    SG_VARIANT(8, false, 3, 2, "w8-gmem-g2"),
    SG_VARIANT(12, true, 2, 2, "w12-smem-g2"),
    SG_VARIANT_L2(8, 2, 2, "w8-l2-g2"),
    SG_VARIANT_L2(8, 2, 4, "w8-l2-g4"),
    SG_VARIANT_L2(10, 2, 2, "w10-l2-g2"),
    SG_VARIANT_L2(16, 1, 2, "w16-l2-g2"),
};
#define SG_NVARIANTS ((int)(sizeof(g_variants) / sizeof(g_variants[0])))

/* Batched persistent decoder configurations: warps per CTA (one CTA per
 * SM), codeword slots per CTA. */
struct SgPVariant {
    const char* name;
    int nw;
    int slots;
    size_t smem;
    const void* fn;    /* table-driven exp/log */
    const void* fn_cr; /* correctly rounded exp/log (the reference-exact mode) */
};
#define SG_PVARIANT(NW, C, G, NAME)                                                                \
    { NAME, NW, C, sizeof(SgPersistSmem<NW, C>), (const void*)sg_persist_kernel<NW, C, G, false>, \
      (const void*)sg_persist_kernel<NW, C, G, true> }
static const SgPVariant g_pvariants[] = {
    SG_PVARIANT(24, 3, 1, "p24x3"),
    SG_PVARIANT(28, 3, 1, "p28x3"),
    SG_PVARIANT(16, 3, 1, "p16x3"),
    SG_PVARIANT(20, 4, 1, "p20x4"),
    SG_PVARIANT(32, 3, 1, "p32x3"),
    SG_PVARIANT(32, 3, 2, "p32x3-g2"),
    SG_PVARIANT(24, 3, 2, "p24x3-g2"),
    SG_PVARIANT(28, 3, 2, "p28x3-g2"),
};
#define SG_NPVARIANTS ((int)(sizeof(g_pvariants) / sizeof(g_pvariants[0])))

/* 16-byte alignment of the shared tables (double2 loads) and of the bulk
 * copy destination, for every configuration built. */
template <class T>
constexpr bool sg_tables_aligned()
{
    return offsetof(T, etab) % 16 == 0 && offsetof(T, ltab) % 16 == 0;
}
static_assert(sg_tables_aligned<SgPersistSmem<24, 3>>() && sg_tables_aligned<SgPersistSmem<28, 3>>() &&
                  sg_tables_aligned<SgPersistSmem<16, 3>>() && sg_tables_aligned<SgPersistSmem<20, 4>>() && sg_tables_aligned<SgPersistSmem<32, 3>>() &&
                  sg_tables_aligned<SgCwSmem<8, false>>() && sg_tables_aligned<SgCwSmem<8, true>>() &&
                  sg_tables_aligned<SgCwSmem<12, true>>() && sg_tables_aligned<SgCwSmem<16, false>>() &&
                  sg_tables_aligned<SgCwSmem<8, false, 2>>() && sg_tables_aligned<SgCwSmem<10, false, 2>>() &&
                  sg_tables_aligned<SgCwSmem<16, false, 2>>() && sg_tables_aligned<SgLineSmem>(),
              "shared table alignment");
template <class T>
constexpr bool sg_bulk_aligned()
{
    return offsetof(T, lch) == 0 && offsetof(T, mbar) % 8 == 0;
}
static_assert(sg_bulk_aligned<SgCwSmem<8, true>>() && sg_bulk_aligned<SgCwSmem<12, true>>(), "bulk copy");
/* every configuration fits the 227 KB of shared memory a CTA may have */
static_assert(sizeof(SgPersistSmem<32, 3>) <= 227 * 1024 && sizeof(SgPersistSmem<28, 3>) <= 227 * 1024 &&
                  sizeof(SgPersistSmem<24, 3>) <= 227 * 1024 && sizeof(SgPersistSmem<20, 4>) <= 227 * 1024 &&
                  sizeof(SgPersistSmem<16, 3>) <= 227 * 1024 && sizeof(SgCwSmem<8, true>) <= 227 * 1024 &&
                  sizeof(SgCwSmem<16, false>) <= 227 * 1024 && sizeof(SgCwSmem<12, true>) <= 227 * 1024 &&
                  sizeof(SgCwSmem<16, false, 2>) <= 227 * 1024,
              "shared memory per CTA");
/* the two-lines-per-warp configurations built for two CTAs per SM fit them
 * (228 KB per SM, 1 KB of it reserved per CTA) */
static_assert(2 * (sizeof(SgCwSmem<8, false, 2>) + 1024) <= 228 * 1024 &&
                  2 * (sizeof(SgCwSmem<10, false, 2>) + 1024) <= 228 * 1024,
              "two CTAs per SM");

/* Static device memory of the allocation-free entry point: the error flag
 * (first 256 bytes), then per-codeword statistics and bits for at most
 * SG_NOALLOC_MAX_CW codewords; and a private copy of the pattern-order
 * tables.  Host code must not use these names as addresses: the set-up
 * below resolves them with cudaGetSymbolAddress on each device. */
#define SG_NOALLOC_HDR 256
#define SG_NOALLOC_STATS_BYTES (SG_NOALLOC_MAX_CW * sizeof(sg_cw_stats))
#define SG_NOALLOC_BYTES (SG_NOALLOC_HDR + SG_NOALLOC_STATS_BYTES + SG_NOALLOC_MAX_CW * SG_INFO_BYTES)
static __device__ __align__(256) unsigned char g_noalloc_scratch[SG_NOALLOC_BYTES];
static __device__ __align__(256) uint32_t g_noalloc_enum[SG_ENUM_NTAB * SG_ENUM_LEN];

/* One thread per IC builds that IC's pattern order (same source as the host
 * builder); ok[ic] = 1 when complete. */
__global__ void sg_enum_build_kernel(uint32_t* out, unsigned int* ok)
{
    const int ic = blockIdx.x * blockDim.x + threadIdx.x;
    if (ic < SG_ENUM_NTAB)
        ok[ic] = sg_enum_build_impl(ic, out + (size_t)ic * SG_ENUM_LEN) == SG_ENUM_LEN ? 1u : 0u;
}

/* Ceiling of the per-guess floating-point work: each thread evaluates, per
 * iteration, one path-metric addition, exp(-PM) and one P_notGuess
 * subtraction, with no memory traffic beyond the shared exp table.
 * guesses/s of this kernel over all SMs bounds what any decoder with the
 * reference's per-guess arithmetic can reach.  CR: the correctly rounded
 * exp; otherwise the table-driven sg_exp_neg. */
template <bool CR>
__global__ void __launch_bounds__(256) sg_guess_ceiling_kernel(unsigned long long iters, double* sink)
{
    __shared__ alignas(16) double etab[SG_EXP_TAB_LEN];
    for (int i = threadIdx.x; i < SG_EXP_TAB_LEN; i += 256)
        etab[i] = g_etab[i];
    __syncthreads();
    double pm0 = 1e-3 * (threadIdx.x + 1), pm1 = pm0 + 0.37, acc0 = 1.0, acc1 = 1.0;
    for (unsigned long long k = 0; k < iters; k++) {
        pm0 = __dadd_rn(pm0, 1.1e-5);
        pm1 = __dadd_rn(pm1, 1.3e-5);
        acc0 = __dsub_rn(acc0, CR ? sg_exp_cr_neg(-pm0, etab) : sg_exp_neg(-pm0, etab));
        acc1 = __dsub_rn(acc1, CR ? sg_exp_cr_neg(-pm1, etab) : sg_exp_neg(-pm1, etab));
    }
    if (acc0 + acc1 == 12345.0)
        sink[blockIdx.x] = acc0;
}

/* -------------------------------------------------------------- host -- */

namespace {

thread_local std::string t_err;

sg_status fail(sg_status s, const std::string& msg)
{
    t_err = msg;
    return s;
}

sg_status cuda_fail(cudaError_t e, const char* what)
{
    return fail(SG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define SG_CUDA(call)                         \
    do {                                      \
        cudaError_t e_ = (call);              \
        if (e_ != cudaSuccess)                \
            return cuda_fail(e_, #call);      \
    } while (0)

struct DevCtx {
    bool ready = false;
    uint32_t* enum_tabs = nullptr;
    unsigned int* err = nullptr;
    double* err_sink = nullptr; /* never-read output of the ceiling kernel */
    int sms = 0;
};

std::mutex g_mu;
std::atomic<long long> g_wait_limit{SG_WAIT_LIMIT_DEFAULT};
std::atomic<int> g_math_mode{0}; /* 0: table-driven exp/log, 1: correctly rounded */
/* Selected kernel variants, one per math mode (sogrand_b200.autotune
 * measures them): on B200 at 2 dB the table math is fastest with two error
 * patterns per lane (p32x3-g2, w16-gmem-g2), the correctly rounded math,
 * whose larger exp leaves no registers for the second pattern, with one
 * (p32x3, w16-gmem). */
int g_pvariant_by_mode[2] = {5, 4};
int g_variant_by_mode[2] = {4, 3};
#define g_pvariant (g_pvariant_by_mode[g_math_mode.load()])
#define g_variant (g_variant_by_mode[g_math_mode.load()])
DevCtx g_ctx[64];
std::vector<uint32_t> g_enum_host;
sg_code_tables g_code;
bool g_host_ready = false;

const double k_etab_host[SG_EXP_TAB_LEN] = SG_EXP_TAB_INIT;
const double k_ltab_host[SG_LOG_TAB_LEN] = SG_LOG_TAB_INIT;

sg_status host_init_locked()
{
    if (g_host_ready)
        return SG_OK;
    sg_code_build(&g_code);
    g_enum_host.assign((size_t)SG_ENUM_NTAB * SG_ENUM_LEN, 0);
    for (int ic = 0; ic < SG_ENUM_NTAB; ic++)
        if (sg_enum_build_impl(ic, g_enum_host.data() + (size_t)ic * SG_ENUM_LEN) != SG_ENUM_LEN)
            return fail(SG_ERR_ARG, "error-pattern order table incomplete");
    g_host_ready = true;
    return SG_OK;
}

sg_status get_ctx(DevCtx** out)
{
    int dev = 0;
    SG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64)
        return fail(SG_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    DevCtx& c = g_ctx[dev];
    if (!c.ready) {
        sg_status s = host_init_locked();
        if (s != SG_OK)
            return s;
        const size_t bytes = g_enum_host.size() * sizeof(uint32_t);
        SG_CUDA(cudaMalloc(&c.enum_tabs, bytes));
        SG_CUDA(cudaMemcpy(c.enum_tabs, g_enum_host.data(), bytes, cudaMemcpyHostToDevice));
        SG_CUDA(cudaMalloc(&c.err, sizeof(unsigned int)));
        SG_CUDA(cudaMalloc(&c.err_sink, 148 * 64 * sizeof(double)));
        SG_CUDA(cudaMemset(c.err, 0, sizeof(unsigned int)));
        SG_CUDA(cudaMemcpyToSymbol(c_hcol, g_code.hcol, sizeof g_code.hcol));
        SG_CUDA(cudaMemcpyToSymbol(c_prow, g_code.prow, sizeof g_code.prow));
        SG_CUDA(cudaMemcpyToSymbol(c_ptab, g_code.ptab, sizeof g_code.ptab));
        for (int v = 0; v < SG_NVARIANTS; v++) {
            SG_CUDA(cudaFuncSetAttribute(g_variants[v].fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)g_variants[v].smem));
            SG_CUDA(cudaFuncSetAttribute(g_variants[v].fn_cr, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)g_variants[v].smem));
        }
        for (int v = 0; v < SG_NPVARIANTS; v++) {
            SG_CUDA(cudaFuncSetAttribute(g_pvariants[v].fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)g_pvariants[v].smem));
            SG_CUDA(cudaFuncSetAttribute(g_pvariants[v].fn_cr, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)g_pvariants[v].smem));
        }
        SG_CUDA(cudaFuncSetAttribute(sg_backward_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(SgBackSmem<8>)));
        SG_CUDA(cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, dev));
        c.ready = true;
    }
    *out = &c;
    return SG_OK;
}

sg_status check_params(const sg_params* p)
{
    if (!p)
        return fail(SG_ERR_ARG, "params is NULL");
    if (p->L < 1 || p->L > SG_MAX_L)
        return fail(SG_ERR_ARG, "L must be in [1, 8]");
    if (p->Imax < 1 || p->Imax > SG_MAX_IMAX)
        return fail(SG_ERR_ARG, "Imax must be in [1, 50]");
    if (!(p->thres == p->thres))
        return fail(SG_ERR_ARG, "thres is NaN");
    for (int i = 0; i < 3 * p->Imax; i++)
        if (!isfinite(p->alpha[i]))
            return fail(SG_ERR_ARG, "alpha must be finite");
    return SG_OK;
}

uint32_t tmax_eff(uint64_t tmax)
{
    if (tmax == 0)
        return 0x7fffffffu; /* if (Tmax==0) Tmax=Inf, :607 */
    return tmax > 0xffffffffull ? 0xffffffffu : (uint32_t)tmax;
}

int grid_for(unsigned long long n, int cap)
{
    return (int)(n < (unsigned long long)cap ? n : (unsigned long long)cap);
}

/* Host-buffer decode through the batched persistent decoder, defined with
 * the batch handles below. */
sg_status decode_host_pipelined(const double* llr, size_t n_cw, const sg_params* p, uint8_t* bits, double* lapp,
                                sg_cw_stats* stats);
/* The file decoder's pipeline, defined with them. */
sg_status decode_file_pipelined(FILE* fi, FILE* fo, const sg_params* p, size_t chunk_cw, sg_run_summary* sum,
                                bool* any_nonfinite);

} // namespace

extern "C" {

void sg_params_default(sg_params* p)
{
    if (!p)
        return;
    memset(p, 0, sizeof *p);
    p->L = 3;
    p->Imax = 30;
    p->Tmax = UINT64_MAX;
    p->thres = 1.0 - 1e-5;
    for (int i = 0; i < SG_MAX_PHASES; i++)
        p->alpha[i] = 0.7;
}

sg_status sg_decode_device(const double* d_llr, size_t n_cw, const sg_params* p, uint8_t* d_bits,
                           double* d_lapp, sg_cw_stats* d_stats, void* stream)
{
    sg_status s = check_params(p);
    if (s != SG_OK)
        return s;
    if (n_cw == 0)
        return SG_OK;
    if (!d_llr || !d_bits)
        return fail(SG_ERR_ARG, "llr and bits must not be NULL");
    if ((uintptr_t)d_llr & 7u)
        return fail(SG_ERR_ARG, "llr must be 8-byte aligned");
    DevCtx* c = nullptr;
    if ((s = get_ctx(&c)) != SG_OK)
        return s;
    SgDecodeArgs a;
    memset(&a, 0, sizeof a);
    a.llr = d_llr;
    a.bits = d_bits;
    a.lapp = d_lapp;
    a.stats = d_stats;
    a.enum_tabs = c->enum_tabs;
    a.err = c->err;
    a.n_cw = n_cw;
    a.wait_limit = g_wait_limit.load();
    a.L = p->L;
    a.imax = p->Imax;
    a.tmax = tmax_eff(p->Tmax);
    a.use_bulk = ((uintptr_t)d_llr & 15u) == 0;
    a.thres = p->thres;
    memcpy(a.alpha, p->alpha, sizeof a.alpha);
    const SgVariant& v = g_variants[g_variant];
    const int grid = grid_for(n_cw, 1 << 30);
    void* kargs[] = {(void*)&a};
    SG_CUDA(cudaLaunchKernel(g_math_mode.load() ? v.fn_cr : v.fn, dim3(grid), dim3(v.nw * 32), kargs, v.smem,
                             (cudaStream_t)stream));
    return SG_OK;
}

sg_status sg_bitso_device(const double* d_llr, size_t n_lines, int32_t L, uint64_t Tmax, double thres,
                          double* d_lapp, double* d_le, int32_t* d_nguess, int32_t* d_ncw, void* stream)
{
    if (L < 1 || L > SG_MAX_L)
        return fail(SG_ERR_ARG, "L must be in [1, 8]");
    if (n_lines == 0)
        return SG_OK;
    if (!d_llr || !d_lapp || !d_le || !d_nguess)
        return fail(SG_ERR_ARG, "NULL buffer");
    DevCtx* c = nullptr;
    sg_status s = get_ctx(&c);
    if (s != SG_OK)
        return s;
    SgLineParams lp;
    lp.L = L;
    lp.tmax = tmax_eff(Tmax);
    lp.thres = thres;
    const unsigned long long blocks = (n_lines + SG_WARPS - 1) / SG_WARPS;
    if (g_math_mode.load())
        sg_bitso_kernel<true><<<grid_for(blocks, 148 * 64), SG_THREADS, 0, (cudaStream_t)stream>>>(
            d_llr, n_lines, lp, d_lapp, d_le, d_nguess, d_ncw, c->enum_tabs);
    else
        sg_bitso_kernel<false><<<grid_for(blocks, 148 * 64), SG_THREADS, 0, (cudaStream_t)stream>>>(
            d_llr, n_lines, lp, d_lapp, d_le, d_nguess, d_ncw, c->enum_tabs);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

sg_status sg_bitso_host(const double* llr, size_t n_lines, int32_t L, uint64_t Tmax, double thres,
                        double* lapp, double* le, int32_t* nguess, int32_t* ncw)
{
    if (n_lines == 0)
        return SG_OK;
    if (!llr || !lapp || !le || !nguess)
        return fail(SG_ERR_ARG, "NULL buffer");
    double *dl = nullptr, *da = nullptr, *de = nullptr;
    int32_t *dn = nullptr, *dc = nullptr;
    const size_t vb = n_lines * 16 * sizeof(double), ib = n_lines * sizeof(int32_t);
    sg_status s = SG_OK;
    cudaError_t e;
    if ((e = cudaMalloc(&dl, vb)) != cudaSuccess || (e = cudaMalloc(&da, vb)) != cudaSuccess ||
        (e = cudaMalloc(&de, vb)) != cudaSuccess || (e = cudaMalloc(&dn, ib)) != cudaSuccess ||
        (e = cudaMalloc(&dc, ib)) != cudaSuccess) {
        s = cuda_fail(e, "cudaMalloc");
    } else if ((e = cudaMemcpy(dl, llr, vb, cudaMemcpyHostToDevice)) != cudaSuccess) {
        s = cuda_fail(e, "cudaMemcpy H2D");
    } else if ((s = sg_bitso_device(dl, n_lines, L, Tmax, thres, da, de, dn, dc, nullptr)) == SG_OK) {
        if ((e = cudaDeviceSynchronize()) != cudaSuccess ||
            (e = cudaMemcpy(lapp, da, vb, cudaMemcpyDeviceToHost)) != cudaSuccess ||
            (e = cudaMemcpy(le, de, vb, cudaMemcpyDeviceToHost)) != cudaSuccess ||
            (e = cudaMemcpy(nguess, dn, ib, cudaMemcpyDeviceToHost)) != cudaSuccess ||
            (ncw && (e = cudaMemcpy(ncw, dc, ib, cudaMemcpyDeviceToHost)) != cudaSuccess))
            s = cuda_fail(e, "bitso copy-out");
    }
    cudaFree(dl);
    cudaFree(da);
    cudaFree(de);
    cudaFree(dn);
    cudaFree(dc);
    return s;
}

sg_status sg_decode_host(const double* llr, size_t n_cw, const sg_params* p, uint8_t* bits, double* lapp,
                         sg_cw_stats* stats)
{
    sg_status s = check_params(p);
    if (s != SG_OK)
        return s;
    if (n_cw == 0)
        return SG_OK;
    if (!llr || !bits)
        return fail(SG_ERR_ARG, "llr and bits must not be NULL");
    return decode_host_pipelined(llr, n_cw, p, bits, lapp, stats);
}

sg_status sg_decode_file(const char* in_path, const char* out_path, const sg_params* p, size_t chunk_cw,
                         sg_run_summary* summary)
{
    sg_status s = check_params(p);
    if (s != SG_OK)
        return s;
    if (!in_path || !out_path)
        return fail(SG_ERR_ARG, "NULL path");
    const auto t0 = std::chrono::steady_clock::now();
    FILE* fi = fopen(in_path, "rb");
    if (!fi)
        return fail(SG_ERR_IO, std::string("Error opening input file: ") + strerror(errno));
    FILE* fo = fopen(out_path, "wb");
    if (!fo) {
        fclose(fi);
        return fail(SG_ERR_IO, std::string("Error opening output file: ") + strerror(errno));
    }
    sg_run_summary sum;
    memset(&sum, 0, sizeof sum);
    bool nonfinite = false;
    s = decode_file_pipelined(fi, fo, p, chunk_cw, &sum, &nonfinite);
    fclose(fi);
    if (fclose(fo) != 0 && s == SG_OK)
        s = fail(SG_ERR_IO, "error closing output file");
    if (s == SG_OK && nonfinite)
        s = fail(SG_ERR_NONFINITE, "input contains non-finite LLRs; those codewords were not decoded");
    sum.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (summary)
        *summary = sum;
    return s;
}

double sg_channel_sigma(double ebn0_db)
{
    const int n = 16, k = 8;
    const double R = pow((double)k / n, 3);
    const double es = ebn0_db + 10 * log10(2 * R);
    return 1.0 / sqrt(pow(10, es / 10.0));
}

sg_status sg_gen_info_host(uint64_t seed, uint64_t cw0, size_t n_cw, uint8_t* info)
{
    if (!info && n_cw)
        return fail(SG_ERR_ARG, "info is NULL");
    for (size_t c = 0; c < n_cw; c++)
        for (int w = 0; w < 8; w++) {
            const uint64_t r = sg_rand(seed, 0, (cw0 + c) * 8 + w);
            for (int q = 0; q < 8; q++)
                info[c * SG_INFO_BYTES + w * 8 + q] = (uint8_t)(r >> (8 * q));
        }
    return SG_OK;
}

sg_status sg_encode_host(const uint8_t* info, size_t n_cw, uint8_t* code_bits)
{
    if ((!info || !code_bits) && n_cw)
        return fail(SG_ERR_ARG, "NULL buffer");
    {
        std::lock_guard<std::mutex> lk(g_mu);
        sg_status s = host_init_locked();
        if (s != SG_OK)
            return s;
    }
    uint16_t W[256];
    for (size_t c = 0; c < n_cw; c++) {
        sg_encode_words(info + c * SG_INFO_BYTES, g_code.prow, g_code.ptab, W);
        for (int p = 0; p < SG_CUBE; p++)
            code_bits[c * SG_CUBE + p] = (uint8_t)((W[p >> 4] >> (p & 15)) & 1);
    }
    return SG_OK;
}

sg_status sg_gen_llr_host(uint64_t seed, uint64_t cw0, size_t n_cw, double sigma, double ebn0_lo_db,
                          double ebn0_hi_db, uint8_t* info, double* llr)
{
    if (!llr && n_cw)
        return fail(SG_ERR_ARG, "llr is NULL");
    {
        std::lock_guard<std::mutex> lk(g_mu);
        sg_status s = host_init_locked();
        if (s != SG_OK)
            return s;
    }
    uint8_t ib[SG_INFO_BYTES];
    uint16_t W[256];
    for (size_t c = 0; c < n_cw; c++) {
        const uint64_t gc = cw0 + c;
        sg_gen_info_host(seed, gc, 1, ib);
        if (info)
            memcpy(info + c * SG_INFO_BYTES, ib, SG_INFO_BYTES);
        sg_encode_words(ib, g_code.prow, g_code.ptab, W);
        const double s = sigma > 0.0 ? sigma : sg_sigma_draw(seed, gc, ebn0_lo_db, ebn0_hi_db, k_etab_host);
        for (int p = 0; p < SG_CUBE; p++) {
            const int bit = (W[p >> 4] >> (p & 15)) & 1;
            llr[c * SG_CUBE + p] = sg_llr_of(bit, s, sg_normal(seed, gc, (uint32_t)p, k_ltab_host));
        }
    }
    return SG_OK;
}

sg_status sg_gen_llr_device(uint64_t seed, uint64_t cw0, size_t n_cw, double sigma, double ebn0_lo_db,
                            double ebn0_hi_db, uint8_t* d_info, double* d_llr, void* stream)
{
    if (n_cw == 0)
        return SG_OK;
    if (!d_llr)
        return fail(SG_ERR_ARG, "llr is NULL");
    if ((uintptr_t)d_llr & 7u)
        return fail(SG_ERR_ARG, "llr must be 8-byte aligned");
    DevCtx* c = nullptr;
    sg_status s = get_ctx(&c);
    if (s != SG_OK)
        return s;
    sg_gen_kernel<<<grid_for(n_cw, 148 * 16), SG_THREADS, 0, (cudaStream_t)stream>>>(
        seed, cw0, n_cw, sigma, ebn0_lo_db, ebn0_hi_db, d_info, d_llr);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

size_t sg_pattern_order(int32_t ic, uint32_t* out, size_t cap)
{
    if (ic < 0 || !out)
        return 0;
    std::vector<uint32_t> t(SG_ENUM_LEN);
    const size_t n = sg_enum_build_impl(ic, t.data());
    const size_t m = n < cap ? n : cap;
    for (size_t i = 0; i < m; i++)
        out[i] = sg_ent_pattern(t[i]) | (t[i] & SG_ENUM_GS);
    return m;
}

sg_status sg_decode_summary_device(const double* d_llr, size_t n_cw, const sg_params* p,
                                   const uint8_t* d_ref_info, uint8_t* d_bits, sg_decode_summary* d_summary,
                                   void* stream)
{
    if (!d_summary)
        return fail(SG_ERR_ARG, "summary must not be NULL");
    if (d_ref_info && ((uintptr_t)d_ref_info & 15u))
        return fail(SG_ERR_ARG, "ref_info must be 16-byte aligned");
    if (d_bits && ((uintptr_t)d_bits & 15u))
        return fail(SG_ERR_ARG, "bits must be 16-byte aligned");
    sg_status s = check_params(p);
    if (s != SG_OK)
        return s;
    cudaStream_t st = (cudaStream_t)stream;
    SG_CUDA(cudaMemsetAsync(d_summary, 0, sizeof(sg_decode_summary), st));
    if (n_cw == 0)
        return SG_OK;
    const size_t stat_bytes = ((n_cw * sizeof(sg_cw_stats) + 255) / 256) * 256;
    const size_t bit_bytes = d_bits ? 0 : n_cw * SG_INFO_BYTES;
    unsigned char* scratch = nullptr;
    SG_CUDA(cudaMallocAsync((void**)&scratch, stat_bytes + bit_bytes, st));
    sg_cw_stats* stats = reinterpret_cast<sg_cw_stats*>(scratch);
    uint8_t* bits = d_bits ? d_bits : scratch + stat_bytes;
    s = sg_decode_device(d_llr, n_cw, p, bits, nullptr, stats, stream);
    if (s == SG_OK) {
        DevCtx* c = nullptr;
        if ((s = get_ctx(&c)) == SG_OK) {
            sg_summary_kernel<<<grid_for((n_cw + 255) / 256, 148 * 8), 256, 0, st>>>(stats, bits, d_ref_info,
                                                                                      n_cw, c->err, d_summary);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess)
                s = cuda_fail(e, "summary kernel");
        }
    }
    cudaError_t e = cudaFreeAsync(scratch, st);
    if (s == SG_OK && e != cudaSuccess)
        s = cuda_fail(e, "cudaFreeAsync");
    return s;
}

sg_status sg_wilson_interval(uint64_t k, uint64_t n, double z, double* lo, double* hi)
{
    if (!lo || !hi || n == 0 || k > n || !(z > 0))
        return fail(SG_ERR_ARG, "wilson interval needs 0 <= k <= n, n > 0, z > 0");
    const double nn = (double)n, ph = (double)k / nn, z2 = z * z;
    const double den = 1.0 + z2 / nn;
    const double c = (ph + z2 / (2 * nn)) / den;
    const double h = z * sqrt(ph * (1 - ph) / nn + z2 / (4 * nn * nn)) / den;
    *lo = (k == 0 || c - h < 0) ? 0.0 : c - h;
    *hi = (k == n || c + h > 1) ? 1.0 : c + h;
    return SG_OK;
}

namespace {

struct NoAllocCtx {
    bool ready = false;
    unsigned char* scratch = nullptr; /* device address of g_noalloc_scratch */
    uint32_t* enum_tabs = nullptr;    /* device address of g_noalloc_enum */
};
NoAllocCtx g_noalloc[64];

/* Once per device, with that device current: resolve the static arrays'
 * device addresses, load the code tables, build the pattern orders on the
 * device, allow the decode kernels their shared memory.  No allocation. */
sg_status noalloc_setup(NoAllocCtx** out)
{
    int dev = 0;
    SG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64)
        return fail(SG_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    NoAllocCtx& c = g_noalloc[dev];
    if (!c.ready) {
        sg_code_tables code;
        sg_code_build(&code);
        SG_CUDA(cudaGetSymbolAddress((void**)&c.scratch, g_noalloc_scratch));
        SG_CUDA(cudaGetSymbolAddress((void**)&c.enum_tabs, g_noalloc_enum));
        SG_CUDA(cudaMemcpyToSymbol(c_hcol, code.hcol, sizeof code.hcol));
        SG_CUDA(cudaMemcpyToSymbol(c_prow, code.prow, sizeof code.prow));
        SG_CUDA(cudaMemcpyToSymbol(c_ptab, code.ptab, sizeof code.ptab));
        for (int v = 0; v < SG_NVARIANTS; v++) {
            SG_CUDA(cudaFuncSetAttribute(g_variants[v].fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)g_variants[v].smem));
            SG_CUDA(cudaFuncSetAttribute(g_variants[v].fn_cr, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)g_variants[v].smem));
        }
        /* the completion flags of the build borrow the scratch array */
        unsigned int* ok = reinterpret_cast<unsigned int*>(c.scratch);
        SG_CUDA(cudaMemset(ok, 0, SG_ENUM_NTAB * sizeof(unsigned int)));
        sg_enum_build_kernel<<<1, 64>>>(c.enum_tabs, ok);
        SG_CUDA(cudaGetLastError());
        unsigned int hok[SG_ENUM_NTAB];
        SG_CUDA(cudaMemcpy(hok, ok, sizeof hok, cudaMemcpyDeviceToHost));
        for (int i = 0; i < SG_ENUM_NTAB; i++)
            if (hok[i] != 1u)
                return fail(SG_ERR_ARG, "device pattern-order build incomplete");
        c.ready = true;
    }
    *out = &c;
    return SG_OK;
}

} // namespace

sg_status sg_decode_summary_device_noalloc(const double* d_llr, size_t n_cw, const sg_params* p,
                                           const uint8_t* d_ref_info, uint8_t* d_bits,
                                           sg_decode_summary* d_summary, void* stream)
{
    if (!d_summary)
        return fail(SG_ERR_ARG, "summary must not be NULL");
    if (n_cw > SG_NOALLOC_MAX_CW)
        return fail(SG_ERR_ARG, "n_cw exceeds SG_NOALLOC_MAX_CW (16384) for the allocation-free entry point");
    if (d_ref_info && ((uintptr_t)d_ref_info & 15u))
        return fail(SG_ERR_ARG, "ref_info must be 16-byte aligned");
    if (d_bits && ((uintptr_t)d_bits & 15u))
        return fail(SG_ERR_ARG, "bits must be 16-byte aligned");
    if (n_cw && !d_llr)
        return fail(SG_ERR_ARG, "llr must not be NULL");
    if ((uintptr_t)d_llr & 7u)
        return fail(SG_ERR_ARG, "llr must be 8-byte aligned");
    sg_status s = check_params(p);
    if (s != SG_OK)
        return s;
    NoAllocCtx* c = nullptr;
    if ((s = noalloc_setup(&c)) != SG_OK)
        return s;
    cudaStream_t st = (cudaStream_t)stream;
    SG_CUDA(cudaMemsetAsync(d_summary, 0, sizeof(sg_decode_summary), st));
    if (n_cw == 0)
        return SG_OK;
    /* the scratch keeps the previous call's contents: clear the error flag;
     * statistics and bits are overwritten for every codeword */
    unsigned int* err = reinterpret_cast<unsigned int*>(c->scratch);
    sg_cw_stats* stats = reinterpret_cast<sg_cw_stats*>(c->scratch + SG_NOALLOC_HDR);
    uint8_t* bits = d_bits ? d_bits : c->scratch + SG_NOALLOC_HDR + SG_NOALLOC_STATS_BYTES;
    SG_CUDA(cudaMemsetAsync(err, 0, sizeof(unsigned int), st));
    SgDecodeArgs a;
    memset(&a, 0, sizeof a);
    a.llr = d_llr;
    a.bits = bits;
    a.lapp = nullptr;
    a.stats = stats;
    a.enum_tabs = c->enum_tabs;
    a.err = err;
    a.n_cw = n_cw;
    a.wait_limit = g_wait_limit.load();
    a.L = p->L;
    a.imax = p->Imax;
    a.tmax = tmax_eff(p->Tmax);
    a.use_bulk = ((uintptr_t)d_llr & 15u) == 0;
    a.thres = p->thres;
    memcpy(a.alpha, p->alpha, sizeof a.alpha);
    const SgVariant& v = g_variants[g_variant];
    void* kargs[] = {(void*)&a};
    SG_CUDA(cudaLaunchKernel(g_math_mode.load() ? v.fn_cr : v.fn, dim3(grid_for(n_cw, 1 << 30)),
                             dim3(v.nw * 32), kargs, v.smem, st));
    sg_summary_kernel<<<grid_for((n_cw + 255) / 256, 148 * 8), 256, 0, st>>>(stats, bits, d_ref_info, n_cw, err,
                                                                              d_summary);
    SG_CUDA(cudaGetLastError());
    return SG_OK;
}

} // extern "C"

struct sg_batch_s {
    int device = -1;
    SgQueue* q = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

sg_status batch_enqueue(sg_batch b, const double* d_llr, size_t n_cw, const sg_params* p, uint8_t* d_bits,
                        double* d_lapp, sg_cw_stats* d_stats, cudaStream_t st)
{
    sg_status s = check_params(p);
    if (s != SG_OK)
        return s;
    if (!b || !b->q)
        return fail(SG_ERR_ARG, "invalid batch handle");
    if (n_cw && (!d_llr || !d_bits))
        return fail(SG_ERR_ARG, "llr and bits must not be NULL");
    if ((uintptr_t)d_llr & 7u)
        return fail(SG_ERR_ARG, "llr must be 8-byte aligned");
    int dev = 0;
    SG_CUDA(cudaGetDevice(&dev));
    if (dev != b->device)
        return fail(SG_ERR_ARG, "batch handle belongs to another device");
    DevCtx* c = nullptr;
    if ((s = get_ctx(&c)) != SG_OK)
        return s;
    SG_CUDA(cudaMemsetAsync(b->q, 0, sizeof(SgQueue), st));
    if (n_cw == 0)
        return SG_OK;
    SgDecodeArgs a;
    memset(&a, 0, sizeof a);
    a.llr = d_llr;
    a.bits = d_bits;
    a.lapp = d_lapp;
    a.stats = d_stats;
    a.enum_tabs = c->enum_tabs;
    a.err = c->err;
    a.n_cw = n_cw;
    a.wait_limit = g_wait_limit.load();
    a.L = p->L;
    a.imax = p->Imax;
    a.tmax = tmax_eff(p->Tmax);
    a.use_bulk = 0;
    a.thres = p->thres;
    memcpy(a.alpha, p->alpha, sizeof a.alpha);
    const SgPVariant& v = g_pvariants[g_pvariant];
    SgQueue* q = b->q;
    void* kargs[] = {(void*)&a, (void*)&q};
    const int grid = (int)(n_cw < (size_t)c->sms ? n_cw : (size_t)c->sms);
    SG_CUDA(cudaLaunchKernel(g_math_mode.load() ? v.fn_cr : v.fn, dim3(grid), dim3(v.nw * 32), kargs, v.smem,
                             st));
    return SG_OK;
}

/* One half of the host-buffer pipeline: device buffers for one chunk, its
 * stream and its work queue. */
struct HostLane {
    double* dl = nullptr;
    double* da = nullptr;
    uint8_t* db = nullptr;
    sg_cw_stats* dst = nullptr;
    cudaStream_t st = nullptr;
    sg_batch_s b;
    size_t off = 0, n = 0;
};

/* Device resources of the host-buffer pipeline, kept per device across
 * calls so that a call allocates nothing after the first: two lanes of
 * chunk buffers, their streams and work queues.  Calls on one device are
 * serialised by the mutex. */
constexpr int SG_HOST_LANES = 2;
constexpr size_t SG_HOST_CHUNK = 16384;
/* Pinned host staging of the file decoder: SG_FILE_BUFS chunks of LLR cubes
 * (a reader thread fills one while the lanes decode the others) and the
 * bits and statistics of each lane's chunk. */
constexpr size_t SG_FILE_CHUNK = 8192;
constexpr int SG_FILE_BUFS = 3;
struct FileStage {
    double* llr[SG_FILE_BUFS] = {};
    uint8_t* bits[SG_HOST_LANES] = {};
    sg_cw_stats* st[SG_HOST_LANES] = {};
    bool ready = false;
};
struct HostPipe {
    std::mutex mu;
    HostLane ln[SG_HOST_LANES];
    bool ready = false;     /* buffers (without L_APP), streams and queues */
    bool has_lapp = false;  /* L_APP buffers too */
    FileStage fs;           /* pinned staging, allocated by the first file decode */
};
constexpr int SG_HOST_MAX_DEV = 64;
HostPipe g_host_pipe[SG_HOST_MAX_DEV];

sg_status host_pipe_setup(HostPipe& hp, int dev, bool want_lapp)
{
    cudaError_t e = cudaSuccess;
    if (!hp.ready) {
        for (HostLane& L : hp.ln) {
            L.b.device = dev;
            if ((e = cudaMalloc(&L.dl, SG_HOST_CHUNK * SG_CUBE * sizeof(double))) != cudaSuccess ||
                (e = cudaMalloc(&L.db, SG_HOST_CHUNK * SG_INFO_BYTES)) != cudaSuccess ||
                (e = cudaMalloc(&L.dst, SG_HOST_CHUNK * sizeof(sg_cw_stats))) != cudaSuccess ||
                (e = cudaMalloc(&L.b.q, sizeof(SgQueue))) != cudaSuccess ||
                (e = cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking)) != cudaSuccess)
                break;
        }
        if (e != cudaSuccess) { /* undo a partial set-up; the next call retries */
            for (HostLane& L : hp.ln) {
                cudaFree(L.dl);
                cudaFree(L.db);
                cudaFree(L.dst);
                cudaFree(L.b.q);
                if (L.st)
                    cudaStreamDestroy(L.st);
                L = HostLane();
            }
            return cuda_fail(e, "host pipeline buffers");
        }
        hp.ready = true;
    }
    if (want_lapp && !hp.has_lapp) {
        for (HostLane& L : hp.ln)
            if ((e = cudaMalloc(&L.da, SG_HOST_CHUNK * SG_CUBE * sizeof(double))) != cudaSuccess)
                break;
        if (e != cudaSuccess) {
            for (HostLane& L : hp.ln) {
                cudaFree(L.da);
                L.da = nullptr;
            }
            return cuda_fail(e, "host pipeline L_APP buffers");
        }
        hp.has_lapp = true;
    }
    return SG_OK;
}

/* Chunks of at most 16384 codewords (512 MiB of LLRs) alternate between the
 * two lanes: while chunk k decodes, chunk k + 1 is copied in and queued
 * behind it, so copies overlap decoding and the next chunk's CTAs take each
 * SM as soon as the current chunk's CTA there runs out of work.  Results
 * are read back chunk by chunk in order; a lane is refilled only after its
 * chunk has been read back. */
sg_status decode_host_pipelined(const double* llr, size_t n_cw, const sg_params* p, uint8_t* bits, double* lapp,
                                sg_cw_stats* stats)
{
    const size_t chunk = n_cw < SG_HOST_CHUNK ? n_cw : SG_HOST_CHUNK;
    const size_t nk = (n_cw + chunk - 1) / chunk;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= SG_HOST_MAX_DEV)
        return fail(SG_ERR_ARG, "device index beyond the host pipeline's table");
    HostPipe& hp = g_host_pipe[dev];
    std::lock_guard<std::mutex> lk(hp.mu);
    sg_status s = host_pipe_setup(hp, dev, lapp != nullptr);
    if (s != SG_OK)
        return s;
    HostLane* ln = hp.ln;
    std::vector<sg_cw_stats> hst(chunk);
    bool any_nonfinite = false;
    auto enqueue = [&](size_t k) -> sg_status {
        HostLane& L = ln[k % SG_HOST_LANES];
        L.off = k * chunk;
        L.n = (n_cw - L.off) < chunk ? (n_cw - L.off) : chunk;
        SG_CUDA(cudaMemcpyAsync(L.dl, llr + L.off * SG_CUBE, L.n * SG_CUBE * sizeof(double), cudaMemcpyHostToDevice,
                                L.st));
        return batch_enqueue(&L.b, L.dl, L.n, p, L.db, lapp ? L.da : nullptr, L.dst, L.st);
    };
    auto drain = [&](size_t k) -> sg_status {
        HostLane& L = ln[k % SG_HOST_LANES];
        SgQueue hq;
        SG_CUDA(cudaMemcpyAsync(bits + L.off * SG_INFO_BYTES, L.db, L.n * SG_INFO_BYTES, cudaMemcpyDeviceToHost,
                                L.st));
        SG_CUDA(cudaMemcpyAsync(hst.data(), L.dst, L.n * sizeof(sg_cw_stats), cudaMemcpyDeviceToHost, L.st));
        if (lapp)
            SG_CUDA(cudaMemcpyAsync(lapp + L.off * SG_CUBE, L.da, L.n * SG_CUBE * sizeof(double),
                                    cudaMemcpyDeviceToHost, L.st));
        SG_CUDA(cudaMemcpyAsync(&hq, L.b.q, sizeof hq, cudaMemcpyDeviceToHost, L.st));
        SG_CUDA(cudaStreamSynchronize(L.st));
        if (hq.err)
            return fail(SG_ERR_TIMEOUT, "a persistent-decoder warp gave up waiting for work");
        for (size_t i = 0; i < L.n; i++)
            any_nonfinite |= hst[i].converged < 0;
        if (stats)
            memcpy(stats + L.off, hst.data(), L.n * sizeof(sg_cw_stats));
        return SG_OK;
    };
    for (size_t k = 0; k < (size_t)SG_HOST_LANES && k < nk && s == SG_OK; k++)
        s = enqueue(k);
    for (size_t k = 0; k < nk && s == SG_OK; k++) {
        if ((s = drain(k)) != SG_OK)
            break;
        if (k + SG_HOST_LANES < nk)
            s = enqueue(k + SG_HOST_LANES);
    }
    /* leave no work of this call running on the lanes' streams */
    for (HostLane& L : hp.ln)
        cudaStreamSynchronize(L.st);
    if (s == SG_OK && any_nonfinite)
        return fail(SG_ERR_NONFINITE, "input contains non-finite LLRs; those codewords were not decoded");
    return s;
}

sg_status file_stage_setup(FileStage& fs)
{
    if (fs.ready)
        return SG_OK;
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < SG_FILE_BUFS && e == cudaSuccess; b++)
        e = cudaHostAlloc((void**)&fs.llr[b], SG_FILE_CHUNK * SG_CUBE * sizeof(double), cudaHostAllocDefault);
    for (int l = 0; l < SG_HOST_LANES && e == cudaSuccess; l++) {
        e = cudaHostAlloc((void**)&fs.bits[l], SG_FILE_CHUNK * SG_INFO_BYTES, cudaHostAllocDefault);
        if (e == cudaSuccess)
            e = cudaHostAlloc((void**)&fs.st[l], SG_FILE_CHUNK * sizeof(sg_cw_stats), cudaHostAllocDefault);
    }
    if (e != cudaSuccess) {
        for (int b = 0; b < SG_FILE_BUFS; b++)
            cudaFreeHost(fs.llr[b]);
        for (int l = 0; l < SG_HOST_LANES; l++) {
            cudaFreeHost(fs.bits[l]);
            cudaFreeHost(fs.st[l]);
        }
        fs = FileStage();
        return cuda_fail(e, "pinned staging buffers of the file decoder");
    }
    fs.ready = true;
    return SG_OK;
}

/* The file decoder's pipeline.  A reader thread fills pinned staging
 * buffers with chunks of whole cubes (fread, as the reference's loop reads
 * them; a trailing partial cube is ignored); the calling thread copies each
 * chunk to a lane of the host pipeline, decodes it with the batched decoder
 * and copies bits and statistics back, alternating between the two lanes,
 * and writes a chunk's bits when its lane is taken again (chunks are
 * written in order).  File reading, both copy directions and decoding
 * overlap.  chunk_cw: codewords per chunk, 0 or above SG_FILE_CHUNK for
 * SG_FILE_CHUNK. */
sg_status decode_file_pipelined(FILE* fi, FILE* fo, const sg_params* p, size_t chunk_cw, sg_run_summary* sum,
                                bool* any_nonfinite)
{
    const size_t chunk = (chunk_cw == 0 || chunk_cw > SG_FILE_CHUNK) ? SG_FILE_CHUNK : chunk_cw;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= SG_HOST_MAX_DEV)
        return fail(SG_ERR_ARG, "device index beyond the host pipeline's table");
    HostPipe& hp = g_host_pipe[dev];
    std::lock_guard<std::mutex> lk(hp.mu);
    sg_status s = host_pipe_setup(hp, dev, false);
    if (s == SG_OK)
        s = file_stage_setup(hp.fs);
    if (s != SG_OK)
        return s;
    FileStage& fs = hp.fs;

    /* reader: chunk k goes to buffer k % SG_FILE_BUFS once the chunk that
     * used it before has been decoded and read back */
    std::mutex m;
    std::condition_variable cv;
    size_t count[SG_FILE_BUFS] = {};
    bool full[SG_FILE_BUFS] = {};
    bool stop = false, read_err = false;
    std::thread reader([&] {
        for (size_t k = 0;; k++) {
            const int b = (int)(k % SG_FILE_BUFS);
            {
                std::unique_lock<std::mutex> ul(m);
                cv.wait(ul, [&] { return !full[b] || stop; });
                if (stop)
                    return;
            }
            const size_t got = fread(fs.llr[b], sizeof(double) * SG_CUBE, chunk, fi);
            const bool err = got < chunk && ferror(fi);
            {
                std::lock_guard<std::mutex> g(m);
                count[b] = got;
                full[b] = true;
                read_err = read_err || err;
            }
            cv.notify_all();
            if (got < chunk)
                return; /* end of file, or a read error */
        }
    });

    HostLane* ln = hp.ln;
    long pending[SG_HOST_LANES] = {-1, -1}; /* chunk held by each lane */
    size_t pend_n[SG_HOST_LANES] = {0, 0};
    auto drain = [&](int l) -> sg_status {
        if (pending[l] < 0)
            return SG_OK;
        HostLane& L = ln[l];
        SgQueue hq;
        SG_CUDA(cudaMemcpyAsync(&hq, L.b.q, sizeof hq, cudaMemcpyDeviceToHost, L.st));
        SG_CUDA(cudaStreamSynchronize(L.st));
        const size_t n = pend_n[l];
        {
            std::lock_guard<std::mutex> g(m);
            full[pending[l] % SG_FILE_BUFS] = false; /* its input buffer is free again */
        }
        cv.notify_all();
        pending[l] = -1;
        if (hq.err)
            return fail(SG_ERR_TIMEOUT, "a persistent-decoder warp gave up waiting for work");
        if (fwrite(fs.bits[l], SG_INFO_BYTES, n, fo) != n)
            return fail(SG_ERR_IO, "short write to output file");
        for (size_t i = 0; i < n; i++) {
            const sg_cw_stats& c = fs.st[l][i];
            *any_nonfinite |= c.converged < 0;
            sum->total_iterations += c.iterations;
            sum->total_ng += c.ng;
            sum->total_ng_p += c.ng_p;
        }
        sum->blocks += n;
        return SG_OK;
    };
    for (size_t k = 0; s == SG_OK; k++) {
        const int b = (int)(k % SG_FILE_BUFS), l = (int)(k % SG_HOST_LANES);
        size_t n;
        {
            std::unique_lock<std::mutex> ul(m);
            cv.wait(ul, [&] { return full[b]; });
            n = count[b];
        }
        if ((s = drain(l)) != SG_OK)
            break;
        if (n == 0)
            break;
        HostLane& L = ln[l];
        cudaError_t ce = cudaMemcpyAsync(L.dl, fs.llr[b], n * SG_CUBE * sizeof(double), cudaMemcpyHostToDevice,
                                         L.st);
        if (ce != cudaSuccess) {
            s = cuda_fail(ce, "cudaMemcpyAsync H2D");
            break;
        }
        if ((s = batch_enqueue(&L.b, L.dl, n, p, L.db, nullptr, L.dst, L.st)) != SG_OK)
            break;
        if ((ce = cudaMemcpyAsync(fs.bits[l], L.db, n * SG_INFO_BYTES, cudaMemcpyDeviceToHost, L.st)) !=
                cudaSuccess ||
            (ce = cudaMemcpyAsync(fs.st[l], L.dst, n * sizeof(sg_cw_stats), cudaMemcpyDeviceToHost, L.st)) !=
                cudaSuccess) {
            s = cuda_fail(ce, "cudaMemcpyAsync D2H");
            break;
        }
        pending[l] = (long)k;
        pend_n[l] = n;
        if (n < chunk)
            break; /* the last chunk */
    }
    /* the lanes' remaining chunks, in order */
    const int first = (pending[0] >= 0 && (pending[1] < 0 || pending[0] < pending[1])) ? 0 : 1;
    for (int i = 0; i < SG_HOST_LANES; i++) {
        const sg_status d = drain((first + i) % SG_HOST_LANES);
        if (s == SG_OK)
            s = d;
    }
    {
        std::lock_guard<std::mutex> g(m);
        stop = true;
    }
    cv.notify_all();
    reader.join();
    for (HostLane& L : hp.ln)
        cudaStreamSynchronize(L.st);
    if (s == SG_OK && read_err)
        s = fail(SG_ERR_IO, "read error on input file");
    return s;
}

} // namespace

extern "C" {

sg_status sg_batch_create(sg_batch* out)
{
    if (!out)
        return fail(SG_ERR_ARG, "NULL handle pointer");
    *out = nullptr;
    DevCtx* c = nullptr;
    sg_status s = get_ctx(&c);
    if (s != SG_OK)
        return s;
    sg_batch b = new (std::nothrow) sg_batch_s;
    if (!b)
        return fail(SG_ERR_NOMEM, "host allocation failed");
    cudaGetDevice(&b->device);
    cudaError_t e = cudaMalloc(&b->q, sizeof(SgQueue));
    if (e != cudaSuccess) {
        delete b;
        return cuda_fail(e, "cudaMalloc");
    }
    *out = b;
    return SG_OK;
}

sg_status sg_batch_destroy(sg_batch b)
{
    if (!b)
        return SG_OK;
    if (b->exec)
        cudaGraphExecDestroy(b->exec);
    cudaFree(b->q);
    delete b;
    return SG_OK;
}

sg_status sg_batch_decode(sg_batch b, const double* d_llr, size_t n_cw, const sg_params* p, uint8_t* d_bits,
                          double* d_lapp, sg_cw_stats* d_stats, void* stream)
{
    return batch_enqueue(b, d_llr, n_cw, p, d_bits, d_lapp, d_stats, (cudaStream_t)stream);
}

sg_status sg_batch_capture(sg_batch b, const double* d_llr, size_t n_cw, const sg_params* p, uint8_t* d_bits,
                           double* d_lapp, sg_cw_stats* d_stats, void* stream)
{
    if (!b)
        return fail(SG_ERR_ARG, "invalid batch handle");
    cudaStream_t st = (cudaStream_t)stream;
    cudaStream_t own = nullptr;
    if (!st) {
        SG_CUDA(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
        st = own;
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    sg_status s = SG_OK;
    if (e != cudaSuccess) {
        s = cuda_fail(e, "cudaStreamBeginCapture");
    } else {
        s = batch_enqueue(b, d_llr, n_cw, p, d_bits, d_lapp, d_stats, st);
        e = cudaStreamEndCapture(st, &g);
        if (s == SG_OK && e != cudaSuccess)
            s = cuda_fail(e, "cudaStreamEndCapture");
    }
    if (s == SG_OK) {
        if (b->exec) {
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
        }
        e = cudaGraphInstantiate(&b->exec, g, 0);
        if (e != cudaSuccess)
            s = cuda_fail(e, "cudaGraphInstantiate");
    }
    if (g)
        cudaGraphDestroy(g);
    if (own)
        cudaStreamDestroy(own);
    return s;
}

sg_status sg_batch_replay(sg_batch b, void* stream)
{
    if (!b || !b->exec)
        return fail(SG_ERR_ARG, "no captured decode in this batch handle");
    SG_CUDA(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
    return SG_OK;
}

sg_status sg_batch_check(sg_batch b)
{
    if (!b)
        return fail(SG_ERR_ARG, "invalid batch handle");
    SgQueue hq;
    SG_CUDA(cudaMemcpy(&hq, b->q, sizeof hq, cudaMemcpyDeviceToHost));
    if (hq.err)
        return fail(SG_ERR_TIMEOUT, "a persistent-decoder warp gave up waiting for work");
    return SG_OK;
}

int sg_batch_variant_count(void) { return SG_NPVARIANTS; }

const char* sg_batch_variant_name(int v) { return (v >= 0 && v < SG_NPVARIANTS) ? g_pvariants[v].name : ""; }

sg_status sg_batch_set_variant(int v)
{
    if (v < 0 || v >= SG_NPVARIANTS)
        return fail(SG_ERR_ARG, "no such batch variant");
    g_pvariant = v;
    return SG_OK;
}

int sg_batch_get_variant(void) { return g_pvariant; }

sg_status sg_guess_ceiling(unsigned long long iters, int32_t mode, double* guesses_per_second)
{
    if (!guesses_per_second || iters == 0 || (mode != 0 && mode != 1))
        return fail(SG_ERR_ARG, "need iters > 0, mode 0 or 1 and an output pointer");
    void (*kern)(unsigned long long, double*) =
        mode == 1 ? sg_guess_ceiling_kernel<true> : sg_guess_ceiling_kernel<false>;
    DevCtx* c = nullptr;
    sg_status s = get_ctx(&c);
    if (s != SG_OK)
        return s;
    const int blocks = c->sms * 8; /* 8 CTAs x 8 warps per SM */
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    SG_CUDA(cudaEventCreate(&e0));
    SG_CUDA(cudaEventCreate(&e1));
    kern<<<blocks, 256>>>(iters / 8 + 1, c->err_sink); /* warm-up */
    SG_CUDA(cudaEventRecord(e0));
    kern<<<blocks, 256>>>(iters, c->err_sink);
    SG_CUDA(cudaEventRecord(e1));
    SG_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    SG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    SG_CUDA(cudaGetLastError());
    *guesses_per_second = 2.0 * (double)iters * blocks * 256 / (ms / 1000.0);
    return SG_OK;
}

sg_status sg_forward_device(const double* d_llr, size_t n_cw, const sg_params* p, uint8_t* d_bits, double* d_lapp,
                            sg_cw_stats* d_stats, double* d_ckpt, void* stream)
{
    sg_status s = check_params(p);
    if (s != SG_OK)
        return s;
    if (n_cw == 0)
        return SG_OK;
    if (!d_llr || !d_bits || !d_stats || !d_ckpt)
        return fail(SG_ERR_ARG, "llr, bits, stats and ckpt must not be NULL");
    if ((uintptr_t)d_llr & 7u)
        return fail(SG_ERR_ARG, "llr must be 8-byte aligned");
    DevCtx* c = nullptr;
    if ((s = get_ctx(&c)) != SG_OK)
        return s;
    SgDecodeArgs a;
    memset(&a, 0, sizeof a);
    a.llr = d_llr;
    a.bits = d_bits;
    a.lapp = d_lapp;
    a.stats = d_stats;
    a.enum_tabs = c->enum_tabs;
    a.err = c->err;
    a.ckpt = d_ckpt;
    a.n_cw = n_cw;
    a.wait_limit = g_wait_limit.load();
    a.L = p->L;
    a.imax = p->Imax;
    a.tmax = tmax_eff(p->Tmax);
    a.use_bulk = ((uintptr_t)d_llr & 15u) == 0;
    a.thres = p->thres;
    memcpy(a.alpha, p->alpha, sizeof a.alpha);
    const SgVariant& v = g_variants[g_variant];
    void* kargs[] = {(void*)&a};
    SG_CUDA(cudaLaunchKernel(v.fn, dim3(grid_for(n_cw, 1 << 30)), dim3(v.nw * 32), kargs, v.smem,
                             (cudaStream_t)stream));
    return SG_OK;
}

sg_status sg_backward_device(const double* d_llr, size_t n_cw, const sg_params* p, const sg_cw_stats* d_stats,
                             const double* d_ckpt, const uint8_t* d_code_bits, int32_t loss_mode, double* d_loss,
                             double* d_grad_alpha, double* d_grad_llr, void* stream)
{
    sg_status s = check_params(p);
    if (s != SG_OK)
        return s;
    if (loss_mode != 0 && loss_mode != 1)
        return fail(SG_ERR_ARG, "loss_mode must be 0 (final APP) or 1 (every phase's APP)");
    if (p->Tmax < SG_ENUM_LEN && p->Tmax != 0)
        return fail(SG_ERR_ARG, "the adjoint needs Tmax >= 65536 (every line stops at a list insertion)");
    if (n_cw == 0)
        return SG_OK;
    if (!d_llr || !d_stats || !d_ckpt || !d_code_bits || !d_loss || !d_grad_alpha)
        return fail(SG_ERR_ARG, "NULL buffer");
    DevCtx* c = nullptr;
    if ((s = get_ctx(&c)) != SG_OK)
        return s;
    SgBackwardArgs a;
    memset(&a, 0, sizeof a);
    a.llr = d_llr;
    a.ckpt = d_ckpt;
    a.stats = d_stats;
    a.code_bits = d_code_bits;
    a.enum_tabs = c->enum_tabs;
    a.loss = d_loss;
    a.grad_alpha = d_grad_alpha;
    a.grad_llr = d_grad_llr;
    a.n_cw = n_cw;
    a.L = p->L;
    a.nph = 3 * p->Imax;
    a.loss_mode = loss_mode;
    a.thres = p->thres;
    memcpy(a.alpha, p->alpha, sizeof a.alpha);
    void* kargs[] = {(void*)&a};
    SG_CUDA(cudaLaunchKernel((const void*)sg_backward_kernel<8>, dim3(grid_for(n_cw, 1 << 30)), dim3(256), kargs,
                             sizeof(SgBackSmem<8>), (cudaStream_t)stream));
    return SG_OK;
}

sg_status sg_set_math_mode(int32_t mode)
{
    if (mode != 0 && mode != 1)
        return fail(SG_ERR_ARG, "math mode must be 0 (table-driven) or 1 (correctly rounded)");
    g_math_mode.store(mode);
    return SG_OK;
}

int32_t sg_get_math_mode(void) { return g_math_mode.load(); }

sg_status sg_set_wait_limit(uint64_t limit)
{
    g_wait_limit.store(limit > (uint64_t)SG_WAIT_LIMIT_DEFAULT ? SG_WAIT_LIMIT_DEFAULT : (long long)limit);
    return SG_OK;
}

uint64_t sg_get_wait_limit(void) { return (uint64_t)g_wait_limit.load(); }

sg_status sg_check_device(void* stream)
{
    DevCtx* c = nullptr;
    sg_status s = get_ctx(&c);
    if (s != SG_OK)
        return s;
    SG_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    unsigned int flags = 0;
    SG_CUDA(cudaMemcpy(&flags, c->err, sizeof flags, cudaMemcpyDeviceToHost));
    if (flags) {
        SG_CUDA(cudaMemset(c->err, 0, sizeof flags));
        return fail(SG_ERR_TIMEOUT, (flags & 2u) ? "a bulk-copy wait gave up and the copy did not complete"
                                                 : "a bulk-copy wait gave up; the affected codewords report "
                                                   "converged = -2");
    }
    return SG_OK;
}

int sg_decoder_variant_count(void) { return SG_NVARIANTS; }

const char* sg_decoder_variant_name(int v)
{
    return (v >= 0 && v < SG_NVARIANTS) ? g_variants[v].name : "";
}

sg_status sg_decoder_set_variant(int v)
{
    if (v < 0 || v >= SG_NVARIANTS)
        return fail(SG_ERR_ARG, "no such decoder variant");
    g_variant = v;
    return SG_OK;
}

int sg_decoder_get_variant(void) { return g_variant; }

const char* sg_status_string(sg_status s)
{
    switch (s) {
    case SG_OK: return "ok";
    case SG_ERR_ARG: return "invalid argument";
    case SG_ERR_CUDA: return "CUDA error";
    case SG_ERR_NONFINITE: return "non-finite input";
    case SG_ERR_IO: return "I/O error";
    case SG_ERR_NOMEM: return "out of memory";
    case SG_ERR_TIMEOUT: return "device wait timed out";
    }
    return "unknown status";
}

const char* sg_last_error(void) { return t_err.c_str(); }

const char* sg_version(void) { return "sogrand_b200 0.1.0 (sm_100a)"; }

} // extern "C"
