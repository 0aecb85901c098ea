/* sg_adjoint.cuh -- FP64 adjoint of the SOGRAND soft-output decoder.
 *
 * The decoder is piecewise smooth in its inputs: the sort, IC, the tested
 * patterns, the codeword list, the stopping guess, the early-termination
 * decisions and the number of phases are piecewise constant, and are held
 * fixed as the branch of the forward pass.  On that branch the soft output
 * of one line (SOGRAND_bitSO, SOGRAND_C/cubic_decoder_final.c:536-577) is
 *   p_j   = exp(-PM_j),  PM_j = sum_k JacLog(-|x_k|) + sum_{k in S_j} delta(|x_k|)
 *   pNL   = 2^-8 (1 - sum_{t <= T} exp(-PM_t))          (all counted guesses t)
 *   pp1_i = 1/(1 + e^{x_i}),  pp0_i = 1 - pp1_i           (clamped to [1e-40, 1])
 *   p0_i  = sum_{j: c_ji = 0} p_j + max(pNL,1e-40) pp0_i,  p1_i likewise
 *   L_APP_i = log max(p0_i,1e-40) - log max(p1_i,1e-40),   L_E_i = L_APP_i - x_i
 * with S_j the positions where pattern j differs from the hard decision and
 *   dPM/dx_i = sign(x_i) (-sigma(-|x_i|) [|x_i| <= 50] + [i in S]),
 * so dpNL/dx_i = 2^-8 sign(x_i) (-sigma(-|x_i|)[|x_i| <= 50] E + E_i) with
 * E = sum_t exp(-PM_t) and E_i the same sum over guesses holding position i.
 * sg_line_vjp applies the transpose of that Jacobian to an upstream vector.
 *
 * The backward kernel re-runs, phase by phase in reverse, every line decode
 * from the checkpointed extrinsic cube entering the phase (the forward
 * writes one 32 KB checkpoint per phase), accumulating E and E_i on the way,
 * and propagates the gradient of the loss
 *   loss = sum_i softplus(s_i L_APP_i),  s_i = +1 for code bit 1, -1 for 0,
 * (the BCE of the final APP against the transmitted bits; loss_mode 1: the
 * sum of that over every phase's APP) to the per-phase extrinsic weights
 * alpha_p, the channel LLRs and the previous phase.
 */
#pragma once

/* sum over lanes 0..15 (lanes 16..31 contribute 0), result in all lanes */
__device__ __forceinline__ double sg_sum16(double v, int lane)
{
    v = lane < 16 ? v : 0.0;
    for (int off = 16; off > 0; off >>= 1)
        v += __shfl_xor_sync(SG_FULL, v, off);
    return v;
}

/* Gradient with respect to the line input x (lanes 0..15) of g . L_APP,
 * g the upstream gradient of L_APP (lanes 0..15). */
__device__ __forceinline__ double sg_line_vjp(double x, double g, const SgAdjOut& a, const double* etab, int lane)
{
    const bool act = lane < 16;
    if (a.curl == 0)
        return act ? g : 0.0; /* L_APP = x */
    const double eps = 1e-40;
    const bool pnl_live = a.pnl > eps;
    const double p_nl = fmax(a.pnl, eps);
    const double ex = sg_exp(act ? x : 0.0, etab);
    const double pp1r = 1.0 / (1.0 + ex);
    const double pp0r = 1.0 - pp1r;
    const double pp1 = fmin(fmax(pp1r, eps), 1.0);
    const double pp0 = fmin(fmax(pp0r, eps), 1.0);
    double p0 = 0.0, p1 = 0.0;
    for (int j = 0; j < a.curl; j++) {
        const double pj = __shfl_sync(SG_FULL, a.my_e, j);
        const uint32_t cj = (__shfl_sync(SG_FULL, a.my_cm, j) >> (lane & 15)) & 1u;
        if (cj)
            p1 += pj;
        else
            p0 += pj;
    }
    p0 += p_nl * pp0;
    p1 += p_nl * pp1;
    const double a0 = (act && p0 > eps) ? g / p0 : 0.0;
    const double a1 = (act && p1 > eps) ? -g / p1 : 0.0;
    const double dsig = pp0r * pp1r; /* d pp0/dx = -d pp1/dx */
    double gx = 0.0;
    if (pp0r > eps)
        gx += a0 * p_nl * dsig;
    if (pp1r > eps)
        gx -= a1 * p_nl * dsig;
    const double ax = fabs(x);
    const double sgn = x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0);
    const double sm = ax <= 50.0 ? 1.0 / (1.0 + sg_exp(ax, etab)) : 0.0; /* sigma(-|x|) */
    for (int j = 0; j < a.curl; j++) {
        const double pj = __shfl_sync(SG_FULL, a.my_e, j);
        const uint32_t cm = __shfl_sync(SG_FULL, a.my_cm, j);
        const uint32_t cj = (cm >> (lane & 15)) & 1u;
        const double gpj = sg_sum16(cj ? a1 : a0, lane);
        const double gpm = -pj * gpj;
        const double inS = (((cm ^ a.hdm) >> (lane & 15)) & 1u) ? 1.0 : 0.0;
        gx += gpm * sgn * (inS - sm);
    }
    if (pnl_live) {
        const double gpnl = sg_sum16(a0 * pp0 + a1 * pp1, lane);
        const double ei = __shfl_sync(SG_FULL, a.esort, a.myrank & 15);
        gx += gpnl * 0x1p-8 * sgn * (ei - sm * a.etot);
    }
    return act ? gx : 0.0;
}

struct SgBackwardArgs {
    const double* llr;
    const double* ckpt;          /* [n_cw][nph][4096]: L_E entering each phase */
    const sg_cw_stats* stats;    /* phases run per codeword (forward output) */
    const uint8_t* code_bits;    /* [n_cw][4096] transmitted bits, 0/1 */
    const uint32_t* enum_tabs;
    double* loss;                /* [n_cw] */
    double* grad_alpha;          /* [n_cw][nph] */
    double* grad_llr;            /* [n_cw][4096] or NULL */
    unsigned long long n_cw;
    int32_t L;
    int32_t nph;                 /* 3 * Imax */
    int32_t loss_mode;           /* 0: BCE of the final APP; 1: summed over all phases' APPs */
    double thres;
    double alpha[SG_MAX_PHASES];
};

template <int NW>
struct SgBackSmem {
    double gle[SG_CUBE]; /* d loss / d L_E of the phase being processed */
    alignas(16) double etab[SG_EXP_TAB_LEN];
    alignas(16) double ltab[SG_LOG_TAB_LEN];
    SgWarpScratch ws[NW];
    double ga;   /* d loss / d alpha of the phase */
    double lsum; /* loss of the codeword */
    int line_next;
};

template <int NW>
__global__ void __launch_bounds__(NW * 32, 3) sg_backward_kernel(const __grid_constant__ SgBackwardArgs args)
{
    constexpr int NT = NW * 32;
    SgBackSmem<NW>& S = *reinterpret_cast<SgBackSmem<NW>*>(sg_smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < SG_EXP_TAB_LEN; i += NT)
        S.etab[i] = g_etab[i];
    for (int i = tid; i < SG_LOG_TAB_LEN; i += NT)
        S.ltab[i] = g_ltab[i];
    SgLineParams lp;
    lp.L = args.L;
    lp.tmax = 0xffffffffu;
    lp.thres = args.thres;
    __syncthreads();
    for (unsigned long long cw = blockIdx.x; cw < args.n_cw; cw += gridDim.x) {
        const int P = args.stats[cw].phases;
        const double* g = args.llr + cw * SG_CUBE;
        for (int i = tid; i < SG_CUBE; i += NT) {
            S.gle[i] = 0.0;
            if (args.grad_llr)
                args.grad_llr[cw * SG_CUBE + i] = 0.0;
        }
        for (int p = tid; p < args.nph; p += NT)
            args.grad_alpha[cw * args.nph + p] = 0.0;
        if (tid == 0)
            S.lsum = 0.0;
        __syncthreads();
        for (int p = P - 1; p >= 0; p--) {
            const int axis = p % 3;
            const double alpha = args.alpha[p];
            const double* ck = args.ckpt + (cw * args.nph + p) * SG_CUBE;
            if (tid == 0) {
                S.line_next = 0;
                S.ga = 0.0;
            }
            __syncthreads();
            for (;;) {
                int l = 0;
                if (lane == 0)
                    l = atomicAdd(&S.line_next, 1);
                l = __shfl_sync(SG_FULL, l, 0);
                if (l >= 256)
                    break;
                const int pos = sg_pos(axis, l, lane & 15);
                const double lep = lane < 16 ? ck[pos] : 0.0;
                const double x = lane < 16 ? __dadd_rn(g[pos], __dmul_rn(alpha, lep)) : 1.0;
                SgAdjOut a;
                const SgLineResult r = sg_decode_line<1, true>(x, lp, args.enum_tabs, S.etab, S.ltab, &S.ws[warp], &a);
                const double gE = lane < 16 ? S.gle[pos] : 0.0;
                double gL = 0.0, lossv = 0.0;
                const bool scored = p == P - 1 || args.loss_mode == 1;
                if (scored && lane < 16) {
                    const double s = args.code_bits[cw * SG_CUBE + pos] ? 1.0 : -1.0;
                    const double z = s * r.lapp;
                    lossv = z > 0.0 ? z + log1p(exp(-z)) : log1p(exp(z)); /* softplus */
                    gL = s / (1.0 + exp(-z));                              /* s * sigmoid(z) */
                }
                const double gx = sg_line_vjp(x, gL + gE, a, S.etab, lane) - gE;
                if (lane < 16) {
                    S.gle[pos] = alpha * gx;
                    if (args.grad_llr)
                        args.grad_llr[cw * SG_CUBE + pos] += gx;
                }
                const double ga = sg_sum16(gx * lep, lane);
                const double ls = sg_sum16(lossv, lane);
                if (lane == 0) {
                    atomicAdd(&S.ga, ga);
                    if (scored)
                        atomicAdd(&S.lsum, ls);
                }
            }
            __syncthreads();
            if (tid == 0)
                args.grad_alpha[cw * args.nph + p] = S.ga;
            __syncthreads();
        }
        if (tid == 0)
            args.loss[cw] = S.lsum;
        __syncthreads();
    }
}
