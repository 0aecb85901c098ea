/* sg_oracle.c -- CPU restatement of the SOGRAND (16,8)^3 cubic decoder.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA decoder, never linked
 * by the product.  Each function cites the lines of the reference it
 * restates; file names are relative to the reference project root.
 *   D = SOGRAND_C/cubic_decoder_final.c
 *   E = SOGRAND_C/cubic_encoder.c
 *   C = SOGRAND_C/channel_sim.c
 *
 * Compile with -DSGO_TWIN=1 to evaluate exp/log with the kernel's own
 * routines instead of libm (-DSG_CR_MATH=1: its correctly rounded ones,
 * sogrand_b200/csrc/sg_crmath.h), and with -DSGO_CRQ=1 with the
 * binary128-based correctly rounded ones of crq.h.
 */
#include "sg_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef SGO_TWIN
#define SGO_TWIN 0
#endif

#ifndef SGO_CRQ
#define SGO_CRQ 0
#endif

#if SGO_CRQ
/* correctly rounded through extended and binary128 precision (crq.h) */
#include "crq.h"
static double ox_exp(double x) { return crq_exp(x); }
static double ox_log(double x) { return crq_log(x); }
static double ox_pow2_neg(double s) { return pow(2.0, -s); }
#elif SGO_TWIN
/* the decoder's own exp/log: the table-driven routines of sg_math.h (its
 * default math mode), or, built with SG_CR_MATH=1, the correctly rounded
 * ones of sg_crmath.h (its reference-exact mode) */
#include "../sogrand_b200/csrc/sg_crmath.h"
static const double k_etab[SG_EXP_TAB_LEN] = SG_EXP_TAB_INIT;
static const double k_ltab[SG_LOG_TAB_LEN] = SG_LOG_TAB_INIT;
#ifndef SG_CR_MATH
#define SG_CR_MATH 0
#endif
#if SG_CR_MATH
static double ox_exp(double x) { return sg_exp_cr(x, k_etab); }
static double ox_log(double x) { return sg_log_cr(x, k_ltab); }
#else
static double ox_exp(double x) { return sg_exp(x, k_etab); }
static double ox_log(double x) { return sg_log(x, k_ltab); }
#endif
static double ox_pow2_neg(double s) { return s == 8.0 ? 0x1p-8 : pow(2.0, -s); }
#else
static double ox_exp(double x) { return exp(x); }
static double ox_log(double x) { return log(x); }
static double ox_pow2_neg(double s) { return pow(2.0, -s); }
#endif

int sgo_math_mode(void) { return SGO_CRQ ? 2 : SGO_TWIN; }

static const double kEps = 1e-40; /* EPSILON, D:16 */

/* ---------------------------------------------------------------- code -- */

/* G = [I | P] and H = [P^T | I] from the CRC polynomial 0xeb, whose Koopman
 * form 0xeb expands to the 9 coefficients 1,1,1,0,1,0,1,1,1 (koopman2matlab,
 * D:454-466; polynomial chosen at D:478).  P row i is the remainder of x^i
 * shifted through the polynomial division (D:491-503). */
void sgo_code_matrices(uint8_t G[SGO_K * SGO_N], uint8_t H[(SGO_N - SGO_K) * SGO_N])
{
    const int r = SGO_N - SGO_K;
    const long long koop = 0xeb;
    int len = (int)floor(log2((double)koop)) + 1;
    int poly[16];
    for (int i = 0; i < len; i++)
        poly[i] = (int)((koop >> (len - 1 - i)) & 1);
    poly[len] = 1;
    int plen = len + 1;
    uint8_t P[SGO_K][SGO_N - SGO_K];
    for (int i = 0; i < SGO_K; i++) {
        int m[SGO_N + 16];
        memset(m, 0, sizeof m);
        m[i] = 1;
        for (int j = 0; j < SGO_K; j++)
            if (m[j] == 1)
                for (int l = 0; l < plen; l++)
                    m[j + l] ^= poly[l];
        for (int j = 0; j < r; j++)
            P[i][j] = (uint8_t)m[SGO_K + j];
    }
    for (int i = 0; i < SGO_K; i++)
        for (int j = 0; j < SGO_N; j++)
            G[i * SGO_N + j] = j < SGO_K ? (uint8_t)(i == j) : P[i][j - SGO_K];
    for (int i = 0; i < r; i++)
        for (int j = 0; j < SGO_N; j++)
            H[i * SGO_N + j] = j < SGO_K ? P[j][i] : (uint8_t)(i == j - SGO_K);
}

static uint8_t g_G[SGO_K * SGO_N], g_H[(SGO_N - SGO_K) * SGO_N];
static int g_code_ready = 0;

static void code_init(void)
{
    if (!g_code_ready) {
        sgo_code_matrices(g_G, g_H);
        g_code_ready = 1;
    }
}

/* --------------------------------------------------------- line decode -- */

static double jaclog(double x) /* D:762 */
{
    if (x > 50)
        return x;
    if (x < -50)
        return 0.0;
    return ox_log(1.0 + ox_exp(x));
}

/* Recursive middle-pivot partition sort of D:763, carrying the index
 * permutation.  Ties are ordered exactly as the reference orders them. */
static void qsort_ref(double* a, int* perm, int n)
{
    if (n < 2)
        return;
    double p = a[n / 2];
    int i = 0, j = n - 1;
    while (i <= j) {
        while (a[i] < p)
            i++;
        while (a[j] > p)
            j--;
        if (i <= j) {
            if (j == 0) { /* the reference's unsigned j would wrap here */
                fprintf(stderr, "sg_oracle: quicksort reached j == 0 at a swap\n");
                abort();
            }
            double t = a[i];
            a[i] = a[j];
            a[j] = t;
            int tt = perm[i];
            perm[i] = perm[j];
            perm[j] = tt;
            i++;
            j--;
        }
    }
    if (j > 0)
        qsort_ref(a, perm, j + 1);
    if (i < n)
        qsort_ref(a + i, perm + i, n - i);
}

/* All 8 parity checks of H satisfied (ParityCheck, D:748-755). */
static int parity_ok(const uint8_t c[SGO_N])
{
    for (int j = 0; j < SGO_N - SGO_K; j++) {
        uint8_t s = 0;
        for (int i = 0; i < SGO_N; i++)
            s ^= (uint8_t)(c[i] * g_H[j * SGO_N + i]);
        if (s == 1)
            return 0;
    }
    return 1;
}

/* Successor fill of the position offsets u (mountain_build, D:775-789). */
static void mountain(int32_t* u, int32_t k, int32_t w, int32_t W1, int32_t n1)
{
    for (int32_t i = k + 1; i < w; i++)
        u[i] = u[k];
    int64_t W2 = W1;
    for (int32_t i = 0; i < w; i++)
        W2 -= u[i];
    int64_t den = n1 - u[k];
    if (W2 < 0 || den <= 0) {
        fprintf(stderr, "sg_oracle: mountain fill outside the reachable domain\n");
        abort();
    }
    int64_t q = W2 / den;
    int64_t rem = W2 - q * den;
    if (q != 0)
        for (int64_t i = w - q; i < w; i++)
            if (i >= 0)
                u[i] = n1;
    if (w > q)
        u[w - q - 1] += (int32_t)rem;
}

typedef struct {
    /* per-line state of sogrand_main_logic (D:587-746) */
    uint8_t cHD[SGO_N];
    int perm[SGO_N];
    double absL[SGO_N]; /* sorted ascending after the sort */
    double delta[SGO_N]; /* JacLog(|L|) - JacLog(-|L|) per sorted position */
    double pm_hd;
    double p_not_guess;
    double T;           /* T_val, a double in the reference */
    int cur_l;
    double pnl;
    double pm_list[8];
    uint8_t chat[8][SGO_N];
    int L;
    uint64_t Tmax;
    double thres;
    double etot;          /* sum of exp(-PM) over the counted guesses */
    double epos[SGO_N];   /* the same over guesses that flip position i */
} line_state;

/* PM of a test error pattern over sorted positions (getPM, D:765).  The
 * reference evaluates the parenthesised difference of JacLogs afresh for
 * every pattern; it is a pure function of the position, so the per-line
 * value in delta[] is the same number. */
static double pattern_pm(const line_state* s, const uint8_t tep[SGO_N])
{
    double pm = s->pm_hd;
    for (int i = 0; i < SGO_N; i++)
        if (tep[i] == 1)
            pm += s->delta[i];
    return pm;
}

/* Confidence of the list (getLConf, D:767-774), even = 0 so s = 8. */
static double list_conf(line_state* s)
{
    double p_pos = 0.0;
    for (int i = 0; i <= s->cur_l; i++)
        p_pos += ox_exp(-s->pm_list[i]);
    double p_neg = ox_pow2_neg((double)(SGO_N - SGO_K)) * s->p_not_guess;
    s->pnl = p_neg;
    return (p_pos + p_neg > kEps) ? (p_pos / (p_pos + p_neg)) : 1.0;
}

/* Test one pattern: AddTEP (D:761), T++, P_notGuess update, ParityCheck and
 * list insertion (D:669-687).  Returns 1 when the line decode stops. */
static int visit(line_state* s, const uint8_t tep[SGO_N])
{
    uint8_t c[SGO_N];
    for (int i = 0; i < SGO_N; i++)
        c[s->perm[i]] = s->cHD[s->perm[i]] ^ tep[i];
    s->T += 1.0;
    double pm = pattern_pm(s, tep);
    double e = ox_exp(-pm);
    s->p_not_guess -= e;
    s->etot += e;
    for (int i = 0; i < SGO_N; i++)
        if (tep[i])
            s->epos[s->perm[i]] += e;
    if (parity_ok(c)) {
        s->pm_list[s->cur_l] = pm;
        memcpy(s->chat[s->cur_l], c, SGO_N);
        double conf = list_conf(s);
        s->cur_l++;
        if (conf > s->thres || s->cur_l == s->L)
            return 1;
    }
    return 0;
}

static int32_t cvt_i32(double v) /* (int32_t) of a double on x86-64 (cvttsd2si) */
{
    if (!(v > -2147483649.0 && v < 2147483648.0))
        return INT32_MIN;
    return (int32_t)v;
}

/* Pattern enumeration of sogrand_main_logic after the hard decision
 * (D:642-744): logistic weights wt = IC+1..wt_max; per weight the Hamming
 * weights w from the bound of D:653 upwards while W = wt - IC*w is still
 * reachable (D:657-659); per (wt, w) the mountain fill and the landslide
 * steps.  cont(ctx) is the loop condition evaluated at each weight (D:652);
 * visit(ctx, tep, first) tests a pattern and returns nonzero to stop. */
typedef int (*sgo_cont_fn)(void* ctx);
typedef int (*sgo_visit_fn)(void* ctx, const uint8_t tep[SGO_N], int first_of_weight);

static void enumerate_patterns(int32_t ic, sgo_cont_fn cont, sgo_visit_fn visit, void* ctx)
{
    const int n = SGO_N;
    uint8_t tep[SGO_N];
    int32_t u[SGO_N], d[SGO_N], D[SGO_N];
    int32_t wt = ic + 1;
    int32_t wt_max = ic * n + n * (n + 1) / 2;
    double temp = 1 + 2 * ((double)n + (double)ic);
    while (cont(ctx) && wt <= wt_max) {
        int first = 1;
        int32_t w = (int32_t)ceil((temp - sqrt(pow(temp, 2.0) - 8 * wt)) / 2);
        if (w < 1)
            w = 1;
        while (w <= n) {
            int32_t W = wt - ic * w;
            if (W < w * (w + 1) / 2)
                break;
            int32_t W1 = W - w * (w + 1) / 2;
            int32_t n1 = n - w;
            for (int i = 0; i < w; i++)
                u[i] = 0;
            if (n1 == 0) {
                /* w = 16: the reference would divide by zero in mountain_build;
                 * the only pattern is all ones (never reached while decoding) */
                memset(tep, 1, sizeof tep);
                if (visit(ctx, tep, first))
                    return;
                first = 0;
                w++;
                continue;
            }
            mountain(u, 0, w, W1, n1);
            for (;;) {
                memset(tep, 0, sizeof tep);
                for (int i = 0; i < w; i++)
                    tep[i + u[i]] = 1;
                if (visit(ctx, tep, first))
                    return;
                first = 0;
                /* landslide step, D:689-734 */
                for (int i = 0; i < w - 1; i++)
                    d[i] = u[i + 1] - u[i];
                d[w - 1] = 0;
                D[w - 1] = d[w - 1];
                for (int i = 1; i < w; i++)
                    D[w - i - 1] = D[w - i] + d[w - i - 1];
                if (!(D[0] >= 2))
                    break;
                int32_t kk = 0;
                for (int i = w - 1; i > 0; i--)
                    if (D[i] >= 2) {
                        kk = i;
                        break;
                    }
                u[kk]++;
                mountain(u, kk, w, W1, n1);
            }
            w++;
        }
        wt++;
    }
}

static int line_cont(void* ctx)
{
    line_state* s = (line_state*)ctx;
    return s->cur_l < s->L && s->T < (double)s->Tmax;
}

static int line_visit(void* ctx, const uint8_t tep[SGO_N], int first)
{
    (void)first;
    return visit((line_state*)ctx, tep);
}

/* Ordered-reliability list GRAND (sogrand_main_logic, D:587-746) with IC
 * chosen from the sorted reliabilities (D:619-622) and even = 0. */
static void main_logic(line_state* s, const double llr[SGO_N])
{
    const int n = SGO_N;
    for (int i = 0; i < n; i++) {
        s->cHD[i] = (llr[i] > 0.0) ? 0 : 1; /* HardDec, D:758 */
        s->perm[i] = i;
        s->absL[i] = fabs(llr[i]);
    }
    s->cur_l = 0;
    s->pnl = 0.0;
    s->p_not_guess = 1.0;
    s->etot = 0.0;
    for (int i = 0; i < n; i++)
        s->epos[i] = 0.0;
    double pm = 0;
    for (int i = 0; i < n; i++) /* getPM_HD before sorting, D:617, D:764 */
        pm += jaclog(-s->absL[i]);
    s->pm_hd = pm;
    qsort_ref(s->absL, s->perm, n);
    for (int i = 0; i < n; i++)
        s->delta[i] = (jaclog(s->absL[i]) - jaclog(-s->absL[i]));
    double beta = (s->absL[(uint64_t)round((double)n / 2) - 1] - s->absL[0]) / (round((double)n / 2) - 1);
    int32_t ic = cvt_i32(round(s->absL[0] / beta - 1));
    if (ic < 0)
        ic = 0;
    if (s->Tmax == 0)
        s->Tmax = 0x7fffffff; /* if (Tmax==0) Tmax=Inf, D:607 */

    uint8_t tep[SGO_N];
    memset(tep, 0, sizeof tep);
    s->T = 0;
    if (visit(s, tep)) /* the hard decision itself, D:624-641 */
        return;
    enumerate_patterns(ic, line_cont, line_visit, s);
}

typedef struct {
    uint32_t* out;
    size_t cap, n;
} order_rec;

static int order_cont(void* ctx)
{
    (void)ctx;
    return 1;
}

static int order_visit(void* ctx, const uint8_t tep[SGO_N], int first)
{
    order_rec* r = (order_rec*)ctx;
    if (r->n >= r->cap)
        return 1;
    uint32_t m = 0;
    for (int i = 0; i < SGO_N; i++)
        m |= (uint32_t)tep[i] << i;
    r->out[r->n++] = m | (first ? 0x10000u : 0u);
    return 0;
}

size_t sgo_pattern_order(int32_t ic, uint32_t* out, size_t cap)
{
    if (cap == 0)
        return 0;
    order_rec r = {out, cap, 0};
    out[r.n++] = 0; /* the hard decision */
    enumerate_patterns(ic, order_cont, order_visit, &r);
    return r.n;
}

double sgo_exp(double x) { return ox_exp(x); }
double sgo_log(double x) { return ox_log(x); }

#if SGO_TWIN
/* Diagnostics of the decoder's math (twin build): the correctly rounded
 * routines' slow paths on their own (finite x; log: x > 0), and the
 * table-driven routines the input generator uses. */
double sgo_exp_cr_slow(double x) { return sg_exp_cr_slow(x, k_etab); }
double sgo_log_cr_slow(double x) { return sg_log_cr_slow(x, k_ltab); }
double sgo_exp_tab(double x) { return sg_exp(x, k_etab); }
double sgo_log_tab(double x) { return sg_log(x, k_ltab); }
#endif

static void bitso_state(const double llr[SGO_N], int L, uint64_t Tmax, double thres, sgo_line_out* out,
                        line_state* sp);

/* Soft output of one line (SOGRAND_bitSO, D:521-585). */
void sgo_bitso(const double llr[SGO_N], int L, uint64_t Tmax, double thres, sgo_line_out* out)
{
    line_state s;
    bitso_state(llr, L, Tmax, thres, out, &s);
}

static void bitso_state(const double llr[SGO_N], int L, uint64_t Tmax, double thres, sgo_line_out* out,
                        line_state* sp)
{
    code_init();
    line_state s;
    s.L = L;
    s.Tmax = Tmax;
    s.thres = thres;
    main_logic(&s, llr);
    out->n_guess = (uint64_t)s.T;
    out->cur_l = s.cur_l;
    out->pnl = s.pnl;
    *sp = s;
    if (s.cur_l == 0) {
        /* The reference reads an uninitialised list size here (D:524, D:536);
         * it is unreachable with Tmax = UINT64_MAX.  The defined behaviour is
         * its curL == 0 branch. */
        for (int i = 0; i < SGO_N; i++) {
            out->lapp[i] = llr[i];
            out->le[i] = 0.0;
        }
        return;
    }
    double p_nl = fmax(s.pnl, kEps);
    double pp1[SGO_N], pp0[SGO_N];
    for (int i = 0; i < SGO_N; i++) {
        pp1[i] = 1.0 / (1.0 + ox_exp(llr[i]));
        pp0[i] = 1.0 - pp1[i];
        pp1[i] = fmax(pp1[i], kEps);
        pp1[i] = fmin(pp1[i], 1.0 - kEps);
        pp0[i] = fmax(pp0[i], kEps);
        pp0[i] = fmin(pp0[i], 1.0 - kEps);
    }
    double p[8];
    for (int j = 0; j < s.cur_l; j++)
        p[j] = ox_exp(-s.pm_list[j]);
    for (int i = 0; i < SGO_N; i++) {
        double p1 = 0, p0 = 0;
        for (int j = 0; j < s.cur_l; j++) {
            double c = (double)s.chat[j][i];
            p1 += c * p[j];
            p0 += (1.0 - c) * p[j];
        }
        p0 += p_nl * pp0[i];
        p1 += p_nl * pp1[i];
        out->lapp[i] = ox_log(fmax(p0, kEps)) - ox_log(fmax(p1, kEps));
        out->le[i] = out->lapp[i] - llr[i];
    }
}

/* ------------------------------------------------------------- cubes -- */

#define IDX(row, col, slice) ((slice) * 256 + (col) * 16 + (row)) /* get_tensor_*, D:434-437 */

/* Systematic product encoding of a cube whose 8x8x8 corner is set: rows
 * (E:45-56), then columns (E:60-71), then slices (E:75-86).  Identical to
 * the re-encoding in early_termination (D:337-377). */
static void encode_from_corner(uint8_t* c)
{
    int t[SGO_K];
    for (int slice = 0; slice < SGO_K; slice++)
        for (int row = 0; row < SGO_K; row++) {
            for (int j = 0; j < SGO_K; j++)
                t[j] = c[IDX(row, j, slice)];
            for (int col = SGO_K; col < SGO_N; col++) {
                int pv = 0;
                for (int m = 0; m < SGO_K; m++)
                    pv += t[m] * g_G[m * SGO_N + col];
                c[IDX(row, col, slice)] = (uint8_t)(pv % 2);
            }
        }
    for (int slice = 0; slice < SGO_K; slice++)
        for (int col = 0; col < SGO_N; col++) {
            for (int j = 0; j < SGO_K; j++)
                t[j] = c[IDX(j, col, slice)];
            for (int row = SGO_K; row < SGO_N; row++) {
                int pv = 0;
                for (int m = 0; m < SGO_K; m++)
                    pv += t[m] * g_G[m * SGO_N + row];
                c[IDX(row, col, slice)] = (uint8_t)(pv % 2);
            }
        }
    for (int row = 0; row < SGO_N; row++)
        for (int col = 0; col < SGO_N; col++) {
            for (int j = 0; j < SGO_K; j++)
                t[j] = c[IDX(row, col, j)];
            for (int slice = SGO_K; slice < SGO_N; slice++) {
                int pv = 0;
                for (int m = 0; m < SGO_K; m++)
                    pv += t[m] * g_G[m * SGO_N + slice];
                c[IDX(row, col, slice)] = (uint8_t)(pv % 2);
            }
        }
}

void sgo_encode(const uint8_t info[SGO_INFO], uint8_t cw[SGO_CUBE])
{
    code_init();
    memset(cw, 0, SGO_CUBE);
    /* u(i,j,l) = info[l*64 + j*8 + i] embedded at c(i,j,l) (E:28-42) */
    for (int l = 0; l < SGO_K; l++)
        for (int j = 0; j < SGO_K; j++)
            for (int i = 0; i < SGO_K; i++)
                cw[IDX(i, j, l)] = info[l * 64 + j * 8 + i];
    encode_from_corner(cw);
}

int sgo_early_termination(const double* lapp) /* D:317-391 */
{
    code_init();
    uint8_t hd[SGO_CUBE], ct[SGO_CUBE];
    for (int i = 0; i < SGO_CUBE; i++)
        hd[i] = (lapp[i] > 0.0) ? 0 : 1;
    memset(ct, 0, sizeof ct);
    for (int l = 0; l < SGO_K; l++)
        for (int j = 0; j < SGO_K; j++)
            for (int i = 0; i < SGO_K; i++)
                ct[IDX(i, j, l)] = hd[IDX(i, j, l)];
    encode_from_corner(ct);
    return memcmp(ct, hd, SGO_CUBE) == 0;
}

void sgo_default_params(sgo_params* p)
{
    memset(p, 0, sizeof *p);
    p->L = 3;
    p->Imax = 30;
    p->Tmax = UINT64_MAX;
    p->thres = 1.0 - 1e-5;
    for (int i = 0; i < SGO_MAX_PHASES; i++)
        p->alpha[i] = 0.7;
}

/* One phase: lines along axis `axis` (0: row index varies, stride 1, the
 * reference's "columns" loop D:157-169; 1: col varies, stride 16, "rows"
 * D:196-208; 2: slice varies, stride 256, "slices" D:235-247). */
static void run_phase(int axis, const double* input, double* lapp, double* le,
                      const sgo_params* p, uint64_t* ng, uint64_t* ngmax)
{
    static const int stride[3] = {1, 16, 256};
    *ngmax = 0;
    for (int a = 0; a < SGO_N; a++)
        for (int b = 0; b < SGO_N; b++) {
            int base;
            if (axis == 0)
                base = IDX(0, b, a); /* slice a, col b */
            else if (axis == 1)
                base = IDX(b, 0, a); /* slice a, row b */
            else
                base = IDX(b, a, 0); /* col a, row b */
            double v[SGO_N];
            for (int i = 0; i < SGO_N; i++)
                v[i] = input[base + i * stride[axis]];
            sgo_line_out o;
            sgo_bitso(v, p->L, p->Tmax, p->thres, &o);
            int ngi = (int)o.n_guess; /* N_guess is an int in the reference */
            *ng += (uint64_t)ngi;
            if ((uint64_t)ngi > *ngmax)
                *ngmax = (uint64_t)ngi;
            for (int i = 0; i < SGO_N; i++) {
                lapp[base + i * stride[axis]] = o.lapp[i];
                le[base + i * stride[axis]] = o.le[i];
            }
        }
}

/* Per-codeword driver loop (main, D:119-289). */
void sgo_decode(const double* llr, size_t n_cw, const sgo_params* p,
                uint8_t* bits, double* lapp_out, sgo_cw_stats* stats)
{
    code_init();
    double* lch = (double*)malloc(sizeof(double) * SGO_CUBE);
    double* lapp = (double*)calloc(SGO_CUBE, sizeof(double));
    double* le = (double*)malloc(sizeof(double) * SGO_CUBE);
    double* input = (double*)malloc(sizeof(double) * SGO_CUBE);
    for (size_t cw = 0; cw < n_cw; cw++) {
        memcpy(lch, llr + cw * SGO_CUBE, sizeof(double) * SGO_CUBE);
        memset(lapp, 0, sizeof(double) * SGO_CUBE);
        memset(le, 0, sizeof(double) * SGO_CUBE);
        double n_iter = 0;
        uint64_t ng = 0, ng_p = 0;
        int phases = 0, conv = 0;
        for (int iter = 1; iter <= p->Imax && !conv; iter++) {
            for (int axis = 0; axis < 3 && !conv; axis++) {
                n_iter += 0.5;
                double al = p->alpha[3 * (iter - 1) + axis];
                for (int i = 0; i < SGO_CUBE; i++) {
                    double la = al * le[i]; /* L_A, rounded, then the sum */
                    input[i] = lch[i] + la;
                }
                uint64_t ngmax;
                run_phase(axis, input, lapp, le, p, &ng, &ngmax);
                ng_p += ngmax;
                phases++;
                if (sgo_early_termination(lapp))
                    conv = 1;
            }
        }
        if (stats) {
            stats[cw].iterations = n_iter;
            stats[cw].ng = ng;
            stats[cw].ng_p = ng_p;
            stats[cw].converged = conv;
            stats[cw].phases = phases;
        }
        if (bits) {
            /* hard_decision (D:393-415) and MSB-first packing (D:272-280) */
            uint8_t* o = bits + cw * (SGO_INFO / 8);
            int b = 0;
            for (int slice = 0; slice < SGO_K; slice++)
                for (int row = 0; row < SGO_K; row++)
                    for (int col = 0; col < SGO_K; col++, b++) {
                        int bit = (lapp[slice * 256 + row * 16 + col] > 0.0) ? 0 : 1;
                        if ((b & 7) == 0)
                            o[b >> 3] = 0;
                        o[b >> 3] = (uint8_t)((o[b >> 3] << 1) | bit);
                    }
        }
        if (lapp_out)
            memcpy(lapp_out + cw * SGO_CUBE, lapp, sizeof(double) * SGO_CUBE);
    }
    free(lch);
    free(lapp);
    free(le);
    free(input);
}

/* ------------------------------------------------------------ adjoint -- */

/* Transpose of d L_APP / d x of one line on the forward branch (the list,
 * the tested patterns and the stop held fixed), applied to g.  The soft
 * output is that of D:536-577; PM_j = sum_k JacLog(-|x_k|) + sum over the
 * positions where pattern j differs from the hard decision of
 * (JacLog(|x_k|) - JacLog(-|x_k|)), so dPM_j/dx_i = sign(x_i) ([i in S_j] -
 * sigma(-|x_i|) [|x_i| <= 50]); pNL = 2^-8 (1 - sum of exp(-PM) over the
 * counted guesses). */
static void line_vjp(const double x[SGO_N], const double g[SGO_N], const line_state* s, double gx[SGO_N])
{
    if (s->cur_l == 0) {
        for (int i = 0; i < SGO_N; i++)
            gx[i] = g[i];
        return;
    }
    const double eps = kEps;
    const int pnl_live = s->pnl > eps;
    const double p_nl = fmax(s->pnl, eps);
    double pj[8], a0[SGO_N], a1[SGO_N], pp0[SGO_N], pp1[SGO_N], sgn[SGO_N], sm[SGO_N];
    for (int j = 0; j < s->cur_l; j++)
        pj[j] = ox_exp(-s->pm_list[j]);
    for (int i = 0; i < SGO_N; i++) {
        const double pp1r = 1.0 / (1.0 + ox_exp(x[i]));
        const double pp0r = 1.0 - pp1r;
        pp1[i] = fmin(fmax(pp1r, eps), 1.0);
        pp0[i] = fmin(fmax(pp0r, eps), 1.0);
        double p0 = 0, p1 = 0;
        for (int j = 0; j < s->cur_l; j++) {
            if (s->chat[j][i])
                p1 += pj[j];
            else
                p0 += pj[j];
        }
        p0 += p_nl * pp0[i];
        p1 += p_nl * pp1[i];
        a0[i] = p0 > eps ? g[i] / p0 : 0.0;
        a1[i] = p1 > eps ? -g[i] / p1 : 0.0;
        const double dsig = pp0r * pp1r;
        gx[i] = 0.0;
        if (pp0r > eps)
            gx[i] += a0[i] * p_nl * dsig;
        if (pp1r > eps)
            gx[i] -= a1[i] * p_nl * dsig;
        const double ax = fabs(x[i]);
        sgn[i] = x[i] > 0 ? 1.0 : (x[i] < 0 ? -1.0 : 0.0);
        sm[i] = ax <= 50.0 ? 1.0 / (1.0 + ox_exp(ax)) : 0.0;
    }
    for (int j = 0; j < s->cur_l; j++) {
        double gp = 0;
        for (int i = 0; i < SGO_N; i++)
            gp += s->chat[j][i] ? a1[i] : a0[i];
        const double gpm = -pj[j] * gp;
        for (int i = 0; i < SGO_N; i++) {
            const double inS = (s->chat[j][i] != s->cHD[i]) ? 1.0 : 0.0;
            gx[i] += gpm * sgn[i] * (inS - sm[i]);
        }
    }
    if (pnl_live) {
        double gpnl = 0;
        for (int i = 0; i < SGO_N; i++)
            gpnl += a0[i] * pp0[i] + a1[i] * pp1[i];
        for (int i = 0; i < SGO_N; i++)
            gx[i] += gpnl * 0x1p-8 * sgn[i] * (s->epos[i] - sm[i] * s->etot);
    }
}

static double softplus(double z) { return z > 0 ? z + log1p(exp(-z)) : log1p(exp(z)); }

void sgo_decode_adjoint(const double* llr, const sgo_params* p, const uint8_t* code_bits, int loss_mode,
                        double* loss_out, double* grad_alpha, double* grad_llr)
{
    code_init();
    static const int stride[3] = {1, 16, 256};
    const int nph = 3 * p->Imax;
    double* ck = (double*)calloc((size_t)nph * SGO_CUBE, sizeof(double));
    double* le = (double*)calloc(SGO_CUBE, sizeof(double));
    double* lapp = (double*)calloc(SGO_CUBE, sizeof(double));
    double* gle = (double*)calloc(SGO_CUBE, sizeof(double));
    int P = 0;
    /* forward (sgo_decode's loop) with a checkpoint of L_E entering each phase */
    for (int ph = 0; ph < nph; ph++) {
        const int axis = ph % 3;
        memcpy(ck + (size_t)ph * SGO_CUBE, le, sizeof(double) * SGO_CUBE);
        for (int a = 0; a < SGO_N; a++)
            for (int b = 0; b < SGO_N; b++) {
                const int base = axis == 0 ? IDX(0, b, a) : axis == 1 ? IDX(b, 0, a) : IDX(b, a, 0);
                double v[SGO_N];
                for (int i = 0; i < SGO_N; i++) {
                    const int q = base + i * stride[axis];
                    double la = p->alpha[ph] * ck[(size_t)ph * SGO_CUBE + q];
                    v[i] = llr[q] + la;
                }
                sgo_line_out o;
                sgo_bitso(v, p->L, p->Tmax, p->thres, &o);
                for (int i = 0; i < SGO_N; i++) {
                    lapp[base + i * stride[axis]] = o.lapp[i];
                    le[base + i * stride[axis]] = o.le[i];
                }
            }
        P = ph + 1;
        if (sgo_early_termination(lapp))
            break;
    }
    /* backward */
    double loss = 0;
    for (int ph = 0; ph < nph; ph++)
        grad_alpha[ph] = 0;
    for (int i = 0; i < SGO_CUBE; i++)
        grad_llr[i] = 0;
    for (int ph = P - 1; ph >= 0; ph--) {
        const int axis = ph % 3;
        const double* lep = ck + (size_t)ph * SGO_CUBE;
        for (int a = 0; a < SGO_N; a++)
            for (int b = 0; b < SGO_N; b++) {
                const int base = axis == 0 ? IDX(0, b, a) : axis == 1 ? IDX(b, 0, a) : IDX(b, a, 0);
                double v[SGO_N], g[SGO_N], gE[SGO_N], gx[SGO_N];
                for (int i = 0; i < SGO_N; i++) {
                    const int q = base + i * stride[axis];
                    double la = p->alpha[ph] * lep[q];
                    v[i] = llr[q] + la;
                }
                sgo_line_out o;
                line_state st;
                bitso_state(v, p->L, p->Tmax, p->thres, &o, &st);
                for (int i = 0; i < SGO_N; i++) {
                    const int q = base + i * stride[axis];
                    gE[i] = gle[q];
                    g[i] = gE[i];
                    if (ph == P - 1 || loss_mode == 1) { /* the final APP, or every phase's */
                        const double sg = code_bits[q] ? 1.0 : -1.0;
                        const double z = sg * o.lapp[i];
                        loss += softplus(z);
                        g[i] += sg / (1.0 + exp(-z));
                    }
                }
                line_vjp(v, g, &st, gx);
                for (int i = 0; i < SGO_N; i++) {
                    const int q = base + i * stride[axis];
                    gx[i] -= gE[i];
                    gle[q] = p->alpha[ph] * gx[i];
                    grad_alpha[ph] += gx[i] * lep[q];
                    grad_llr[q] += gx[i];
                }
            }
    }
    *loss_out = loss;
    free(ck);
    free(le);
    free(lapp);
    free(gle);
}

/* Loss of the forward pass alone (for finite differences). */
double sgo_decode_loss(const double* llr, const sgo_params* p, const uint8_t* code_bits)
{
    double* lapp = (double*)malloc(sizeof(double) * SGO_CUBE);
    uint8_t bits[SGO_INFO / 8];
    sgo_decode(llr, 1, p, bits, lapp, NULL);
    double loss = 0;
    for (int i = 0; i < SGO_CUBE; i++)
        loss += softplus((code_bits[i] ? 1.0 : -1.0) * lapp[i]);
    free(lapp);
    return loss;
}

#if SGO_TWIN
#include "../sogrand_b200/csrc/sg_gen.h"
/* The seeded channel output of the library's generator (sg_gen.h, compiled
 * here from the same source with the same exp/log) for codewords
 * [cw0, cw0+n) at noise deviation sigma: packed info bytes (nullable) and
 * LLR cubes.  Encoding uses this file's restatement of cubic_encoder.c.
 * Lets the CPU timing legs prepare the reference's inputs without loading
 * the library. */
void sgo_gen_llr(uint64_t seed, uint64_t cw0, size_t n, double sigma, uint8_t* info, double* llr)
{
    uint8_t ib[SGO_INFO / 8], bits[SGO_INFO], cw[SGO_CUBE];
    for (size_t c = 0; c < n; c++) {
        const uint64_t gc = cw0 + c;
        for (int w = 0; w < 8; w++) {
            const uint64_t r = sg_rand(seed, 0, gc * 8 + (uint64_t)w);
            for (int q = 0; q < 8; q++)
                ib[w * 8 + q] = (uint8_t)(r >> (8 * q));
        }
        if (info)
            memcpy(info + c * (SGO_INFO / 8), ib, SGO_INFO / 8);
        for (int b = 0; b < SGO_INFO; b++) /* packed MSB first, as generate_bin/comparator files */
            bits[b] = (uint8_t)((ib[b >> 3] >> (7 - (b & 7))) & 1);
        sgo_encode(bits, cw);
        for (int p = 0; p < SGO_CUBE; p++)
            llr[c * SGO_CUBE + p] = sg_llr_of(cw[p], sigma, sg_normal(seed, gc, (uint32_t)p, k_ltab));
    }
}
#endif

double sgo_sigma(double ebn0_db) /* C:34-39, code_dim = 3 */
{
    const int n = 16, k = 8;
    const double R = pow((double)k / n, 3);
    double es = ebn0_db + 10 * log10(2 * R);
    return 1.0 / sqrt(pow(10, es / 10.0));
}
