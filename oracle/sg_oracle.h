/* sg_oracle.h -- CPU restatement of the SOGRAND (16,8)^3 cubic decoder.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA decoder in
 * sogrand_b200/; nothing in the product links it.  It restates, function by
 * function, SOGRAND_C/cubic_decoder_final.c (the decoder that
 * SOGRAND_C/cubic_flow.sh:44 runs) and SOGRAND_C/cubic_encoder.c.
 *
 * Build modes (oracle/Makefile):
 *   libsg_oracle.so       exp/log from the system libm, as the reference.
 *   libsg_oracle_twin.so  exp/log from sogrand_b200/csrc/sg_math.h, the
 *                         routines the CUDA kernel uses; its results must
 *                         equal the kernel's bit for bit, soft values too.
 * Both are compiled with -O2 -ffp-contract=off for baseline x86-64, which
 * matches the reference flow build (plain gcc, no FMA contraction).
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SGO_N 16
#define SGO_K 8
#define SGO_CUBE 4096
#define SGO_INFO 512
#define SGO_MAX_PHASES 150 /* 3 phases x 50 iterations (alpha[100] in the reference) */

typedef struct {
    int L;              /* list size, reference 3 (cubic_decoder_final.c:94) */
    int Imax;           /* iterations, reference 30 (:95) */
    uint64_t Tmax;      /* abandonment cap, reference UINT64_MAX (:96) */
    double thres;       /* 1 - p_ET, reference 1 - 1e-5 (:97-98) */
    double alpha[SGO_MAX_PHASES]; /* one weight per phase, see sgo_default_params */
} sgo_params;

typedef struct {
    double iterations;  /* 0.5 per phase, as n_iter (:145) */
    uint64_t ng;        /* total guesses (NG, :162) */
    uint64_t ng_p;      /* sum over phases of the max line guesses (NG_p, :170) */
    int converged;      /* early termination fired */
    int phases;         /* phases run */
} sgo_cw_stats;

typedef struct {
    double lapp[SGO_N];
    double le[SGO_N];
    uint64_t n_guess;   /* T */
    int cur_l;          /* codewords found */
    double pnl;         /* P(not in list) used for the soft output */
} sgo_line_out;

/* Reference parameters with alpha = 0.7 everywhere (:100-102).  The
 * reference indexes alpha[2*iter-2] for the column phase and alpha[2*iter-1]
 * for the row and slice phases (:149, :188, :227); alpha here is per phase,
 * alpha[3*(iter-1) + p], so a constant array reproduces it exactly. */
void sgo_default_params(sgo_params* p);

/* Component code from Koopman polynomial 0xeb (getGH_sys_CRC, :468-519).
 * G is 8x16, H is 8x16, row-major 0/1 bytes. */
void sgo_code_matrices(uint8_t G[SGO_K * SGO_N], uint8_t H[(SGO_N - SGO_K) * SGO_N]);

/* One component SISO decode (SOGRAND_bitSO, :521-585, with
 * sogrand_main_logic, :587-746). */
void sgo_bitso(const double llr[SGO_N], int L, uint64_t Tmax, double thres, sgo_line_out* out);

/* Early-termination test on an L_APP cube (early_termination, :317-391). */
int sgo_early_termination(const double* lapp);

/* Decode n_cw cubes (layout slice*256 + col*16 + row, C row index fastest).
 * bits: 64 bytes per codeword, MSB first (:267-280).  lapp (nullable):
 * final L_APP cubes.  stats (nullable). */
void sgo_decode(const double* llr, size_t n_cw, const sgo_params* p,
                uint8_t* bits, double* lapp, sgo_cw_stats* stats);

/* Systematic product encoding of 512 info bits (cubic_encoder.c:23-100).
 * info: 512 bytes 0/1 in info order; cw: 4096 bytes 0/1 in cube order. */
void sgo_encode(const uint8_t info[SGO_INFO], uint8_t cw[SGO_CUBE]);

/* Noise standard deviation of channel_sim.c:34-39 for code dimension 3. */
double sgo_sigma(double ebn0_db);

/* Twin build only (libsg_oracle_twin.so): the library generator's seeded
 * channel output, for preparing reference inputs without the library. */
void sgo_gen_llr(uint64_t seed, uint64_t cw0, size_t n, double sigma, uint8_t* info, double* llr);

/* FP64 adjoint of one codeword's decode (the branch of the forward pass
 * held fixed): loss = sum_i softplus(s_i L_APP_i) over the 4096 code bits,
 * s_i = +1 for bit 1, -1 for 0, of the final APP (loss_mode 0) or summed
 * over every phase's APP (loss_mode 1); grad_alpha[3*Imax] and
 * grad_llr[4096] its gradients.  Requires Tmax = UINT64_MAX. */
void sgo_decode_adjoint(const double* llr, const sgo_params* p, const uint8_t* code_bits, int loss_mode,
                        double* loss, double* grad_alpha, double* grad_llr);
double sgo_decode_loss(const double* llr, const sgo_params* p, const uint8_t* code_bits);

/* Which exp/log this build uses: 0 = libm, 1 = sg_math.h. */
int sgo_math_mode(void);

/* exp and log as this build evaluates them. */
double sgo_exp(double x);
double sgo_log(double x);

/* The oracle's own pattern order for reliability shift ic, produced by its
 * restatement of the loops of sogrand_main_logic (D:642-744) without
 * stopping: bits 0..15 the pattern, bit 16 first pattern of a logistic
 * weight.  Returns the count written (65536 when cap allows). */
size_t sgo_pattern_order(int32_t ic, uint32_t* out, size_t cap);

#ifdef __cplusplus
}
#endif
