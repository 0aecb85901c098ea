/* ref_harness.c -- per-codeword driver around the unmodified reference.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles the reference's
 * SOGRAND_C/cubic_decoder_final.c, unmodified, with -Dmain=sgref_ref_main,
 * and links it with this file into oracle/_ref/libsgref.so.  The reference
 * main() prints only averages; this driver restates its per-codeword loop
 * (SOGRAND_C/cubic_decoder_final.c:119-289) around the reference's own
 * SOGRAND_bitSO, early_termination and hard_decision so that fixtures can
 * record per-codeword statistics.  Its averages and decoded bits are checked
 * against the unmodified flow binary by tests/golden/make_golden.py.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    double* data;
    int dim1, dim2, dim3;
} ref_tensor_d; /* Tensor_d, cubic_decoder_final.c:20-23 */

/* Reference symbols (cubic_decoder_final.c:42-45, :439). */
int** create_int_matrix(int rows, int cols);
void free_int_matrix(int** matrix, int rows);
void getGH_sys_CRC(int n, int k, int** G, int** H);
int early_termination(ref_tensor_d L_APP, int** G, int n, int k);
void hard_decision(double* llr, int* bits, int length);
void SOGRAND_bitSO(double* L_APP, double* L_E, int* N_guess, double* llr, int** H_matrix,
                   int n, int k, int L, uint64_t Tmax, double thres, int even);
void sogrand_main_logic(double* chat_list, double* s_list, double* T_val, double* curL_val, double* pNL_val,
                        double* APP_list, double* llr, uint8_t* H_flat, int n, int s, int IC, uint64_t L,
                        uint64_t Tmax, double thres, int even);

static int** g_G;
static int** g_H;
static int g_even = -1;

static void init(void)
{
    if (g_G)
        return;
    g_G = create_int_matrix(8, 16);
    g_H = create_int_matrix(8, 16);
    getGH_sys_CRC(16, 8, g_G, g_H);
    g_even = 1; /* :82-92 */
    for (int i = 0; i < 8 && g_even; i++) {
        int s = 0;
        for (int j = 0; j < 16; j++)
            s += g_G[i][j];
        if (s % 2 != 0)
            g_even = 0;
    }
}

int sgref_even(void)
{
    init();
    return g_even;
}

void sgref_code_matrices(uint8_t* G, uint8_t* H)
{
    init();
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 16; j++) {
            G[i * 16 + j] = (uint8_t)g_G[i][j];
            H[i * 16 + j] = (uint8_t)g_H[i][j];
        }
}

/* One SOGRAND_bitSO call on a 16-LLR line. */
void sgref_bitso(const double* llr, int L, uint64_t Tmax, double thres,
                 double* lapp, double* le, int* n_guess)
{
    init();
    double v[16];
    memcpy(v, llr, sizeof v);
    SOGRAND_bitSO(lapp, le, n_guess, v, g_H, 16, 8, L, Tmax, thres, g_even);
}

/* Whether SOGRAND_bitSO on this line reads its uninitialised list size
 * (cubic_decoder_final.c:524, :536): the reference's sogrand_main_logic is
 * run with that output preset to -1, and a line whose search lists no
 * codeword (possible only under a finite Tmax) leaves it there.  Returns 1
 * for such a line, 0 otherwise; *T_out (nullable) receives its T. */
int sgref_line_undefined(const double* llr, int L, uint64_t Tmax, double thres, double* T_out)
{
    init();
    double v[16], chat[16 * 8], sl[4 * 8], app[8], T = 0, curl = -1.0, pnl = 0;
    uint8_t hf[8 * 16];
    if (L < 1 || L > 8)
        return -1;
    memcpy(v, llr, sizeof v);
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 16; j++)
            hf[i * 16 + j] = (uint8_t)g_H[i][j];
    sogrand_main_logic(chat, sl, &T, &curl, &pnl, app, v, hf, 16, 8, -1, (uint64_t)L, Tmax, thres, g_even);
    if (T_out)
        *T_out = T;
    return curl == -1.0;
}

int sgref_early_termination(const double* lapp)
{
    init();
    ref_tensor_d t = {(double*)lapp, 16, 16, 16};
    return early_termination(t, g_G, 16, 8);
}

/* Decode n_cw cubes with the reference's functions.  alpha has 100 entries
 * indexed as the reference does (alpha[2*iter-2] columns, alpha[2*iter-1]
 * rows and slices).  Any output pointer may be NULL. */
static void decode_impl(const double* llr, size_t n_cw, int L, int Imax, uint64_t Tmax, double thres,
                        const double* alpha, uint8_t* bits, double* lapp_out, double* iters, uint64_t* ng_out,
                        uint64_t* ngp_out, int* conv_out, int* undef_out);

void sgref_decode(const double* llr, size_t n_cw, int L, int Imax, uint64_t Tmax,
                  double thres, const double* alpha, uint8_t* bits, double* lapp_out,
                  double* iters, uint64_t* ng_out, uint64_t* ngp_out, int* conv_out)
{
    decode_impl(llr, n_cw, L, Imax, Tmax, thres, alpha, bits, lapp_out, iters, ng_out, ngp_out, conv_out, NULL);
}

/* sgref_decode that also counts, per codeword, the line decodes that read
 * the reference's uninitialised list size (sgref_line_undefined); the
 * codeword's outputs are undefined when the count is not 0. */
void sgref_decode_checked(const double* llr, size_t n_cw, int L, int Imax, uint64_t Tmax,
                          double thres, const double* alpha, uint8_t* bits, double* lapp_out,
                          double* iters, uint64_t* ng_out, uint64_t* ngp_out, int* conv_out, int* undef_out)
{
    decode_impl(llr, n_cw, L, Imax, Tmax, thres, alpha, bits, lapp_out, iters, ng_out, ngp_out, conv_out,
                undef_out);
}

static void decode_impl(const double* llr, size_t n_cw, int L, int Imax, uint64_t Tmax, double thres,
                        const double* alpha, uint8_t* bits, double* lapp_out, double* iters, uint64_t* ng_out,
                        uint64_t* ngp_out, int* conv_out, int* undef_out)
{
    init();
    const int n = 16, N3 = 4096;
    double* lch = malloc(sizeof(double) * N3);
    double* lapp = malloc(sizeof(double) * N3);
    double* le = malloc(sizeof(double) * N3);
    double* la = malloc(sizeof(double) * N3);
    double* in = malloc(sizeof(double) * N3);
    double vin[16], vapp[16], vle[16];
    int hb[512];
    for (size_t cw = 0; cw < n_cw; cw++) {
        memcpy(lch, llr + cw * N3, sizeof(double) * N3);
        memset(lapp, 0, sizeof(double) * N3);
        memset(le, 0, sizeof(double) * N3);
        double n_iter = 0;
        int NG = 0, NG_p = 0, conv = 0, undef = 0;
        for (int iter = 1; iter <= Imax && !conv; iter++) {
            for (int ph = 0; ph < 3 && !conv; ph++) {
                int NGmax = 0;
                n_iter += 0.5;
                double a = alpha[ph == 0 ? 2 * iter - 2 : 2 * iter - 1];
                for (int i = 0; i < N3; i++)
                    la[i] = a * le[i];
                for (int i = 0; i < N3; i++)
                    in[i] = lch[i] + la[i];
                for (int x = 0; x < n; x++)
                    for (int y = 0; y < n; y++) {
                        int base, st;
                        if (ph == 0) { base = x * 256 + y * 16; st = 1; }        /* slice x, col y */
                        else if (ph == 1) { base = x * 256 + y; st = 16; }       /* slice x, row y */
                        else { base = x * 16 + y; st = 256; }                    /* col x, row y */
                        for (int i = 0; i < n; i++)
                            vin[i] = in[base + i * st];
                        int ngs = 0;
                        if (undef_out)
                            undef += sgref_line_undefined(vin, L, Tmax, thres, NULL) == 1;
                        SOGRAND_bitSO(vapp, vle, &ngs, vin, g_H, n, 8, L, Tmax, thres, g_even);
                        NG += ngs;
                        if (ngs > NGmax)
                            NGmax = ngs;
                        for (int i = 0; i < n; i++) {
                            lapp[base + i * st] = vapp[i];
                            le[base + i * st] = vle[i];
                        }
                    }
                NG_p += NGmax;
                ref_tensor_d t = {lapp, 16, 16, 16};
                if (early_termination(t, g_G, n, 8))
                    conv = 1;
            }
        }
        if (iters) iters[cw] = n_iter;
        if (ng_out) ng_out[cw] = (uint64_t)(unsigned)NG;
        if (ngp_out) ngp_out[cw] = (uint64_t)(unsigned)NG_p;
        if (conv_out) conv_out[cw] = conv;
        if (undef_out) undef_out[cw] = undef;
        if (bits) {
            hard_decision(lapp, hb, 512);
            uint8_t* o = bits + cw * 64;
            for (int b = 0; b < 512; b++) {
                if ((b & 7) == 0)
                    o[b >> 3] = 0;
                o[b >> 3] = (uint8_t)((o[b >> 3] << 1) | hb[b]);
            }
        }
        if (lapp_out)
            memcpy(lapp_out + cw * N3, lapp, sizeof(double) * N3);
    }
    free(lch);
    free(lapp);
    free(le);
    free(la);
    free(in);
}
