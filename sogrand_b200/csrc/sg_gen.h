/* sg_gen.h -- seeded synthetic source, encoder and AWGN channel, shared by
 * the host generator and the device generator so that both produce the
 * same bits.
 *
 * The reference pipeline (generate_bin.c, cubic_encoder.c, channel_sim.c)
 * seeds rand() with time(NULL).  Here every random number is a pure function
 * of (seed, stream, counter), so codeword c is the same whichever batch,
 * device or host produces it:
 *   info word w of codeword c      sg_rand(seed, 0, c*8 + w)
 *   noise of position p, attempt a (u, v) = sg_rand(seed, 1+2a / 2+2a, c*4096+p)
 *   per-codeword Eb/N0 draw        sg_rand(seed, 7, c)
 * Noise is N(0,1) by the Marsaglia polar method with the decoder's own log
 * (sg_math.h), so host and device agree bit for bit.  The LLR is formed as
 * channel_sim.c:61-80 forms it: x = +1 for bit 0, y = x + sigma*z,
 * llr = 2*y / sigma^2.
 */
#pragma once
#include <stdint.h>
#include "sg_math.h"

SG_HD uint64_t sg_mix64(uint64_t z)
{
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ULL;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebULL;
    z ^= z >> 31;
    return z;
}

SG_HD uint64_t sg_rand(uint64_t seed, uint64_t stream, uint64_t ctr)
{
    uint64_t k = sg_mix64(seed + 0x9e3779b97f4a7c15ULL * (stream + 1));
    return sg_mix64(k ^ (ctr * 0xd1b54a32d192ed03ULL + 0x8cb92ba72f3d8dd7ULL));
}

/* uniform in [-1, 1) with 2^-52 spacing */
SG_HD double sg_sym_unit(uint64_t r)
{
    return (double)(r >> 11) * 0x1p-52 - 1.0;
}

/* One standard normal for position (c, p): polar method.  A pair is
 * rejected with probability 1 - pi/4; after SG_POLAR_TRIES rejections in a
 * row (probability < 1e-42) the sample is 0. */
#define SG_POLAR_TRIES 64
SG_HD double sg_normal(uint64_t seed, uint64_t c, uint32_t p, const double* ltab)
{
    uint64_t ctr = c * 4096u + p;
    /* draw until a pair lands inside the unit disc; the transform runs once,
     * after the loop, so that lanes needing different numbers of draws
     * share it on a GPU */
    double u = 0.0, s = 0.0;
    int ok = 0;
    for (uint64_t a = 0; a < SG_POLAR_TRIES; a++) {
        u = sg_sym_unit(sg_rand(seed, 1 + 2 * a, ctr));
        double v = sg_sym_unit(sg_rand(seed, 2 + 2 * a, ctr));
        double uu = u * u;
        double vv = v * v;
        s = uu + vv;
        if (s > 0.0 && s < 1.0) {
            ok = 1;
            break;
        }
    }
    if (!ok)
        return 0.0;
    double l = sg_log(s, ltab);
    double m = -2.0 * l;
    double q = m / s;
#if defined(__CUDA_ARCH__)
    double f = __dsqrt_rn(q);
#else
    double f = sqrt(q);
#endif
    return u * f;
}

/* Noise deviation of codeword c when Eb/N0 is drawn uniformly from
 * [lo, hi] dB: sigma = 1/sqrt(10^(EsN0/10)), EsN0 = EbN0 + 10*log10(2R),
 * R = 1/8 (channel_sim.c:34-39), with 10^x = exp(x*ln 10) by sg_exp. */
SG_HD double sg_sigma_draw(uint64_t seed, uint64_t c, double lo, double hi, const double* etab)
{
    double u = (double)(sg_rand(seed, 7, c) >> 11) * 0x1p-53;
    double eb = lo + (hi - lo) * u;
    double es = eb + 10.0 * -0x1.34413509f79ffp-1; /* log10(0.25) */
    double pw = sg_exp((es / 10.0) * 0x1.26bb1bbb55516p+1, etab); /* ln 10 */
#if defined(__CUDA_ARCH__)
    return 1.0 / __dsqrt_rn(pw);
#else
    return 1.0 / sqrt(pw);
#endif
}

SG_HD double sg_llr_of(int bit, double sigma, double z)
{
    double x = bit ? -1.0 : 1.0;
    double noise = sigma * z;
    double y = x + noise;
    double var = sigma * sigma;
    return 2.0 * y / var;
}

SG_HD uint32_t sg_brev8(uint32_t b)
{
    b = ((b & 0xf0u) >> 4) | ((b & 0x0fu) << 4);
    b = ((b & 0xccu) >> 2) | ((b & 0x33u) << 2);
    b = ((b & 0xaau) >> 1) | ((b & 0x55u) << 1);
    return b;
}

/* Encode one codeword into 256 line words W[slice*16 + col] whose bit `row`
 * is the code bit at cube index slice*256 + col*16 + row.  info: 64 packed
 * bytes, info bit l*64 + j*8 + i sits at (row i, col j, slice l)
 * (cubic_encoder.c:28-42).  The product code is encoded line-wise with the
 * parity tables of sg_code.h: parity columns within the first 8 slices,
 * then parity rows, then parity slices (cubic_encoder.c:45-86; the order
 * does not change the codeword). */
SG_HD void sg_encode_words(const uint8_t* info, const uint8_t* prow, const uint8_t* ptab,
                           uint16_t* W)
{
    for (int i = 0; i < 256; i++)
        W[i] = 0;
    for (int l = 0; l < 8; l++)
        for (int j = 0; j < 8; j++)
            W[l * 16 + j] = (uint16_t)sg_brev8(info[l * 8 + j]);
    for (int l = 0; l < 8; l++)
        for (int jj = 0; jj < 8; jj++) {
            uint16_t acc = 0;
            for (int j = 0; j < 8; j++)
                if ((prow[j] >> jj) & 1)
                    acc ^= W[l * 16 + j];
            W[l * 16 + 8 + jj] = acc;
        }
    for (int l = 0; l < 8; l++)
        for (int j = 0; j < 16; j++) {
            uint16_t x = W[l * 16 + j];
            W[l * 16 + j] = (uint16_t)((x & 0xff) | (ptab[x & 0xff] << 8));
        }
    for (int jj = 0; jj < 8; jj++)
        for (int j = 0; j < 16; j++) {
            uint16_t acc = 0;
            for (int l = 0; l < 8; l++)
                if ((prow[l] >> jj) & 1)
                    acc ^= W[l * 16 + j];
            W[(8 + jj) * 16 + j] = acc;
        }
}
