/* sg_enum.h -- the order in which SOGRAND tests error patterns.
 *
 * sogrand_main_logic (SOGRAND_C/cubic_decoder_final.c:587-746) tests the
 * hard decision first, then loops over logistic weights wt = IC+1 ..
 * 16*IC+136; within a weight over Hamming weights w from the bound of :653
 * upwards; within (wt, w) over the patterns produced by mountain_build
 * (:775-789) and the landslide step (:689-734).  Over the 16 reliability-
 * sorted positions the sequence of patterns depends on IC alone (n = 16,
 * even = 0).  The decoder therefore reads pattern t of a line from a table
 * built once per IC instead of re-running the successor logic per guess.
 *
 * Entry t (t = 0 is the hard decision itself):
 *   bits 0..7    sg_swz(low byte of the pattern over sorted positions):
 *                the decoder's storage index of the low byte's per-line
 *                table entries (sg_swz is its own inverse)
 *   bits 8..15   the high byte of the pattern (bit r = position 8 + r)
 *   bit 16       SG_ENUM_GS: first pattern of a new logistic weight; the
 *                reference checks T < Tmax before such a pattern (:652)
 *   bits 17..23  8 * (1 + j) for the lowest set position 8 + j of the high
 *                byte, 0 if the high byte is empty
 *   bits 24..30  the same for the second-lowest set high position
 *   bit 31       SG_ENUM_HI3: the high byte has three or more set positions
 * Bits 17..31 are derived from bits 0..15; they are byte offsets into a
 * per-line table of path-metric increments whose entry 0 is zero, so the
 * decoder adds the first two high-position increments without a loop.
 * For IC >= SG_ENUM_IC_CANON the weight ranges of different Hamming weights
 * no longer interleave and the table is identical for every IC; the decoder
 * uses table SG_ENUM_IC_CANON for all of them (checked by
 * tests/test_enum.py for IC up to 4096 and sampled larger values).
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "sg_math.h" /* SG_HD */

#define SG_ENUM_LEN 65536u
#define SG_ENUM_GS 0x10000u
#define SG_ENUM_HI3 0x80000000u
#define SG_ENUM_PATTERN_MASK 0x1ffffu /* bits 0..16: the exported order */

/* Storage index of the per-line tables' entry for low byte lo: the low
 * nibble XORed with a function of bits 5..7 (their 8 values, 0, 5, 11, 14,
 * 15, 10, 4, 1, are the nibbles of the constant, low first); it leaves bits
 * 4..7 alone, so it is its own inverse.  The 32 patterns of a warp step
 * concentrate on few residues of lo mod 16, an 8-byte table entry's
 * shared-memory bank pair; this permutation, the best of a search over
 * linear maps on the steps of 2 dB decodes, spreads them: 3.3 wavefronts
 * per lookup on average instead of 5.3. */
SG_HD uint32_t sg_swz(uint32_t lo)
{
    return lo ^ ((0x14AFEB50u >> ((lo >> 3) & 28u)) & 15u);
}

/* The pattern (bits 0..15 over sorted positions) of an order-table entry. */
SG_HD uint32_t sg_ent_pattern(uint32_t ent)
{
    return sg_swz(ent & 0xffu) | (ent & 0xff00u);
}
#define SG_ENUM_IC_CANON 56
#define SG_ENUM_NTAB (SG_ENUM_IC_CANON + 1)

/* mountain_build (cubic_decoder_final.c:775-789): set u[k+1..w) to u[k],
 * then pile the weight still missing onto the high end, n1 at a time. */
SG_HD bool sg_enum_fill(int32_t* u, int32_t k, int32_t w, int32_t W1, int32_t n1)
{
    for (int32_t i = k + 1; i < w; i++)
        u[i] = u[k];
    int64_t rest = W1;
    for (int32_t i = 0; i < w; i++)
        rest -= u[i];
    int64_t room = (int64_t)n1 - u[k];
    if (rest < 0 || room <= 0)
        return false;
    int64_t q = rest / room;
    int64_t r = rest - q * room;
    if (q > w)
        return false;
    for (int64_t i = w - q; i < w; i++)
        u[i] = n1;
    if (w > q)
        u[w - q - 1] += (int32_t)r;
    return true;
}

/* Entry of pattern m (bits 0..15) with flag bits: adds bits 17..31. */
SG_HD uint32_t sg_enum_entry(uint32_t m, uint32_t flag)
{
    uint32_t hi = (m >> 8) & 0xffu, o1 = 0, o2 = 0;
    if (hi) {
        int j = 0;
        while (!((hi >> j) & 1u))
            j++;
        o1 = 8u * (uint32_t)(1 + j);
        hi &= hi - 1u;
    }
    if (hi) {
        int j = 0;
        while (!((hi >> j) & 1u))
            j++;
        o2 = 8u * (uint32_t)(1 + j);
        hi &= hi - 1u;
    }
    return sg_swz(m & 0xffu) | (m & 0xff00u) | flag | (o1 << 17) | (o2 << 24) | (hi ? SG_ENUM_HI3 : 0u);
}

/* The builder, usable on host and device (same source, same order): writes
 * the pattern order for `ic` (ic >= 0) to out[0..SG_ENUM_LEN) and returns the
 * number of patterns written: SG_ENUM_LEN on success, 0 if the successor
 * logic left its domain (never for 0 <= ic < 2^20). */
SG_HD size_t sg_enum_build_impl(int32_t ic, uint32_t* out)
{
    const int32_t n = 16;
    size_t t = 0;
    out[t++] = 0; /* the hard decision, tested before the loop (:624-641) */
    const int32_t wt_max = ic * n + n * (n + 1) / 2;
    const double temp = 1 + 2 * ((double)n + (double)ic);
    int32_t u[16];
    for (int32_t wt = ic + 1; wt <= wt_max; wt++) {
        uint32_t flag = SG_ENUM_GS;
        /* smallest Hamming weight that can reach logistic weight wt (:653) */
        int32_t w = (int32_t)ceil((temp - sqrt(temp * temp - 8.0 * wt)) / 2);
        if (w < 1)
            w = 1;
        for (; w <= n; w++) {
            const int32_t W = wt - ic * w;
            if (W < w * (w + 1) / 2)
                break;
            const int32_t W1 = W - w * (w + 1) / 2;
            const int32_t n1 = n - w;
            if (n1 == 0) { /* the all-ones pattern; the reference divides by zero here */
                if (t >= SG_ENUM_LEN)
                    return 0;
                out[t++] = sg_enum_entry(0xffffu, flag);
                flag = 0;
                continue;
            }
            for (int i = 0; i < 16; i++)
                u[i] = 0;
            if (!sg_enum_fill(u, 0, w, W1, n1))
                return 0;
            for (;;) {
                if (t >= SG_ENUM_LEN)
                    return 0;
                uint32_t m = 0;
                for (int32_t i = 0; i < w; i++)
                    m |= 1u << (i + u[i]);
                out[t++] = sg_enum_entry(m, flag);
                flag = 0;
                /* landslide (:689-734): move the highest position that is at
                 * least 2 below the top one place up and refill above it */
                if (u[w - 1] - u[0] < 2)
                    break;
                int32_t k = 0;
                for (int32_t i = w - 1; i > 0; i--)
                    if (u[w - 1] - u[i] >= 2) {
                        k = i;
                        break;
                    }
                u[k]++;
                if (!sg_enum_fill(u, k, w, W1, n1))
                    return 0;
            }
        }
    }
    return t;
}
