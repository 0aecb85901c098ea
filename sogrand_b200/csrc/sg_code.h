/* sg_code.h -- the (16,8) component code and its product-code tables.
 *
 * The component code is the systematic CRC code of getGH_sys_CRC
 * (SOGRAND_C/cubic_decoder_final.c:468-519) for n = 16, k = 8 and the
 * Koopman polynomial 0xeb (:478): G = [I | P], H = [P^T | I].  Bits of a
 * line are held in a 16-bit word, bit i = position i of the line; positions
 * 0..7 carry information and 8..15 parity.
 *
 *   prow[i]  parity byte contributed by info position i (row i of P)
 *   hcol[i]  syndrome byte of position i (column i of H)
 *   ptab[m]  parity byte of info byte m; a line word x is a codeword iff
 *            (x >> 8) == ptab[x & 0xff]
 */
#pragma once
#include <stdint.h>

typedef struct {
    uint8_t prow[8];
    uint8_t hcol[16];
    uint8_t ptab[256];
} sg_code_tables;

/* Long division of x^(7-i) * x^8 ... restated: P row i is the remainder of
 * the unit message e_i divided by the generator whose coefficients are the
 * Koopman form 0xeb followed by a trailing 1 (koopman2matlab, :454-466). */
static inline void sg_code_build(sg_code_tables* t)
{
    const unsigned koop = 0xeb;
    int len = 0;
    while ((koop >> len) > 1u)
        len++;
    len += 1; /* floor(log2(0xeb)) + 1 = 8 */
    int poly[16] = {0};
    for (int i = 0; i < len; i++)
        poly[i] = (int)((koop >> (len - 1 - i)) & 1u);
    poly[len] = 1;
    for (int i = 0; i < 8; i++) {
        int m[32] = {0};
        m[i] = 1;
        for (int j = 0; j < 8; j++)
            if (m[j])
                for (int l = 0; l <= len; l++)
                    m[j + l] ^= poly[l];
        uint8_t row = 0;
        for (int j = 0; j < 8; j++)
            row |= (uint8_t)(m[8 + j] << j);
        t->prow[i] = row;
    }
    for (int i = 0; i < 8; i++)
        t->hcol[i] = t->prow[i];
    for (int j = 0; j < 8; j++)
        t->hcol[8 + j] = (uint8_t)(1u << j);
    for (int m = 0; m < 256; m++) {
        uint8_t p = 0;
        for (int i = 0; i < 8; i++)
            if ((m >> i) & 1)
                p ^= t->prow[i];
        t->ptab[m] = p;
    }
}
