/* sg_enum.cpp -- builds the error-pattern order tables (see sg_enum.h). */
#include "sg_enum.h"

#include <math.h>
#include <string.h>

namespace {

/* mountain_build (cubic_decoder_final.c:775-789): set u[k+1..w) to u[k],
 * then pile the weight still missing onto the high end, n1 at a time. */
bool fill(int32_t* u, int32_t k, int32_t w, int32_t W1, int32_t n1)
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

uint32_t pattern(const int32_t* u, int32_t w)
{
    uint32_t m = 0;
    for (int32_t i = 0; i < w; i++)
        m |= 1u << (i + u[i]);
    return m;
}

} // namespace

extern "C" size_t sg_enum_build(int32_t ic, uint32_t* out)
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
                out[t++] = 0xffffu | flag;
                flag = 0;
                continue;
            }
            memset(u, 0, sizeof u);
            if (!fill(u, 0, w, W1, n1))
                return 0;
            for (;;) {
                if (t >= SG_ENUM_LEN)
                    return 0;
                out[t++] = pattern(u, w) | flag;
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
                if (!fill(u, k, w, W1, n1))
                    return 0;
            }
        }
    }
    return t;
}
