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
 *   bits 0..15   the pattern over sorted positions (bit r = position r)
 *   bit 16       SG_ENUM_GS: first pattern of a new logistic weight; the
 *                reference checks T < Tmax before such a pattern (:652)
 * For IC >= SG_ENUM_IC_CANON the weight ranges of different Hamming weights
 * no longer interleave and the table is identical for every IC; the decoder
 * uses table SG_ENUM_IC_CANON for all of them (checked by
 * tests/test_enum.py for IC up to 4096 and sampled larger values).
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

#define SG_ENUM_LEN 65536u
#define SG_ENUM_GS 0x10000u
#define SG_ENUM_IC_CANON 56
#define SG_ENUM_NTAB (SG_ENUM_IC_CANON + 1)

#ifdef __cplusplus
extern "C" {
#endif
/* Writes the pattern order for `ic` (ic >= 0) to out[0..SG_ENUM_LEN) and
 * returns the number of patterns written: SG_ENUM_LEN on success, 0 if the
 * successor logic left its domain (never for 0 <= ic < 2^20). */
size_t sg_enum_build(int32_t ic, uint32_t* out);
#ifdef __cplusplus
}
#endif
