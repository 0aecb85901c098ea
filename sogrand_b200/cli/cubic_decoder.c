/* cubic_decoder -- drop-in replacement for the reference decoder process.
 *
 * Same invocation, files and statistics as SOGRAND_C/cubic_decoder_final.c
 * (usage :63-66, input/output :104-119 and :271-294, statistics :299-304)
 * plus the throughput line of SOGRAND_CUDA/cubic_decoder1.cu:1159-1164.
 * Totals are 64-bit here (the reference's int totals overflow above about
 * 1,090 codewords at 2 dB).  "Total CPU time" reports the wall time of the
 * decode call.
 */
#include <stdio.h>

#include "sogrand_b200.h"

int main(int argc, char* argv[])
{
    if (argc != 3) {
        fprintf(stderr, "Usage: %s <input_llr_file> <output_file>\n", argv[0]);
        return 1;
    }
    sg_params p;
    sg_params_default(&p);
    sg_run_summary s;
    sg_status st = sg_decode_file(argv[1], argv[2], &p, 0, &s);
    if (st != SG_OK) {
        fprintf(stderr, "%s\n", sg_last_error());
        return 1;
    }
    const double blocks = (double)s.blocks;
    printf("Decoding complete. %llu block(s) decoded.\n", (unsigned long long)s.blocks);
    printf("Average iterations per block: %.2f\n", s.total_iterations / blocks);
    printf("Average NG per block: %.2f\n", (double)s.total_ng / blocks);
    printf("Average NG per info bit: %.2f\n", (double)s.total_ng / (blocks * SG_INFO_BITS));
    printf("Average NG_p per block: %.2f\n", (double)s.total_ng_p / blocks);
    printf("Total CPU time: %.2f seconds\n", s.seconds);
    printf("Throughput: %.2f blocks/sec\n", s.seconds > 0 ? blocks / s.seconds : 0.0);
    return 0;
}
