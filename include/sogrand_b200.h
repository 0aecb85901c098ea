/* sogrand_b200.h -- C ABI of the B200 SOGRAND decoder for the (16,8)^3
 * cubic product code.
 *
 * The reference has no library API: its decoder is a process,
 *   cubic_decoder <input_llr_file> <output_file>
 * (SOGRAND_C/cubic_decoder_final.c:62-314), with one internal per-line
 * boundary, SOGRAND_bitSO (SOGRAND_C/cubic_decoder_final.c:521).  This
 * library replaces both: sg_decode_file() is the process contract (same
 * file formats, same statistics), sg_decode_host()/sg_decode_device() are
 * the per-codeword loop of main() (:119-289) as a call, and sg_bitso_*()
 * is SOGRAND_bitSO over a batch of lines.
 *
 * Conventions
 *  - All entry points return sg_status; none calls exit().  The text of the
 *    last error on the calling thread is available from sg_last_error().
 *  - *_host entry points take host pointers and are synchronous.
 *  - *_device entry points take device pointers on the current CUDA device,
 *    enqueue work on `stream` (a cudaStream_t, NULL for the legacy default
 *    stream) and return without synchronising.
 *  - The caller owns every buffer.  The library keeps, per device, a
 *    read-only table of error-pattern orders (15 MB) built on first use.
 *  - LLR cube layout, as in the reference files: 4096 float64 per codeword,
 *    index slice*256 + col*16 + row in the reference's (row, col, slice)
 *    tensor terms (SOGRAND_C/cubic_decoder_final.c:434-437), i.e. the order
 *    in which cubic_encoder writes bits (SOGRAND_C/cubic_encoder.c:89-97).
 *  - Decoded bits: 64 bytes per codeword, the 512 info bits packed MSB
 *    first in the order of hard_decision (SOGRAND_C/cubic_decoder_final.c:
 *    393-415, packing :272-280).
 */
#ifndef SOGRAND_B200_H
#define SOGRAND_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SG_N 16
#define SG_K 8
#define SG_CUBE 4096
#define SG_INFO_BITS 512
#define SG_INFO_BYTES 64
#define SG_MAX_IMAX 50                  /* alpha[100] in the reference */
#define SG_MAX_PHASES (3 * SG_MAX_IMAX)
#define SG_MAX_L 8

typedef enum {
    SG_OK = 0,
    SG_ERR_ARG = 1,       /* invalid argument or parameter */
    SG_ERR_CUDA = 2,      /* a CUDA runtime call failed */
    SG_ERR_NONFINITE = 3, /* an input LLR is NaN or infinite */
    SG_ERR_IO = 4,        /* file could not be opened, read or written */
    SG_ERR_NOMEM = 5,     /* host or device allocation failed */
    SG_ERR_TIMEOUT = 6    /* a bounded device-side wait gave up */
} sg_status;

/* Decoder parameters (SOGRAND_C/cubic_decoder_final.c:94-102). */
typedef struct {
    int32_t L;        /* list size, 1..SG_MAX_L; reference 3 */
    int32_t Imax;     /* iterations, 1..SG_MAX_IMAX; reference 30 */
    uint64_t Tmax;    /* per-line abandonment cap, checked where the
                         reference checks it (once per logistic weight);
                         UINT64_MAX = none (reference) */
    double thres;     /* list-confidence stop, reference 1 - 1e-5 */
    /* extrinsic weight of each phase: phase p of iteration i (1-based,
       p = 0 columns, 1 rows, 2 slices) uses alpha[3*(i-1) + p].  The
       reference uses alpha[2i-2] for columns and alpha[2i-1] for rows and
       slices of a constant 0.7 array (:101-102, :149, :188, :227). */
    double alpha[SG_MAX_PHASES];
} sg_params;

/* Per-codeword statistics (the reference prints only their averages,
 * :299-304; its int totals overflow above ~1,090 codewords at 2 dB). */
typedef struct {
    double iterations; /* 0.5 per phase run, as n_iter (:145, :184, :223) */
    uint64_t ng;       /* guesses, summed over all line decodes (NG) */
    uint64_t ng_p;     /* sum over phases of the largest line NG (NG_p) */
    int32_t converged; /* 1: early termination fired; 0: Imax reached;
                          -1: input not finite, codeword not decoded;
                          -2: not decoded because a bounded device wait
                          gave up (see sg_check_device) */
    int32_t phases;    /* phases run */
} sg_cw_stats;

/* Totals of a file decode (the stdout block of :299-304). */
typedef struct {
    uint64_t blocks;
    double total_iterations;
    uint64_t total_ng;
    uint64_t total_ng_p;
    double seconds;    /* wall time of the whole call */
} sg_run_summary;

/* Reference parameters: L=3, Imax=30, Tmax=UINT64_MAX, thres=1-1e-5,
 * alpha=0.7. */
void sg_params_default(sg_params* p);

/* Decode n_cw LLR cubes on the GPU (device pointers, asynchronous).
 * d_llr must be 8-byte aligned (16-byte aligned uses bulk async copies in
 * the variants that stage the channel cube in shared memory).
 * d_lapp (nullable): final L_APP cubes, 4096 float64 per codeword.
 * d_stats (nullable): one sg_cw_stats per codeword.  A codeword whose
 * bulk-copy wait gave up is reported with converged = -2 and zero bits, and
 * the device's error flag is set (sg_check_device).
 * Replaces the per-codeword loop of main(), cubic_decoder_final.c:119-289. */
sg_status sg_decode_device(const double* d_llr, size_t n_cw, const sg_params* p,
                           uint8_t* d_bits, double* d_lapp, sg_cw_stats* d_stats,
                           void* stream);

/* Same with host buffers: copies in, decodes, copies out, synchronises.
 * Runs the batched persistent decoder (current sg_batch variant) over
 * chunks of at most 16384 codewords, two in flight on two streams, so
 * copies overlap decoding (pinned host buffers let the copies run
 * asynchronously).  The chunk buffers, streams and queues are allocated by
 * the first call on each device (about 1 GiB, 1 GiB more once L_APP is
 * requested) and kept until the process exits; calls on one device are
 * serialised.  Results
 * are bit-identical to sg_decode_device.  Returns SG_ERR_NONFINITE (after
 * decoding the rest) if any codeword had a non-finite LLR; those codewords
 * report converged = -1. */
sg_status sg_decode_host(const double* llr, size_t n_cw, const sg_params* p,
                         uint8_t* bits, double* lapp, sg_cw_stats* stats);

/* SOGRAND_bitSO (cubic_decoder_final.c:521-585) on n_lines independent
 * 16-LLR lines: d_llr [n_lines][16] -> d_lapp, d_le [n_lines][16],
 * d_nguess [n_lines] (the N_guess output), d_ncw [n_lines] (nullable:
 * codewords found, the reference's curL).  Device pointers, asynchronous. */
sg_status sg_bitso_device(const double* d_llr, size_t n_lines, int32_t L, uint64_t Tmax,
                          double thres, double* d_lapp, double* d_le, int32_t* d_nguess,
                          int32_t* d_ncw, void* stream);
sg_status sg_bitso_host(const double* llr, size_t n_lines, int32_t L, uint64_t Tmax,
                        double thres, double* lapp, double* le, int32_t* nguess, int32_t* ncw);

/* The process contract of cubic_decoder (cubic_decoder_final.c:62-314):
 * reads whole cubes of float64 LLRs from in_path (a trailing partial cube is
 * ignored, as the reference's fread loop does), writes packed bits to
 * out_path (a final partial byte, never produced for 512-bit blocks, would
 * be left-shifted), fills *summary (nullable).  Decodes in chunks of at most
 * chunk_cw codewords (0 = automatic, at most 8192): a reader thread reads
 * the next chunk into pinned host memory while earlier chunks are copied
 * and decoded on the host pipeline's two lanes (the first call on a device
 * pins 768 MB of staging and keeps it).  Returns SG_ERR_NONFINITE after
 * decoding the rest if a cube held a non-finite LLR. */
sg_status sg_decode_file(const char* in_path, const char* out_path, const sg_params* p,
                         size_t chunk_cw, sg_run_summary* summary);

/* Totals of a device decode, with the comparator's bit and block errors
 * (SOGRAND_C/comparator.c:31-60) when reference info bits are given. */
typedef struct {
    uint64_t blocks;          /* codewords decoded */
    uint64_t converged;       /* codewords whose early termination fired */
    uint64_t nonfinite;       /* codewords rejected for non-finite LLRs */
    uint64_t total_ng;        /* sum of per-codeword NG */
    uint64_t total_ng_p;      /* sum of per-codeword NG_p */
    uint64_t bits_compared;   /* 512 per codeword when ref_info is given */
    uint64_t bit_errors;      /* decoded info bits differing from ref_info */
    uint64_t block_errors;    /* codewords with at least one bit error */
    double total_iterations;  /* sum of per-codeword iterations (exact) */
    uint64_t timeouts;        /* codewords not decoded because a bounded
                                 device wait gave up (converged = -2) */
    uint32_t device_error;    /* the library's device error flags when the
                                 summary was formed: bit 0 a bulk-copy wait
                                 gave up, bit 1 that copy never completed.
                                 The allocation-free entry point reports its
                                 own call's flags; the regular one reports the
                                 device's flags since the last sg_check_device */
    uint32_t reserved;
} sg_decode_summary;

/* Decode and reduce on the device: bits (nullable: not returned) and one
 * sg_decode_summary at d_summary (device memory, overwritten).  d_ref_info
 * (nullable): the transmitted info bits, 64 packed bytes per codeword, for
 * the bit and block error counts.  Per-codeword statistics are held in
 * stream-ordered scratch (cudaMallocAsync) for the duration of the call. */
sg_status sg_decode_summary_device(const double* d_llr, size_t n_cw, const sg_params* p,
                                   const uint8_t* d_ref_info, uint8_t* d_bits,
                                   sg_decode_summary* d_summary, void* stream);

/* ---- allocation-free variant of sg_decode_summary_device.
 *
 * For callers that must not allocate device memory at all: code that runs
 * while another component owns the device allocator (a framework's caching
 * pool, a real-time process that forbids allocation after start-up), or
 * code whose every device buffer is budgeted up front.  The regular entry
 * point takes stream-ordered scratch per call and its first call on a device
 * allocates the 15 MB error-pattern order table; this one uses only memory
 * that the library declares statically:
 *   - scratch for at most SG_NOALLOC_MAX_CW codewords (statistics and bits,
 *     1.5 MB in all), held by every GPU that loads the library until exit;
 *   - its own copy of the pattern-order table (15 MB, also static), built on
 *     the device by a kernel during the first call on each device.
 * That first call also resolves the device addresses of these arrays and
 * sets up the device; make it before any stream capture.  n_cw above
 * SG_NOALLOC_MAX_CW is rejected with SG_ERR_ARG.  All calls share the one
 * scratch array: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller.  Results equal those
 * of sg_decode_summary_device.  This entry point has no counterpart in the
 * reference, which is a single-process file pipeline. */
#define SG_NOALLOC_MAX_CW 16384
sg_status sg_decode_summary_device_noalloc(const double* d_llr, size_t n_cw, const sg_params* p,
                                           const uint8_t* d_ref_info, uint8_t* d_bits,
                                           sg_decode_summary* d_summary, void* stream);

/* Wilson score interval for k successes in n trials at standard-normal
 * quantile z (1.959963984540054 for 95%): *lo <= k/n <= *hi. */
sg_status sg_wilson_interval(uint64_t k, uint64_t n, double z, double* lo, double* hi);

/* ---- synthetic source, encoder and channel (pipeline stages before the
 * decoder: generate_bin.c, cubic_encoder.c, channel_sim.c).  The reference
 * seeds with time(NULL) and rand(); these are seeded and counter-based, so
 * codeword c of a stream is the same on host and device and independent of
 * batching.  Noise is Gaussian by the Marsaglia polar method; LLR = 2y/s^2
 * with s the noise deviation of channel_sim.c:34-39 (code dimension 3). */

/* Noise deviation for Eb/N0 in dB, as channel_sim.c:34-39 computes it. */
double sg_channel_sigma(double ebn0_db);

/* Info bits of codewords [cw0, cw0+n_cw) of stream `seed`: 64 packed bytes
 * each, the layout of generate_bin/comparator files. */
sg_status sg_gen_info_host(uint64_t seed, uint64_t cw0, size_t n_cw, uint8_t* info);

/* Systematic (16,8)^3 encoding of packed info blocks (cubic_encoder.c:
 * 23-100): 64 bytes in, 4096 bytes of 0/1 code bits out per codeword. */
sg_status sg_encode_host(const uint8_t* info, size_t n_cw, uint8_t* code_bits);

/* Full synthetic channel output for codewords [cw0, cw0+n_cw): info bits
 * (nullable) and float64 LLR cubes.  sigma > 0 fixes the noise deviation;
 * sigma <= 0 draws each codeword's Eb/N0 uniformly from
 * [ebn0_lo_db, ebn0_hi_db] with the decoder's own exp.  The device form
 * writes the same values on the device (asynchronously on `stream`); its
 * llr must be 8-byte aligned (16-byte aligned output is stored faster). */
sg_status sg_gen_llr_host(uint64_t seed, uint64_t cw0, size_t n_cw, double sigma,
                          double ebn0_lo_db, double ebn0_hi_db, uint8_t* info, double* llr);
sg_status sg_gen_llr_device(uint64_t seed, uint64_t cw0, size_t n_cw, double sigma,
                            double ebn0_lo_db, double ebn0_hi_db, uint8_t* d_info,
                            double* d_llr, void* stream);

/* ---- differentiation.  The soft output is piecewise smooth in the LLRs
 * and the extrinsic weights: sorts, tested patterns, codeword lists, stops,
 * early terminations and phase counts are held fixed as the branch of the
 * forward pass.  sg_forward_device is sg_decode_device that also writes the
 * L_E cube entering every phase, d_ckpt[n_cw][3*Imax][4096] (float64);
 * sg_backward_device re-runs every line decode from those checkpoints in
 * reverse phase order and returns, per codeword, the loss
 *   sum_i softplus(s_i L_APP_i),  s_i = +1 for transmitted bit 1, -1 for 0
 * (loss_mode 0: BCE of the final APP, over all 4096 code bits; loss_mode 1:
 * the same summed over the APP of every phase run), its gradient with
 * respect to the per-phase weights alpha (d_grad_alpha[n_cw][3*Imax]) and,
 * optionally, to the channel LLRs (d_grad_llr[n_cw][4096]).  Requires
 * Tmax >= 65536.  d_code_bits: [n_cw][4096] bytes 0/1 in cube order.
 * Both use the table-driven exp/log (math mode 0) whatever the mode set. */
sg_status sg_forward_device(const double* d_llr, size_t n_cw, const sg_params* p, uint8_t* d_bits,
                            double* d_lapp, sg_cw_stats* d_stats, double* d_ckpt, void* stream);
sg_status sg_backward_device(const double* d_llr, size_t n_cw, const sg_params* p,
                             const sg_cw_stats* d_stats, const double* d_ckpt,
                             const uint8_t* d_code_bits, int32_t loss_mode, double* d_loss,
                             double* d_grad_alpha, double* d_grad_llr, void* stream);

/* ---- batched persistent decoder.  One resident CTA per SM holds several
 * codeword slots; warps take lines from any slot with work, the warp that
 * completes a phase runs early termination and either opens the slot's next
 * phase or retires the codeword and admits the next one from a device work
 * queue.  No CTA-wide barrier, so codewords of very uneven cost (mixed
 * Eb/N0) do not stall each other.  Outputs are bit-identical to
 * sg_decode_device.  A handle owns the work-queue word (device memory
 * allocated by sg_batch_create on the current device) and an optional CUDA
 * graph of one decode. */
typedef struct sg_batch_s* sg_batch;
sg_status sg_batch_create(sg_batch* out);
sg_status sg_batch_destroy(sg_batch b);
/* Enqueue one batched decode on `stream` (capturable; one in flight per handle). */
sg_status sg_batch_decode(sg_batch b, const double* d_llr, size_t n_cw, const sg_params* p,
                          uint8_t* d_bits, double* d_lapp, sg_cw_stats* d_stats, void* stream);
/* Record the same decode (queue reset + kernel) as a CUDA graph held by the
 * handle; sg_batch_replay launches it again on any stream. */
sg_status sg_batch_capture(sg_batch b, const double* d_llr, size_t n_cw, const sg_params* p,
                           uint8_t* d_bits, double* d_lapp, sg_cw_stats* d_stats, void* stream);
sg_status sg_batch_replay(sg_batch b, void* stream);
/* After the decode completed: SG_ERR_TIMEOUT if a bounded wait gave up. */
sg_status sg_batch_check(sg_batch b);
int sg_batch_variant_count(void);
const char* sg_batch_variant_name(int v);
sg_status sg_batch_set_variant(int v);
int sg_batch_get_variant(void);

/* ---- math mode (process-wide; launches after the call).  The reference's
 * guess counts depend on the last bits of its libm's exp and log.
 *   0 (default): the decoder's table-driven exp/log (within 0.51 ulp; Tang's
 *     method): fastest; every result equals the oracle restatement built
 *     with the same routines, and the glibc-linked reference on all but a
 *     few tenths of a percent of codewords (where glibc's own misrounding
 *     moves a discrete decision);
 *   1: correctly rounded exp/log: every result -- bits, statistics and soft
 *     values -- equals the unmodified reference compiled against any
 *     correctly rounded libm; about 1.6x the decode time.
 * Applies to sg_decode_device, sg_decode_host, sg_decode_file,
 * sg_decode_summary_device(_noalloc), sg_batch_* and sg_bitso_*; the
 * differentiable pair sg_forward_device / sg_backward_device always uses
 * mode 0. */
sg_status sg_set_math_mode(int32_t mode);
int32_t sg_get_math_mode(void);

/* ---- kernel configuration (process-wide).  Variants differ in warps per
 * codeword CTA, in where the 32 KB channel cube is held (shared memory,
 * staged by a bulk asynchronous copy, or global memory through L2), in
 * error patterns per lane per step, and in lines per warp (one line on 32
 * lanes, or two lines on 16 lanes each: the "-l2-" variants); all give
 * identical results.
 * sogrand_b200.autotune() measures them.  The selection is kept per math
 * mode: the setters change the current mode's. */
int sg_decoder_variant_count(void);
const char* sg_decoder_variant_name(int v);
sg_status sg_decoder_set_variant(int v);
int sg_decoder_get_variant(void);

/* ---- device-side waits.  Every wait in the library's kernels is bounded.
 * A bulk-copy wait that gives up marks its CTA's remaining codewords
 * converged = -2 and sets the device's error flag; a persistent-decoder warp
 * that finds no work for too long exits and sets its batch's flag
 * (sg_batch_check; the other warps finish the batch).  The limit applies to
 * launches made after the call, process-wide: polls of a bulk-copy wait,
 * idle rounds of a persistent warp.  The default, and the largest value
 * accepted (larger values are clamped), is 2^22.  A limit of 0 makes every
 * wait that is not already complete give up; it exists so that tests can
 * exercise the error paths without a faulty GPU. */
sg_status sg_set_wait_limit(uint64_t limit);
uint64_t sg_get_wait_limit(void);

/* Synchronise `stream`, then read and clear the current device's error
 * flag: SG_ERR_TIMEOUT if a bounded wait of a plain-decoder kernel
 * (sg_decode_device, sg_decode_summary_device, sg_forward_device) gave up
 * since the last check, SG_OK otherwise.  The flag is shared by all
 * streams of the device. */
sg_status sg_check_device(void* stream);

/* ---- diagnostics */

/* Measured ceiling of the per-guess floating-point work on the current
 * device: one path-metric addition, one exp(-PM) and one P_notGuess
 * subtraction per guess, all SMs, no memory traffic; 2*iters guesses per
 * thread.  mode 0: with the table-driven exp (math mode 0); mode 1: with the
 * correctly rounded exp (math mode 1).  Synchronous.  The decoder's
 * guesses/s divided by the figure of its math mode is its fraction of the
 * arithmetic bound. */
sg_status sg_guess_ceiling(unsigned long long iters, int32_t mode, double* guesses_per_second);

/* The order in which a line decode tests error patterns when its
 * reliability shift is IC (the loops of sogrand_main_logic,
 * cubic_decoder_final.c:642-744, with mountain_build :775-789).  Writes up to
 * cap entries: bits 0..15 the pattern over reliability-sorted positions,
 * bit 16 set on the first pattern of each logistic weight.  Entry 0 is the
 * hard decision.  Returns the number of entries (65536 when cap allows). */
size_t sg_pattern_order(int32_t ic, uint32_t* out, size_t cap);

const char* sg_status_string(sg_status s);
const char* sg_last_error(void);    /* thread-local text of the last failure */
const char* sg_version(void);

#ifdef __cplusplus
}
#endif
#endif /* SOGRAND_B200_H */
