/*
 * epik2_probe.h -- measured integer-pipe and tensor-core peaks of a device (libepik2_probe.so).
 *
 * No reference counterpart.  The roofline of the integer search kernel is the POPC
 * issue rate, which no vendor table gives for this GPU; these probes measure it (and
 * the LOP3 and IADD rates) with independent instruction chains on every SM, timed with
 * CUDA events.  Each probe runs about 10-30 ms.
 */
#ifndef EPIK2_PROBE_H
#define EPIK2_PROBE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Results in instructions per second per device (thread-level operations). */
int epik2_probe_int_peaks(int device, double *popc_per_s, double *lop3_per_s, double *iadd_per_s);

/* Dense int8 tensor-core rate: one CTA per SM issues back-to-back tcgen05.mma kind::i8
 * (M=128, N=256, K=32, shared-memory operands in the search kernel's layout, int32
 * accumulators in tensor memory); result in multiply-accumulates per second.  Waits are
 * bounded; returns -6 if one expired. */
int epik2_probe_tc_i8(int device, double *mac_per_s);

/* Dense block-scaled FP4 tensor-core rate in the search kernel's FP4 shape: back-to-back
 * tcgen05.mma kind::mxf4 (M=128, N=224, K=64, E2M1 operands, UE8M0 scale factors in tensor
 * memory, FP32 accumulators); multiply-accumulates per second.  Same waits and errors. */
int epik2_probe_tc_fp4(int device, double *mac_per_s);

#ifdef __cplusplus
}
#endif
#endif
