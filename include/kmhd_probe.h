/*
 * kmhd_probe.h -- measurement support for the benchmark harness (not part of
 * the drop-in transform surface; no counterpart in the reference).
 */
#ifndef KMHD_PROBE_H
#define KMHD_PROBE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Peak FP64 tensor-pipe throughput (mma.sync m8n8k4 f64 chains, no memory
 * traffic) on `device`, in TFLOP/s, measured with CUDA events over ~50 ms. */
int kmhd_probe_fp64_tflops(int device, double *tflops);

/* One tcgen05 kind::i8 MMA, D(128x64, int32) = A(128x32, int8, row-major) *
 * B(64x32, int8, row-major)^T, with the shared-memory descriptor's leading /
 * stride byte offsets given by the caller; host arrays.  Self-test of the
 * tensor-core operand layout used by the split-precision tiers. */
int kmhd_selftest_i8_mma(int lbo, int sbo, const signed char *A, const signed char *B, int *D);

#ifdef __cplusplus
}
#endif
#endif
