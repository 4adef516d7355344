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

#ifdef __cplusplus
}
#endif
#endif
