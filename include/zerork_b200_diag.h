/*
 * zerork_b200_diag.h -- diagnostics of the sm_100a library.
 *
 * No counterpart in the reference (Zero-RK reports no hardware peaks); the
 * rate kernels are FP64 SIMT work, so their roofline needs the FP64 pipe's
 * measured throughput next to the HBM bandwidth.
 */
#ifndef ZERORK_B200_DIAG_H
#define ZERORK_B200_DIAG_H

#ifdef __cplusplus
extern "C" {
#endif

/* Measure FP64 FMA throughput (GFLOP/s, 2 flops per FMA) and double
 * precision exp() throughput (G exp/s) on the current device (~0.5 s). */
int zrk_measure_fp64(double *fma_gflops, double *exp_gps);

#ifdef __cplusplus
}
#endif
#endif
