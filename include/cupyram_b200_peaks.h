/*
 * cupyram_b200_peaks.h - FMA throughput microbenchmark of the device.
 *
 * No counterpart in the reference: it measures the ALU roofline that the
 * march's FP64 / FP32 arithmetic is compared with (the HBM roofline is the
 * measured copy bandwidth).  Runs on the current device and stream 0.
 */
#ifndef CUPYRAM_B200_PEAKS_H
#define CUPYRAM_B200_PEAKS_H

#ifdef __cplusplus
extern "C" {
#endif

enum cr_peaks_status {
    CR_PEAKS_EINVAL = 1,  /* iters < 1 or a NULL output   */
    CR_PEAKS_ECUDA = 2    /* a CUDA runtime call failed   */
};

/* FMA throughput in TFLOP/s (2 flops per FMA) and the timed launch's
 * duration in ms: fp64 != 0 for FP64 FMA, else FP32; iters FMAs per chain
 * (8 chains per thread, 8 CTAs of 256 threads per SM).  Returns 0 or a
 * cr_peaks_status. */
int cr_peak_fma(int fp64, int iters, double* tflops, double* ms);

#ifdef __cplusplus
}
#endif

#endif
