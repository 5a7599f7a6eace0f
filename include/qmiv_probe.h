/*
  qmiv_probe.h — measurement utilities of the QMIV B200 library (no counterpart in the reference).

  The corresponding-pixel-shift search is bound by the SM's integer/FP32 issue rate, not by HBM or
  tensor cores. These probes measure, on the device they run on, the sustained rate of the simple
  32-bit integer operations (add, min) and of FP32 FMAs, so that the search kernel's roofline is a
  fraction of a measured number; the FP64 probe does the same for the regular-window SSIM kernel.
*/
#ifndef QMIV_PROBE_H
#define QMIV_PROBE_H
#include <stdint.h>
#include "qmiv_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Sustained 32-bit integer add/min throughput in tera-operations per second (each add and each min
   counts as one operation), measured with CUDA events over `iters` iterations per thread. */
QMIV_API qmiv_status qmiv_probe_int32_peak(int32_t device, int32_t iters, double* tops);

/* Sustained FP32 FMA throughput in TFLOP/s (2 flops per FMA). */
QMIV_API qmiv_status qmiv_probe_fp32_peak(int32_t device, int32_t iters, double* tflops);

/* Sustained FP64 multiply and add throughput in tera-operations per second (each separately rounded
   DMUL and DADD counts as one operation), the instruction mix of the SSIM window sums. */
QMIV_API qmiv_status qmiv_probe_fp64_peak(int32_t device, int32_t iters, double* tops);

#ifdef __cplusplus
}
#endif
#endif
