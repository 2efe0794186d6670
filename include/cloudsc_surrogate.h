/*
 * cloudsc_surrogate.h -- C ABI of the learned CLOUDSC surrogate's kernels
 * (in libcloudsc_b200.so).  No reference counterpart: OpenIFS has no learned
 * cloud scheme; these entry points serve the surrogate path next to the
 * cloudsc_b200_* drop-in.  All pointers are device pointers; every call is
 * asynchronous on `stream` (a cudaStream_t, NULL = default stream).
 *
 * Activation layout: row-major [rows][C] bf16, LP rows per atmospheric column
 * (level l of a column at row 2 + l, the other rows zero padding).
 */
#ifndef CLOUDSC_SURROGATE_H
#define CLOUDSC_SURROGATE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CS_OK 0
#define CS_E_ARG (-2)
#define CS_E_CUDA (-4)

/* GEMM epilogues */
#define CS_EPI_SILU 0       /* out = SiLU(acc + bias) (+ resid); out_pre = acc + bias          */
#define CS_EPI_LINEAR_F32 1 /* outf = acc + bias (f32)                                          */
#define CS_EPI_BWD 2        /* g = acc (+ resid); gout = g; out = g * SiLU'(zprev)              */

typedef struct cs_gemm_desc {
  const void *a;      /* [rows][k] bf16, 16-byte aligned                         */
  const void *w;      /* [taps][n][k] bf16                                        */
  int32_t rows;       /* rows of a and of the output                             */
  int32_t k;          /* multiple of 64                                           */
  int32_t n;          /* 64 or 128                                                */
  int32_t taps;       /* 1, or 5 (rows shifted by -2..+2: a convolution over levels) */
  int32_t lp, klev;   /* column layout; rows outside levels are written as 0 (lp 0: all rows valid) */
  int32_t epi;        /* CS_EPI_*                                                 */
  const float *bias;  /* [n] or NULL                                              */
  void *out;          /* bf16 [rows][n]                                           */
  void *out_pre;      /* bf16 [rows][n] or NULL                                   */
  const void *resid;  /* bf16 [rows][n] or NULL                                   */
  const void *zprev;  /* bf16 [rows][n] (CS_EPI_BWD)                              */
  void *gout;         /* bf16 [rows][n] or NULL (CS_EPI_BWD)                      */
  float *outf;        /* f32 [rows][n] (CS_EPI_LINEAR_F32)                        */
  uint32_t *err;      /* device word or NULL: bit 0 / 1 set if a pipeline wait timed out */
} cs_gemm_desc;

/* D = sum over taps of A(shifted) x W[tap]^T with the epilogue `epi`
 * (tcgen05, one persistent CTA per SM). */
int cs_conv_gemm(const cs_gemm_desc *g, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CLOUDSC_SURROGATE_H */
