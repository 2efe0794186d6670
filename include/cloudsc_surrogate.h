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

/* The network's MLP layer and output head in one kernel (inference):
 * h = SiLU(a w1^T + b1) kept on chip as bf16, y = h w2^T + b2 (f32); rows
 * outside the levels of the lp/klev layout written as zero, as
 * cs_conv_gemm's CS_EPI_SILU then CS_EPI_LINEAR_F32 would (same bits).
 * a [rows][k] and w1 [k][k], w2 [64][k] bf16 (16-byte aligned), y f32
 * [rows][64] (32-byte aligned); k 64 or 128; b1, b2 or NULL; err as in
 * cs_gemm_desc. */
int cs_mlp_head(const void *a, const void *w1, const float *b1, const void *w2, const float *b2, int32_t rows,
                int32_t k, int32_t lp, int32_t klev, float *y, uint32_t *err, void *stream);

/* Which kernel cs_conv_gemm runs: 0 (default) the warp-specialised one
 * (weights resident in shared memory, one halo tile per K block for the 5
 * taps, double-buffered TMEM accumulator), 1 the simple single-thread
 * pipeline (kept as a cross-check). */
int cs_set_gemm_impl(int32_t impl);

/* ------------------------------------------------------------------------
 * Column data in CLOUDSC's batched storage (NPROMA, dims, NGPBLKS), device
 * pointers, double precision (LDCUM int32).  Column c = ib * NPROMA + jl.
 * The surrogate reads the inputs and writes LOC_T, LOC_Q, LOC_A, LOC_CLD(1:4),
 * PLUDE, PFPLSL/PFPLSN and PFHPSL/PFHPSN; it predicts no DDH flux.
 */
typedef struct cs_columns {
  const double *pt, *pq, *pap, *paph, *pclv, *pa, *pmfu, *pmfd;
  const double *cml_t, *cml_q, *cml_a, *cml_cld, *plu, *pludeli, *psnde;
  const int32_t *ldcum;
  double *plude; /* INOUT: read as the input detrainment, written as CLOUDSC does */
  const double *plude_in; /* if not NULL, the input detrainment is read here instead, so
                           * that repeated calls on one batch see the same input */
  const double *plsm;
  const float *colsum; /* [ncol][klev][2] from cs_column_sums: condensate and
                        * precipitation mass above each level (kg m-2) */
  double *loc_t, *loc_q, *loc_a, *loc_cld, *pfplsl, *pfplsn, *pfhpsl, *pfhpsn;
  /* saturation constants (cloudsc_params names) for the humidity features */
  double r2es, r3les, r3ies, r4les, r4ies, rtt, rtice, rtwat, retv, ptsphy;
  int32_t nproma, klev, ngpblks, lp; /* lp: padded rows per column (>= klev + 4) */
} cs_columns;

#define CS_NIN 25   /* input channels per level (also the slot stride of one tap) */
#define CS_FSTRIDE 28 /* floats per row of the raw-feature buffer (16-byte rows) */
#define CS_NOUT 9   /* output channels per level */

/* Input feature transform: f = use_log ? log(x + eps) : x; (f - mean) * inv_std */
typedef struct cs_norm {
  float mean[32], inv_std[32], eps[32];
  int32_t use_log[32];
} cs_norm;

/* Column-integrated inputs the 5-level convolutions cannot reach: for every
 * level, sum over the levels above of dp/g (l + i + r + s) and of dp/g (r + s)
 * of the input condensates (PCLV); writes colsum (f32 [ncol][klev][2]). */
int cs_column_sums(const cs_columns *c, float *colsum, void *stream);

/* Network input: x0[c*lp + 2 + l][tap*CS_NIN + ch] = feature ch of level
 * l+tap-2 (zero outside the column); bf16 [ncol*lp][128].  fbuf: work
 * buffer, bf16 [ncol*lp][32] (the normalised features of every level). */
int cs_prep_inputs(const cs_columns *c, const cs_norm *nrm, void *fbuf, void *x0, void *stream);
/* Raw (untransformed) input features, f32 [ncol*lp][CS_FSTRIDE]. */
int cs_raw_features(const cs_columns *c, float *feat, void *stream);
/* Training targets from CLOUDSC's outputs, divided by scale[ch]: f32
 * [ncol*lp][16] (LOC_T, LOC_Q, LOC_A, LOC_CLD l,i,r,s, PFPLSL, PFPLSN at the
 * half level below the level). */
int cs_prep_targets(const cs_columns *c, const float *scale16, float *t, void *stream);

/* Training batch from stored features: for j < nb, batch column j is data
 * column cols[j] (device int32): x0 (bf16 [nb*lp][128]) as cs_prep_inputs
 * builds it from feat (f32 [*][CS_FSTRIDE], cs_raw_features layout), and tb (f32
 * [nb*lp][16]) copied from tgt (cs_prep_targets layout). */
int cs_prep_batch(const float *feat, const float *tgt, const int32_t *cols, int32_t nb, int32_t lp,
                  int32_t klev, const cs_norm *nrm, void *x0, float *tb, void *stream);

/* MSE loss over valid rows and the first CS_NOUT channels of each of the
 * nheads (1 or 2) output heads; y f32 and dy bf16 are [rows][64] (head h in
 * columns 32h..32h+CS_NOUT-1):
 * dy = 2 w (y - t) / count, loss_sum += sum w (y - t)^2 / count. */
int cs_loss(const float *y, const float *t, int32_t rows, int32_t lp, int32_t klev, const float *w16,
            int32_t nheads, void *dy, double *loss_sum, void *stream);

/* dw[t][n][k] += sum_r dz[r][n] * x[r + t - taps/2][k] (bf16 products, f32
 * accumulation on the tcgen05 tensor cores, cs_wgrad_tc); db[n] += sum_r
 * dz[r][n] when db is not NULL.  n and k are 64 or 128, taps 1 or 5; rows of
 * x outside [0, rows) count as zero. */
int cs_wgrad(const void *dz, const void *x, int32_t rows, int32_t n, int32_t k, int32_t taps, float *dw,
             float *db, void *stream);

/* The weight-gradient GEMM alone: dw[t][n][k] += sum_r dz[r][n] *
 * x[r + t - taps/2][k] on the tensor cores.  dz [rows][n] and x [rows][k] bf16
 * row-major, dw f32 [taps][n][k], all 16-byte aligned; n, k in {64, 128}.
 * err (or NULL): bit 1 or 2 set when a bounded wait in the kernel ran out. */
int cs_wgrad_tc(const void *dz, const void *x, int32_t rows, int32_t n, int32_t k, int32_t taps, float *dw,
                unsigned *err, void *stream);

typedef struct cs_adam {
  float lr, beta1, beta2, eps, weight_decay, bc1, bc2; /* bc = 1 - beta^step */
} cs_adam;
/* AdamW step on f32 master weights p [taps][n][k] (or a bias: taps = 1,
 * k = 1); zeroes g; writes bf16 copies w (same layout) and wt
 * ([taps][k][n], taps reversed: the backward-data operand) when not NULL. */
int cs_adamw(float *p, float *g, float *m, float *v, int32_t taps, int32_t n, int32_t k, const cs_adam *hp,
             void *w, void *wt, void *stream);

/* Guard of the surrogate's output.  The small parameter structs (cs_norm,
 * cs_adam, cs_guard) and the w16 / scale16 arrays of the calls above and
 * below are read from HOST memory at the call; everything else is device
 * memory. */
typedef struct cs_guard {
  float out_scale[16];   /* de-normalisation of the network outputs            */
  double rg, ralvdcp, ralsdcp, rlvtt, rlstt, ptsphy;
  int32_t ncldtop;       /* first level of CLOUDSC's level loop (1-based)      */
  double neg_tol;        /* refilled condensate / column condensate above this: flag */
  double closure_tol;    /* raw water/enthalpy non-closure above this: flag     */
  double spread_tol;     /* RMS head disagreement (normalised) above this: flag */
  int32_t capacity;      /* length of the flagged-column list                   */
} cs_guard;

/* Turn the network output y ([rows][64] f32, head h at column 32h, 16-byte
 * aligned: CS_E_ARG otherwise) into CLOUDSC outputs: mean of the heads,
 * de-normalised; condensates that the step would
 * drive negative are refilled from vapour with their latent heat (as
 * CLOUDSC's own clean-up does, cloudsc.F90:3779-3809); LOC_Q is then shifted
 * by a column constant so that the water budget closes with the predicted
 * surface precipitation, and LOC_T by one so that the enthalpy budget closes;
 * PLUDE and the enthalpy fluxes as CLOUDSC defines them.  Columns failing
 * the guard are appended to flagged[0..capacity) (count in *nflagged, which
 * must start at 0); diag (float4 per column, or NULL) = {raw water
 * non-closure, raw enthalpy non-closure, head spread, refilled condensate
 * relative to the column's condensate}. */
int cs_post(const cs_columns *c, const float *y, int32_t nheads, const cs_guard *g, int32_t *nflagged,
            int32_t *flagged, float *diag, void *stream);

/* One array of column data for cs_move_columns: per-column rows and element
 * size, base pointers in two batched layouts. */
typedef struct cs_colarray {
  const void *src;
  void *dst;
  int32_t rows, esize;
} cs_colarray;
/* gather (dir 0): dst column j <- src column idx[min(j, n-1)] for j < cap,
 *                 n = min(*count, cap) (all from column 0 when n = 0);
 * scatter (dir 1): dst column idx[j] <- src column j for j < n.
 * arrays: device array of narr descriptors. */
int cs_move_columns(const cs_colarray *arrays, int32_t narr, int32_t nproma_src, int32_t nproma_dst,
                    const int32_t *idx, const int32_t *count, int32_t cap, int32_t dir, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CLOUDSC_SURROGATE_H */
