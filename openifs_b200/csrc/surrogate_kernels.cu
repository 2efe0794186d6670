// Data, training and guard kernels of the learned CLOUDSC surrogate (sm_100a).
// The network's GEMMs are in surrogate_gemm.cu; see include/cloudsc_surrogate.h
// for the interfaces.
//
// Column budgets used by the guard (both hold to rounding for CLOUDSC itself;
// the oracle tests check them):
//   water     sum_k dp/g (LOC_Q + LOC_L + LOC_I + LOC_R + LOC_S)
//               = S_l + S_i + S_r + S_s - P_rain - P_snow
//   enthalpy  sum_k dp/g (LOC_T - RALVDCP (LOC_L + LOC_R) - RALSDCP (LOC_I + LOC_S))
//               = RALVDCP (P_rain - S_l - S_r) + RALSDCP (P_snow - S_i - S_s)
// with S the column sums of the convective detrainment sources CLOUDSC applies
// (PLUDELI where PLUDE is detrained, PSNDE on the loop levels, cloudsc.F90:
// 1362-1398) and P the surface precipitation fluxes (PFPLSL, PFPLSN at KLEV+1).
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>
#include "cloudsc_surrogate.h"

namespace sk {

constexpr double ZEPSEC = 1.0e-14;

// 16 floats passed by value (host arrays of the C ABI)
struct F16 {
  float v[16];
};

struct Cols {
  cs_columns c;
  __device__ __forceinline__ size_t o2(int col, int k) const {  // (NPROMA,KLEV) element
    const int ib = col / c.nproma, jl = col - ib * c.nproma;
    return ((size_t)ib * c.klev + k) * c.nproma + jl;
  }
  __device__ __forceinline__ size_t oh(int col, int k) const {  // (NPROMA,KLEV+1)
    const int ib = col / c.nproma, jl = col - ib * c.nproma;
    return ((size_t)ib * (c.klev + 1) + k) * c.nproma + jl;
  }
  __device__ __forceinline__ size_t o3(int col, int m, int n, int k) const {  // (NPROMA,KLEV,n)
    const int ib = col / c.nproma, jl = col - ib * c.nproma;
    return (((size_t)ib * n + m) * c.klev + k) * c.nproma + jl;
  }
  __device__ __forceinline__ size_t o1(int col) const { return (size_t)col; }
};

// The CS_NIN raw input features of (column, level): the 14 fields T, q, p,
// the four condensates, PLUDE (detrained condensate), cloud fraction, the
// convective mass flux PMFU + PMFD and the forcing tendencies of T, q, a and
// l + i; then the other fields CLOUDSC reads: PMFU and PMFD apart, the
// updraught condensate PLU, the detrained liquid + ice PLUDELI and rain +
// snow PSNDE, the layer thickness dp, the first-guess relative humidity over
// the mixed phase and over ice (the scheme's own saturation formulas,
// fcttre.func.h FOEEWM / FOEEICE, at T + dt CML_T and q + dt CML_Q), PLSM, and
// the condensate and precipitation mass above the level (cs_column_sums).
// PVFL and PVFI are left out: in CLOUDSC they enter only the DDH flux
// diagnostics; LDCUM is implied by PLUDE and the mass fluxes.
__device__ __forceinline__ void raw_features(const Cols &C, int col, int k, float f[CS_NIN]) {
  const cs_columns &c = C.c;
  const size_t o = C.o2(col, k);
  f[0] = (float)c.pt[o];
  f[1] = (float)c.pq[o];
  f[2] = (float)c.pap[o];
#pragma unroll
  for (int m = 0; m < 4; ++m) f[3 + m] = (float)c.pclv[C.o3(col, m, 5, k)];
  f[7] = (float)(c.plude_in ? c.plude_in : c.plude)[o];
  f[8] = (float)c.pa[o];
  f[9] = (float)(c.pmfu[o] + c.pmfd[o]);
  f[10] = (float)c.cml_t[o];
  f[11] = (float)c.cml_q[o];
  f[12] = (float)c.cml_a[o];
  f[13] = (float)(c.cml_cld[C.o3(col, 0, 5, k)] + c.cml_cld[C.o3(col, 1, 5, k)]);
  f[14] = (float)c.pmfu[o];
  f[15] = (float)c.pmfd[o];
  f[16] = (float)c.plu[o];
  f[17] = (float)(c.pludeli[C.o3(col, 0, 4, k)] + c.pludeli[C.o3(col, 1, 4, k)]);
  f[18] = (float)(c.psnde[C.o3(col, 0, 2, k)] + c.psnde[C.o3(col, 1, 2, k)]);
  f[19] = (float)(c.paph[C.oh(col, k + 1)] - c.paph[C.oh(col, k)]);
  {
    const double t = c.pt[o] + c.ptsphy * c.cml_t[o], q = c.pq[o] + c.ptsphy * c.cml_q[o], p = c.pap[o];
    const double x = (fmax(c.rtice, fmin(c.rtwat, t)) - c.rtice) / (c.rtwat - c.rtice);
    const double alfa = fmin(1.0, x * x);
    const double el = exp(c.r3les * (t - c.rtt) / (t - c.r4les));
    const double ei = exp(c.r3ies * (t - c.rtt) / (t - c.r4ies));
    const double emix = fmin(c.r2es * (alfa * el + (1.0 - alfa) * ei) / p, 0.5);
    const double eice = fmin(c.r2es * ei / p, 0.5);
    const double qsmix = emix / (1.0 - c.retv * emix), qsice = eice / (1.0 - c.retv * eice);
    f[20] = (float)(q / qsmix);
    f[24] = (float)(q / qsice);
  }
  f[21] = (float)c.plsm[C.o1(col)];
  const float *cs = c.colsum + ((size_t)col * c.klev + k) * 2;
  f[22] = cs[0];
  f[23] = cs[1];
}

__device__ __forceinline__ void norm_features(const cs_norm &nrm, const float f[CS_NIN], __nv_bfloat16 *dst) {
#pragma unroll
  for (int ch = 0; ch < CS_NIN; ++ch) {
    float x = f[ch];
    if (nrm.use_log[ch]) x = __logf(fmaxf(x, 0.0f) + nrm.eps[ch]);
    dst[ch] = __float2bfloat16((x - nrm.mean[ch]) * nrm.inv_std[ch]);
  }
}

// Threads are numbered level-major (row r of every column, then the next
// row) so that a warp reads one level of 32 neighbouring columns.
__global__ void raw_features_kernel(Cols C, float *feat) {
  const int ncol = C.c.nproma * C.c.ngpblks, lp = C.c.lp;
  const long long n = (long long)ncol * lp;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / ncol), col = (int)(t - (long long)r * ncol);
    const int k = r - 2;
    __align__(16) float f[CS_FSTRIDE];
#pragma unroll
    for (int i = 0; i < CS_FSTRIDE; ++i) f[i] = 0.0f;
    if (k >= 0 && k < C.c.klev) raw_features(C, col, k, f);
    float4 *d = (float4 *)(feat + ((size_t)col * lp + r) * CS_FSTRIDE);
#pragma unroll
    for (int i = 0; i < CS_FSTRIDE / 4; ++i) d[i] = ((float4 *)f)[i];
  }
}

// Input preparation in two passes: (1) the normalised features of every
// (column, level) once, bf16 [ncol*lp][32]; (2) the 5-level im2col window of
// every row.
// A CTA takes tiles of 32 consecutive columns x FT_ROWS consecutive rows:
// warp w computes row r0 + w of the 32 columns (a warp reads one level of 32
// neighbouring columns), the rows meet in shared memory, and each warp then
// stores one column's FT_ROWS rows, FT_ROWS x 64 contiguous bytes.
constexpr int FT_ROWS = 8;

__global__ void __launch_bounds__(32 * FT_ROWS) features_kernel(Cols C, cs_norm nrm, __nv_bfloat16 *fb) {
  __shared__ __align__(16) __nv_bfloat16 st[FT_ROWS][32][32];
  const int ncol = C.c.nproma * C.c.ngpblks, lp = C.c.lp, klev = C.c.klev;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int ctiles = (ncol + 31) / 32, rtiles = (lp + FT_ROWS - 1) / FT_ROWS;
  const long long ntiles = (long long)ctiles * rtiles;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r0 = (int)(tile / ctiles) * FT_ROWS, col0 = (int)(tile % ctiles) * 32;
    {
      const int r = r0 + w, col = col0 + lane, k = r - 2;
      __align__(16) __nv_bfloat16 row[32];
#pragma unroll
      for (int i = 0; i < 32; ++i) row[i] = __float2bfloat16(0.0f);
      if (col < ncol && k >= 0 && k < klev) {
        float f[CS_NIN];
        raw_features(C, col, k, f);
        norm_features(nrm, f, row);
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) ((uint4 *)st[w][lane])[i] = ((uint4 *)row)[i];
    }
    __syncthreads();
    // 32 columns x FT_ROWS rows x 4 chunks of 16 bytes; 32 consecutive
    // chunks are one column's FT_ROWS rows
    for (int i = threadIdx.x; i < 32 * FT_ROWS * 4; i += 32 * FT_ROWS) {
      const int c = i / (FT_ROWS * 4), q = i - c * (FT_ROWS * 4), rr = q >> 2, part = q & 3;
      const int col = col0 + c, r = r0 + rr;
      if (col < ncol && r < lp)
        ((uint4 *)(fb + ((size_t)col * lp + r) * 32))[part] = ((const uint4 *)st[rr][c])[part];
    }
    __syncthreads();
  }
}

// Slot e = tap * CS_NIN + ch of row r (level k = r % lp - 2) holds feature ch
// of level k + tap - 2; slots 125..127, padding rows and levels outside the
// column are zero.  A CTA takes IM_ROWS consecutive rows: it stages their
// feature rows and two on either side in shared memory (16-byte loads), then
// assembles each 16-byte chunk of the window there.
constexpr int IM_ROWS = 64;
constexpr int IM_THREADS = 256;  // a multiple of 16: each thread keeps one chunk j of every row it writes

__global__ void __launch_bounds__(IM_THREADS) im2col_kernel(const __nv_bfloat16 *__restrict__ fb, long long rows,
                                                            int lp, int klev, __nv_bfloat16 *x0) {
  __shared__ __align__(16) __nv_bfloat16 st[(IM_ROWS + 4) * 32];
  // this thread's chunk j and, per slot q of it, the tap and the staged offset tap * 32 + ch
  const int j = threadIdx.x & 15;
  int tapq[8], offq[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int e = 8 * j + q, tap = e / CS_NIN;
    tapq[q] = tap;
    offq[q] = tap * 32 + (e - tap * CS_NIN);
  }
  const long long ntiles = (rows + IM_ROWS - 1) / IM_ROWS;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long r0 = tile * IM_ROWS;
    for (int i = threadIdx.x; i < (IM_ROWS + 4) * 4; i += IM_THREADS) {
      const long long rs = r0 - 2 + i / 4;  // staged row i / 4 is feature row rs
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (rs >= 0 && rs < rows) v = __ldg((const uint4 *)(fb + rs * 32) + (i & 3));
      ((uint4 *)st)[i] = v;
    }
    const int rr0 = (int)(r0 % lp);  // row of r0 within its column
    __syncthreads();
    for (int lr = threadIdx.x >> 4; lr < IM_ROWS; lr += IM_THREADS / 16) {
      const long long r = r0 + lr;
      if (r >= rows) break;
      int rr = rr0 + lr;  // row r within its column
      while (rr >= lp) rr -= lp;
      const int k = rr - 2;
      const bool kin = k >= 0 && k < klev;
      __align__(16) __nv_bfloat16 v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int ks = k + tapq[q] - 2;
        // feature row r + tap - 2 is staged row lr + tap
        v[q] = (kin && tapq[q] < 5 && ks >= 0 && ks < klev) ? st[lr * 32 + offq[q]] : __float2bfloat16(0.0f);
      }
      ((uint4 *)(x0 + r * 128))[j] = *(const uint4 *)v;
    }
    __syncthreads();
  }
}

__global__ void column_sums_kernel(Cols C, float *colsum) {
  const int ncol = C.c.nproma * C.c.ngpblks, klev = C.c.klev;
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < ncol; col += gridDim.x * blockDim.x) {
    const cs_columns &c = C.c;
    double all = 0.0, prc = 0.0;
    for (int k = 0; k < klev; ++k) {
      float *d = colsum + ((size_t)col * klev + k) * 2;
      d[0] = (float)all;
      d[1] = (float)prc;
      const double dpg = (c.paph[C.oh(col, k + 1)] - c.paph[C.oh(col, k)]) / 9.80665;
      const double ql = c.pclv[C.o3(col, 0, 5, k)], qi = c.pclv[C.o3(col, 1, 5, k)];
      const double qr = c.pclv[C.o3(col, 2, 5, k)], qs = c.pclv[C.o3(col, 3, 5, k)];
      all += dpg * (fmax(ql, 0.0) + fmax(qi, 0.0) + fmax(qr, 0.0) + fmax(qs, 0.0));
      prc += dpg * (fmax(qr, 0.0) + fmax(qs, 0.0));
    }
  }
}

__global__ void prep_targets_kernel(Cols C, F16 scale, float *tgt) {
  const int ncol = C.c.nproma * C.c.ngpblks, lp = C.c.lp, klev = C.c.klev;
  const long long n = (long long)ncol * lp;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / ncol), col = (int)(t - (long long)r * ncol);
    const int k = r - 2;
    float v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = 0.0f;
    if (k >= 0 && k < klev) {
      const cs_columns &c = C.c;
      const size_t o = C.o2(col, k);
      v[0] = (float)c.loc_t[o];
      v[1] = (float)c.loc_q[o];
      v[2] = (float)c.loc_a[o];
#pragma unroll
      for (int m = 0; m < 4; ++m) v[3 + m] = (float)c.loc_cld[C.o3(col, m, 5, k)];
      v[7] = (float)c.pfplsl[C.oh(col, k + 1)];
      v[8] = (float)c.pfplsn[C.oh(col, k + 1)];
#pragma unroll
      for (int i = 0; i < CS_NOUT; ++i) v[i] = v[i] / scale.v[i];
    }
    float4 *d = (float4 *)(tgt + ((size_t)col * lp + r) * 16);
#pragma unroll
    for (int i = 0; i < 4; ++i) d[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
  }
}

// Training batch: thread per (batch row r, batch column j), level-major.
__global__ void prep_batch_kernel(const float *__restrict__ feat, const float *__restrict__ tgt,
                                  const int *__restrict__ cols, int nb, int lp, int klev, cs_norm nrm,
                                  __nv_bfloat16 *x0, float *tb) {
  const long long n = (long long)nb * lp;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / nb), j = (int)(t - (long long)r * nb);
    const size_t src = (size_t)cols[j] * lp;
    const int k = r - 2;
    __align__(16) __nv_bfloat16 row[128];
#pragma unroll
    for (int i = 0; i < 128; ++i) row[i] = __float2bfloat16(0.0f);
    if (k >= 0 && k < klev) {
#pragma unroll
      for (int tap = 0; tap < 5; ++tap) {
        const int ks = k + tap - 2;
        if (ks < 0 || ks >= klev) continue;
        const float4 *f4 = (const float4 *)(feat + (src + 2 + ks) * CS_FSTRIDE);
        __align__(16) float f[CS_FSTRIDE];
#pragma unroll
        for (int q = 0; q < CS_FSTRIDE / 4; ++q) ((float4 *)f)[q] = f4[q];
        norm_features(nrm, f, row + tap * CS_NIN);
      }
    }
    uint4 *d = (uint4 *)(x0 + ((size_t)j * lp + r) * 128);
#pragma unroll
    for (int i = 0; i < 16; ++i) d[i] = ((uint4 *)row)[i];
    const float4 *ts = (const float4 *)(tgt + (src + r) * 16);
    float4 *td = (float4 *)(tb + ((size_t)j * lp + r) * 16);
#pragma unroll
    for (int i = 0; i < 4; ++i) td[i] = ts[i];
  }
}

// ---------------------------------------------------------------- loss
__global__ void loss_kernel(const float *__restrict__ y, const float *__restrict__ tg, int rows, int lp, int klev,
                            F16 w, int nheads, float inv_count, __nv_bfloat16 *dy, double *loss_sum) {
  double acc = 0.0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    const int pos = r % lp;
    const bool valid = pos >= 2 && pos < 2 + klev;
    __align__(16) __nv_bfloat16 g[64];
#pragma unroll
    for (int i = 0; i < 64; ++i) g[i] = __float2bfloat16(0.0f);
    if (valid) {
      for (int h = 0; h < nheads; ++h) {
#pragma unroll
        for (int i = 0; i < CS_NOUT; ++i) {
          const float d = y[(size_t)r * 64 + 32 * h + i] - tg[(size_t)r * 16 + i];
          acc += (double)(w.v[i] * d * d * inv_count);
          g[32 * h + i] = __float2bfloat16(2.0f * w.v[i] * d * inv_count);
        }
      }
    }
    uint4 *dd = (uint4 *)(dy + (size_t)r * 64);
#pragma unroll
    for (int i = 0; i < 8; ++i) dd[i] = ((uint4 *)g)[i];
  }
  // block reduction of the loss
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss_sum, red[0]);
}

// ---------------------------------------------------------------- gradients
// The weight gradients run on the tensor cores (cs_wgrad_tc, surrogate_gemm.cu);
// the bias gradient is a column sum of dz over chunks of rows.
constexpr int BG_CHUNK = 128;
__global__ void bgrad_kernel(const __nv_bfloat16 *__restrict__ dz, int rows, int n, float *db) {
  const int r0 = blockIdx.x * BG_CHUNK, r1 = min(rows, r0 + BG_CHUNK);
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    float s[4] = {0.0f, 0.0f, 0.0f, 0.0f};  // four independent sums: the loads overlap
    int r = r0;
    for (; r + 4 <= r1; r += 4) {
#pragma unroll
      for (int q = 0; q < 4; ++q) s[q] += __bfloat162float(dz[(size_t)(r + q) * n + j]);
    }
    for (; r < r1; ++r) s[0] += __bfloat162float(dz[(size_t)r * n + j]);
    atomicAdd(&db[j], (s[0] + s[1]) + (s[2] + s[3]));
  }
}

// ---------------------------------------------------------------- AdamW
__global__ void adamw_kernel(float *p, float *g, float *m, float *v, int taps, int n, int k, cs_adam hp,
                             __nv_bfloat16 *w, __nv_bfloat16 *wt) {
  const long long cnt = (long long)taps * n * k;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cnt; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = hp.beta1 * m[i] + (1.0f - hp.beta1) * gi;
    const float vi = hp.beta2 * v[i] + (1.0f - hp.beta2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    g[i] = 0.0f;
    float pi = p[i];
    pi -= hp.lr * ((mi / hp.bc1) / (sqrtf(vi / hp.bc2) + hp.eps) + hp.weight_decay * pi);
    p[i] = pi;
    if (w) w[i] = __float2bfloat16(pi);
    if (wt) {
      const int t = (int)(i / ((long long)n * k));
      const int rem = (int)(i - (long long)t * n * k);
      const int nn = rem / k, kk = rem - nn * k;
      wt[((size_t)(taps - 1 - t) * k + kk) * n + nn] = __float2bfloat16(pi);
    }
  }
}

// ---------------------------------------------------------------- guard
// One thread per column.  Pass 1 over the levels: de-normalise, refill
// condensates the step would drive negative (from vapour, with the latent
// heat), write the outputs, accumulate the budgets and the guard quantities.
// Pass 2: the column-constant LOC_Q and LOC_T shifts that close the water and
// enthalpy budgets with the predicted surface precipitation, and the enthalpy
// fluxes.
// 64 registers (8 CTAs of 128 per SM) with a small spill, against 96
// registers and 5 CTAs per SM uncapped.
__global__ void __launch_bounds__(128, 8) post_kernel(Cols C, const float *__restrict__ y, int nheads, cs_guard gd,
                                                     int *nflagged, int *flagged, float4 *diag) {
  const int ys = 64;
  const int ncol = C.c.nproma * C.c.ngpblks, lp = C.c.lp, klev = C.c.klev;
  const int k0 = gd.ncldtop - 1;  // first level of CLOUDSC's level loop
  const double dt = gd.ptsphy, rg = gd.rg;
  const double ral[4] = {gd.ralvdcp, gd.ralsdcp, gd.ralvdcp, gd.ralsdcp};  // l, i, r, s
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < ncol; col += gridDim.x * blockDim.x) {
    const cs_columns &c = C.c;
    double w_lhs = 0.0, w_abs = 0.0, e_lhs = 0.0, e_abs = 0.0;
    double s_l = 0.0, s_i = 0.0, s_r = 0.0, s_s = 0.0, mass = 0.0, spread2 = 0.0;
    double refill = 0.0, cond = 0.0;
    int spread_n = 0;
    const bool ldcum = c.ldcum[C.o1(col)] != 0;
    double pr = 0.0, ps = 0.0;
    for (int k = 0; k < klev; ++k) {
      const size_t r = (size_t)col * lp + 2 + k;
      // channels 0..11 of each head as three 16-byte loads (rows are 256 bytes)
      __align__(16) float ya[12], yb[12];
      const float4 *yr = (const float4 *)(y + r * ys);
#pragma unroll
      for (int q = 0; q < 3; ++q) ((float4 *)ya)[q] = __ldg(yr + q);
      if (nheads == 2) {
#pragma unroll
        for (int q = 0; q < 3; ++q) ((float4 *)yb)[q] = __ldg(yr + 8 + q);
      }
      float yv[CS_NOUT];
#pragma unroll
      for (int i = 0; i < CS_NOUT; ++i) {
        float a = ya[i];
        if (nheads == 2) {
          const float b = yb[i];
          if (i < 7) {
            spread2 += (double)(a - b) * (double)(a - b);
            ++spread_n;
          }
          a = 0.5f * (a + b);
        }
        yv[i] = a * gd.out_scale[i];
      }
      const size_t o = C.o2(col, k);
      const double dp = c.paph[C.oh(col, k + 1)] - c.paph[C.oh(col, k)];
      const double dpg = dp / rg;
      double lt = yv[0], lq = yv[1];
      const double la = yv[2];
      double lc[4] = {yv[3], yv[4], yv[5], yv[6]};
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const double q0 = c.pclv[C.o3(col, m, 5, k)] + dt * c.cml_cld[C.o3(col, m, 5, k)];
        cond += dpg * fmax(q0, 0.0);
        const double qn = q0 + dt * lc[m];
        if (qn < 0.0) {  // refill from vapour (cloudsc.F90:3779-3809 does the same for l, i)
          const double d = -qn / dt;
          lc[m] += d;
          lq -= d;
          lt += ral[m] * d;
          refill += dpg * d * dt;
        }
      }
      c.loc_a[o] = la;
#pragma unroll
      for (int m = 0; m < 4; ++m) c.loc_cld[C.o3(col, m, 5, k)] = lc[m];
      c.loc_q[o] = lq;
      c.loc_t[o] = lt;
      if (k + 1 < klev) {
        c.pfplsl[C.oh(col, k + 1)] = fmax((double)yv[7], 0.0);
        c.pfplsn[C.oh(col, k + 1)] = fmax((double)yv[8], 0.0);
      } else {
        pr = fmax((double)yv[7], 0.0);
        ps = fmax((double)yv[8], 0.0);
      }
      // convective detrainment exactly as CLOUDSC applies it (cloudsc.F90:1362-1398)
      if (k >= k0 && k + 1 < klev) {
        const double zdtgdp = dt * (rg / dp);  // ZDTGDP = PTSPHY * ZGDP, ZGDP = RG / ZDP
        const double pl = (c.plude_in ? c.plude_in : c.plude)[o] * zdtgdp;
        const double plu1 = c.plu[C.o2(col, k + 1)];
        double plude_out = 0.0;
        if (ldcum && pl > ZEPSEC && plu1 > ZEPSEC) {
          plude_out = pl;
          s_l += c.pludeli[C.o3(col, 0, 4, k)];
          s_i += c.pludeli[C.o3(col, 1, 4, k)];
        }
        s_r += c.psnde[C.o3(col, 0, 2, k)];
        s_s += c.psnde[C.o3(col, 1, 2, k)];
        c.plude[o] = plude_out;
      }
      w_lhs += dpg * (lq + lc[0] + lc[1] + lc[2] + lc[3]);
      w_abs += fabs(dpg * lq) + fabs(dpg * (lc[0] + lc[1] + lc[2] + lc[3]));
      e_lhs += dpg * (lt - gd.ralvdcp * (lc[0] + lc[2]) - gd.ralsdcp * (lc[1] + lc[3]));
      e_abs += fabs(dpg * lt);
      mass += dpg;
    }
    // water: shift LOC_Q so that sum dp/g (q + condensates) = S - P
    const double w_rhs = (s_l + s_i + s_r + s_s) - (pr + ps);
    const double w_res = w_lhs - w_rhs;
    const double w_raw = fabs(w_res) / (w_abs + fabs(w_rhs) + 1e-30);
    const double qshift = w_res / mass;
    // enthalpy: shift LOC_T (the LOC_Q shift does not enter this budget)
    const double e_rhs = gd.ralvdcp * (pr - s_l - s_r) + gd.ralsdcp * (ps - s_i - s_s);
    const double e_res = e_lhs - e_rhs;
    const double e_raw = fabs(e_res) / (e_abs + fabs(e_rhs) + 1e-30);
    const double tshift = e_res / mass;
    for (int k = 0; k < klev; ++k) {
      const size_t o = C.o2(col, k);
      c.loc_q[o] = c.loc_q[o] - qshift;
      c.loc_t[o] = c.loc_t[o] - tshift;
    }
    c.pfplsl[C.oh(col, klev)] = pr;
    c.pfplsn[C.oh(col, klev)] = ps;
    c.pfplsl[C.oh(col, 0)] = 0.0;
    c.pfplsn[C.oh(col, 0)] = 0.0;
    for (int k = 0; k <= klev; ++k) {
      const size_t oo = C.oh(col, k);
      c.pfhpsl[oo] = -gd.rlvtt * c.pfplsl[oo];
      c.pfhpsn[oo] = -gd.rlstt * c.pfplsn[oo];
    }
    const double spread = spread_n ? sqrt(spread2 / spread_n) : 0.0;
    const double refill_rel = refill / (cond + 1e-12);
    const bool flag = refill_rel > gd.neg_tol || w_raw > gd.closure_tol || e_raw > gd.closure_tol ||
                      (nheads == 2 && spread > gd.spread_tol);
    if (diag) diag[col] = make_float4((float)w_raw, (float)e_raw, (float)spread, (float)refill_rel);
    if (flag) {
      const int slot = atomicAdd(nflagged, 1);
      if (slot < gd.capacity) flagged[slot] = col;
    }
  }
}

// ---------------------------------------------------------------- column moves
__global__ void move_columns_kernel(const cs_colarray *__restrict__ arrays, int narr, int nps, int npd,
                                    const int *__restrict__ idx, const int *__restrict__ count, int cap,
                                    int dir) {
  const int n = min(*count, cap);
  const int ncols = dir == 0 ? cap : n;
  // blockIdx.y: array; threads over (row, slot j) with j fastest
  const int a = blockIdx.y;
  if (a >= narr) return;
  const cs_colarray A = arrays[a];
  const long long total = (long long)A.rows * ncols;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(t / ncols), j = (int)(t - (long long)row * ncols);
    int cs, cd;
    if (dir == 0) {
      cs = n > 0 ? idx[min(j, n - 1)] : 0;
      cd = j;
    } else {
      cs = j;
      cd = idx[j];
    }
    const int ibs = cs / nps, jls = cs - ibs * nps, ibd = cd / npd, jld = cd - ibd * npd;
    const size_t os = ((size_t)ibs * A.rows + row) * nps + jls;
    const size_t od = ((size_t)ibd * A.rows + row) * npd + jld;
    if (A.esize == 8)
      ((double *)A.dst)[od] = ((const double *)A.src)[os];
    else
      ((int32_t *)A.dst)[od] = ((const int32_t *)A.src)[os];
  }
}

int grid_1d(long long n, int threads) {
  long long g = (n + threads - 1) / threads;
  const long long cap = 148LL * 32;
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

bool cols_ok(const cs_columns *c) {
  return c && c->nproma > 0 && c->klev > 0 && c->ngpblks > 0 && c->lp >= c->klev + 4;
}

}  // namespace sk

extern "C" {

int cs_raw_features(const cs_columns *c, float *feat, void *stream) {
  using namespace sk;
  if (!cols_ok(c) || !feat || !c->colsum) return CS_E_ARG;
  Cols C{*c};
  const long long n = (long long)c->nproma * c->ngpblks * c->lp;
  raw_features_kernel<<<grid_1d(n, 256), 256, 0, (cudaStream_t)stream>>>(C, feat);
  return cudaGetLastError() == cudaSuccess ? CS_OK : CS_E_CUDA;
}

int cs_column_sums(const cs_columns *c, float *colsum, void *stream) {
  using namespace sk;
  if (!cols_ok(c) || !colsum) return CS_E_ARG;
  Cols C{*c};
  column_sums_kernel<<<grid_1d((long long)c->nproma * c->ngpblks, 128), 128, 0, (cudaStream_t)stream>>>(C, colsum);
  return cudaGetLastError() == cudaSuccess ? CS_OK : CS_E_CUDA;
}

int cs_prep_inputs(const cs_columns *c, const cs_norm *nrm, void *fbuf, void *x0, void *stream) {
  using namespace sk;
  if (!cols_ok(c) || !nrm || !x0 || !fbuf || !c->colsum) return CS_E_ARG;
  Cols C{*c};
  const long long n = (long long)c->nproma * c->ngpblks * c->lp;
  const long long ftiles = (long long)((c->nproma * c->ngpblks + 31) / 32) * ((c->lp + FT_ROWS - 1) / FT_ROWS);
  const int ft_grid = (int)(ftiles < 148LL * 8 ? ftiles : 148LL * 8);
  features_kernel<<<ft_grid, 32 * FT_ROWS, 0, (cudaStream_t)stream>>>(C, *nrm, (__nv_bfloat16 *)fbuf);
  const long long tiles = (n + IM_ROWS - 1) / IM_ROWS;
  const int im_grid = (int)(tiles < 148LL * 8 ? tiles : 148LL * 8);
  im2col_kernel<<<im_grid, IM_THREADS, 0, (cudaStream_t)stream>>>((const __nv_bfloat16 *)fbuf, n, c->lp, c->klev,
                                                           (__nv_bfloat16 *)x0);
  return cudaGetLastError() == cudaSuccess ? CS_OK : CS_E_CUDA;
}

int cs_prep_targets(const cs_columns *c, const float *scale16, float *t, void *stream) {
  using namespace sk;
  if (!cols_ok(c) || !scale16 || !t) return CS_E_ARG;
  Cols C{*c};
  const long long n = (long long)c->nproma * c->ngpblks * c->lp;
  F16 sc;
  memcpy(sc.v, scale16, sizeof(sc.v));
  prep_targets_kernel<<<grid_1d(n, 256), 256, 0, (cudaStream_t)stream>>>(C, sc, t);
  return cudaGetLastError() == cudaSuccess ? CS_OK : CS_E_CUDA;
}

int cs_prep_batch(const float *feat, const float *tgt, const int32_t *cols, int32_t nb, int32_t lp, int32_t klev,
                  const cs_norm *nrm, void *x0, float *tb, void *stream) {
  using namespace sk;
  if (!feat || !tgt || !cols || nb <= 0 || lp < klev + 4 || !nrm || !x0 || !tb) return CS_E_ARG;
  const long long n = (long long)nb * lp;
  prep_batch_kernel<<<grid_1d(n, 128), 128, 0, (cudaStream_t)stream>>>(feat, tgt, cols, nb, lp, klev, *nrm,
                                                                       (__nv_bfloat16 *)x0, tb);
  return cudaGetLastError() == cudaSuccess ? CS_OK : CS_E_CUDA;
}

int cs_loss(const float *y, const float *t, int32_t rows, int32_t lp, int32_t klev, const float *w16,
            int32_t nheads, void *dy, double *loss_sum, void *stream) {
  using namespace sk;
  if (!y || !t || !w16 || !dy || !loss_sum || rows <= 0 || lp < klev + 4 || nheads < 1 || nheads > 2)
    return CS_E_ARG;
  const long long nvalid = (long long)(rows / lp) * klev * CS_NOUT;
  const float inv = 1.0f / (float)(nvalid > 0 ? nvalid : 1);
  F16 w;
  memcpy(w.v, w16, sizeof(w.v));
  loss_kernel<<<grid_1d(rows, 256), 256, 0, (cudaStream_t)stream>>>(y, t, rows, lp, klev, w, nheads, inv,
                                                                     (__nv_bfloat16 *)dy, loss_sum);
  return cudaGetLastError() == cudaSuccess ? CS_OK : CS_E_CUDA;
}

int cs_wgrad(const void *dz, const void *x, int32_t rows, int32_t n, int32_t k, int32_t taps, float *dw,
             float *db, void *stream) {
  using namespace sk;
  if (!dz || !x || !dw || rows <= 0 || (n != 64 && n != 128) || (k != 64 && k != 128) || (taps != 1 && taps != 5))
    return CS_E_ARG;
  const int rc = cs_wgrad_tc(dz, x, rows, n, k, taps, dw, nullptr, stream);
  if (rc != CS_OK) return rc;
  if (db) bgrad_kernel<<<(rows + BG_CHUNK - 1) / BG_CHUNK, 128, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16 *)dz, rows, n, db);
  return cudaGetLastError() == cudaSuccess ? CS_OK : CS_E_CUDA;
}

int cs_adamw(float *p, float *g, float *m, float *v, int32_t taps, int32_t n, int32_t k, const cs_adam *hp, void *w,
             void *wt, void *stream) {
  using namespace sk;
  if (!p || !g || !m || !v || !hp || taps <= 0 || n <= 0 || k <= 0) return CS_E_ARG;
  const long long cnt = (long long)taps * n * k;
  adamw_kernel<<<grid_1d(cnt, 256), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, taps, n, k, *hp,
                                                                     (__nv_bfloat16 *)w, (__nv_bfloat16 *)wt);
  return cudaGetLastError() == cudaSuccess ? CS_OK : CS_E_CUDA;
}

int cs_post(const cs_columns *c, const float *y, int32_t nheads, const cs_guard *g, int32_t *nflagged,
            int32_t *flagged, float *diag, void *stream) {
  using namespace sk;
  if (!cols_ok(c) || !y || (uintptr_t)y % 16 || !g || !nflagged || (g->capacity > 0 && !flagged) || nheads < 1 ||
      nheads > 2)
    return CS_E_ARG;
  Cols C{*c};
  const int ncol = c->nproma * c->ngpblks;
  post_kernel<<<grid_1d(ncol, 128), 128, 0, (cudaStream_t)stream>>>(C, y, nheads, *g, nflagged, flagged,
                                                                      (float4 *)diag);
  return cudaGetLastError() == cudaSuccess ? CS_OK : CS_E_CUDA;
}

int cs_move_columns(const cs_colarray *arrays, int32_t narr, int32_t nproma_src, int32_t nproma_dst,
                    const int32_t *idx, const int32_t *count, int32_t cap, int32_t dir, void *stream) {
  using namespace sk;
  if (!arrays || narr <= 0 || narr > 65535 || nproma_src <= 0 || nproma_dst <= 0 || !idx || !count || cap <= 0 ||
      (dir != 0 && dir != 1))
    return CS_E_ARG;
  dim3 grid(grid_1d((long long)cap * 140, 256) / 4 + 1, narr);
  move_columns_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(arrays, narr, nproma_src, nproma_dst, idx, count, cap,
                                                              dir);
  return cudaGetLastError() == cudaSuccess ? CS_OK : CS_E_CUDA;
}

}  // extern "C"
