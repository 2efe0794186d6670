// Column-network GEMMs on the tcgen05 tensor cores (sm_100a).
//
// Activations are row-major [rows][C] bf16 with one row per (column, padded
// level): a column occupies LP consecutive rows, level l at row 2 + l, the
// other rows are zero padding.  A 1-D convolution with 5 taps over levels is
// then five GEMMs whose A operands are the same matrix shifted by -2..+2 rows,
// all accumulated into one TMEM tile:
//
//   D[r][n] = sum_t sum_k A[r + t + tap_origin][k] * W[t][n][k]
//
// TMA fetches each (tap, 64-wide K block) of A (128 rows) and of W (N rows)
// into a 4-stage shared-memory ring; rows outside [0, rows) read as zero.
// Thread 0 issues TMA and tcgen05.mma; the four warps then drain TMEM through
// a fused epilogue (bias, SiLU, residual, padding rows forced to zero, bf16 or
// f32 store; or, for the backward pass, residual gradient and SiLU').
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>
#include <mutex>
#include "tc_gemm.cuh"
#include "cloudsc_surrogate.h"

namespace sg {

constexpr int BM = 128;
constexpr int BK = 64;
constexpr int STAGES = 4;
constexpr int A_BYTES = BM * BK * 2;  // 16 KB

struct Args {
  int rows;        // rows of A and D (tiles past it are masked)
  int kb_per_tap;  // K / 64
  int taps;        // 1 or 5
  int tap_origin;  // row offset of tap 0
  int lp, klev;    // column layout: LP rows per column, levels at rows 2..klev+1
  int epi;
  const float *bias;          // [N] or null
  __nv_bfloat16 *out;         // [rows][N]
  __nv_bfloat16 *out_pre;     // [rows][N] pre-activation (forward) or null
  const __nv_bfloat16 *resid; // [rows][N] residual input (forward) / gradient (backward) or null
  const __nv_bfloat16 *zprev; // [rows][N] pre-activation whose SiLU' scales the gradient (backward)
  __nv_bfloat16 *gout;        // [rows][N] gradient before SiLU' (backward) or null
  float *outf;                // [rows][N] f32 output (linear epilogue)
  unsigned *err;              // or null
};

__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = __fdividef(1.0f, 1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}
__device__ __forceinline__ void flag(unsigned *err, unsigned bit) {
  if (err) atomicOr(err, bit);
}

template <int BN, int EPI>
__global__ void __launch_bounds__(128, 1)
    conv_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Args a) {
  constexpr int B_BYTES = BN * BK * 2;
  constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  constexpr uint32_t IDESC = tcg::idesc_bf16_f32(BM, BN);
  constexpr int TMEM_COLS = BN < 32 ? 32 : BN;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *full = (uint64_t *)(smem + STAGES * STAGE_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *done = empty + STAGES;
  uint32_t *tmem_slot = (uint32_t *)(done + 1);
  volatile int *abort_flag = (volatile int *)(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tcg::mbar_init(&full[s], 1);
      tcg::mbar_init(&empty[s], 1);
    }
    tcg::mbar_init(done, 1);
    *abort_flag = 0;
    tcg::mbar_fence_init();
    tcg::tma_prefetch_desc(&tmA);
    tcg::tma_prefetch_desc(&tmB);
  }
  if (warp == 0) {
    tcg::tmem_alloc(tmem_slot, TMEM_COLS);
    tcg::tmem_relinquish();
  }
  tcg::tc_fence_before();
  __syncthreads();
  tcg::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int ntiles = (a.rows + BM - 1) / BM;
  const int nk = a.taps * a.kb_per_tap;
  uint32_t pc = 0, cc = 0;  // produced / consumed stage counters (thread 0)
  uint32_t tile_iter = 0;

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++tile_iter) {
    const int row0 = tile * BM;
    if (tid == 0) {
      bool ok = true;
      auto produce = [&](int k) {
        const int s = pc % STAGES;
        if (pc >= STAGES) ok = ok && tcg::mbar_wait(&empty[s], ((pc / STAGES) - 1) & 1);
        if (!ok) return;
        const int tap = k / a.kb_per_tap, kb = k - tap * a.kb_per_tap;
        uint8_t *sa = smem + s * STAGE_BYTES;
        tcg::mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
        tcg::tma_load_2d(sa, &tmA, &full[s], kb * BK, row0 + a.tap_origin + tap);
        tcg::tma_load_2d(sa + A_BYTES, &tmB, &full[s], kb * BK, tap * BN);
        ++pc;
      };
      const int pre = nk < STAGES - 1 ? nk : STAGES - 1;
      for (int k = 0; k < pre && ok; ++k) produce(k);
      for (int k = 0; k < nk && ok; ++k) {
        const int s = cc % STAGES;
        ok = tcg::mbar_wait(&full[s], (cc / STAGES) & 1);
        if (!ok) break;
        tcg::tc_fence_after();
        const uint32_t sa = tcg::smem_u32(smem + s * STAGE_BYTES);
        const uint64_t da = tcg::sdesc_k_sw128(sa), db = tcg::sdesc_k_sw128(sa + A_BYTES);
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk)  // 16 bf16 = 32 bytes per MMA step
          tcg::mma_bf16(tmem, da + 2 * kk, db + 2 * kk, IDESC, (k > 0 || kk > 0) ? 1u : 0u);
        tcg::mma_commit(&empty[s]);
        ++cc;
        if (k + STAGES - 1 < nk) produce(k + STAGES - 1);
      }
      if (ok) {
        tcg::mma_commit(done);
      } else {
        flag(a.err, 1u);
        *abort_flag = 1;
      }
    }
    __syncthreads();
    if (*abort_flag) break;
    if (!tcg::mbar_wait(done, tile_iter & 1)) {
      flag(a.err, 2u);
      *abort_flag = 1;
    }
    tcg::tc_fence_after();

    // ---------------- epilogue: this thread owns output row `row`
    const int row = row0 + warp * 32 + lane;
    const int pos = a.lp > 0 ? row % a.lp : 2;
    const bool in_range = row < a.rows;
    const bool valid = in_range && (a.lp <= 0 || (pos >= 2 && pos < 2 + a.klev));
    if (!*abort_flag) {
#pragma unroll 1
      for (int c0 = 0; c0 < BN; c0 += 32) {
        float v[32];
        tcg::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
        if (!in_range) continue;
        const size_t o = (size_t)row * BN + c0;
        if (EPI == CS_EPI_SILU) {
          __align__(32) __nv_bfloat16 h[32], z[32];
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            float zz = v[i] + (a.bias ? a.bias[c0 + i] : 0.0f);
            float hh = silu(zz);
            if (a.resid) hh += __bfloat162float(a.resid[o + i]);
            if (!valid) {
              zz = 0.0f;
              hh = 0.0f;
            }
            z[i] = __float2bfloat16(zz);
            h[i] = __float2bfloat16(hh);
          }
          uint4 *dh = (uint4 *)(a.out + o);
#pragma unroll
          for (int i = 0; i < 4; ++i) dh[i] = ((uint4 *)h)[i];
          if (a.out_pre) {
            uint4 *dz = (uint4 *)(a.out_pre + o);
#pragma unroll
            for (int i = 0; i < 4; ++i) dz[i] = ((uint4 *)z)[i];
          }
        } else if (EPI == CS_EPI_LINEAR_F32) {
          float4 *d = (float4 *)(a.outf + o);
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            float4 w;
            w.x = valid ? v[4 * i + 0] + (a.bias ? a.bias[c0 + 4 * i + 0] : 0.0f) : 0.0f;
            w.y = valid ? v[4 * i + 1] + (a.bias ? a.bias[c0 + 4 * i + 1] : 0.0f) : 0.0f;
            w.z = valid ? v[4 * i + 2] + (a.bias ? a.bias[c0 + 4 * i + 2] : 0.0f) : 0.0f;
            w.w = valid ? v[4 * i + 3] + (a.bias ? a.bias[c0 + 4 * i + 3] : 0.0f) : 0.0f;
            d[i] = w;
          }
        } else {  // CS_EPI_BWD: g = acc (+ residual gradient); dz = g * SiLU'(zprev)
          __align__(32) __nv_bfloat16 g[32], dz[32];
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            float gg = v[i];
            if (a.resid) gg += __bfloat162float(a.resid[o + i]);
            float d = gg * dsilu(__bfloat162float(a.zprev[o + i]));
            if (!valid) {
              gg = 0.0f;
              d = 0.0f;
            }
            g[i] = __float2bfloat16(gg);
            dz[i] = __float2bfloat16(d);
          }
          uint4 *dd = (uint4 *)(a.out + o);
#pragma unroll
          for (int i = 0; i < 4; ++i) dd[i] = ((uint4 *)dz)[i];
          if (a.gout) {
            uint4 *dg = (uint4 *)(a.gout + o);
#pragma unroll
            for (int i = 0; i < 4; ++i) dg[i] = ((uint4 *)g)[i];
          }
        }
      }
    }
    tcg::tc_fence_before();
    __syncthreads();
    if (*abort_flag) break;
  }

  // On an abort, let every copy and MMA this CTA issued land before the
  // shared memory and TMEM are released (bounded waits).
  if (tid == 0 && *abort_flag) {
    for (uint32_t q = cc; q < pc; ++q) (void)tcg::mbar_wait(&full[q % STAGES], (q / STAGES) & 1);
    tcg::mma_commit(done);
    (void)tcg::mbar_wait(done, tile_iter & 1);
  }
  __syncthreads();
  if (warp == 0) tcg::tmem_dealloc(tmem, TMEM_COLS);
}

// ------------------------------------------------------------------ epilogue
// 32 accumulator columns c0..c0+31 of output row `row` (fused epilogue).
// Each thread owns 64 (bf16) or 128 (f32) contiguous bytes of one row and
// moves them with 32-byte accesses (sm_100 256-bit loads and stores): a warp
// access then fills whole 32-byte sectors.  Every address is a multiple of
// 32 bytes: rows are 128 or 256 bytes, c0 is a multiple of 32 elements, and
// cs_conv_gemm requires 32-byte aligned epilogue arrays.
__device__ __forceinline__ void st256(void *p, const uint32_t *w) {
  asm volatile("st.global.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "r"(w[0]), "r"(w[1]), "r"(w[2]),
               "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7])
               : "memory");
}
__device__ __forceinline__ void ld256_nc(const void *p, uint32_t *w) {
  asm volatile("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7])
               : "l"(p));
}
// 32 bf16 of row-major storage as 2 x 32-byte loads.
__device__ __forceinline__ void load_bf16x32(const __nv_bfloat16 *p, float (&f)[32]) {
  __align__(32) __nv_bfloat16 t[32];
  ld256_nc(p, (uint32_t *)t);
  ld256_nc(p + 16, (uint32_t *)t + 8);
#pragma unroll
  for (int i = 0; i < 32; ++i) f[i] = __bfloat162float(t[i]);
}
// 32 bf16 as 2 x 32-byte stores.
__device__ __forceinline__ void store_bf16x32(__nv_bfloat16 *p, const __nv_bfloat16 (&h)[32]) {
  st256(p, (const uint32_t *)h);
  st256(p + 16, (const uint32_t *)h + 8);
}

template <int BN, int EPI>
__device__ __forceinline__ void epilogue32(const Args &a, const float (&v)[32], int row, bool valid, int c0,
                                           const float *bias) {
  const size_t o = (size_t)row * BN + c0;
  if (EPI == CS_EPI_SILU) {
    float r[32];
    if (a.resid) load_bf16x32(a.resid + o, r);
    __align__(32) __nv_bfloat16 h[32], z[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      float zz = v[i] + bias[c0 + i];
      float hh = silu(zz);
      if (a.resid) hh += r[i];
      if (!valid) {
        zz = 0.0f;
        hh = 0.0f;
      }
      z[i] = __float2bfloat16(zz);
      h[i] = __float2bfloat16(hh);
    }
    store_bf16x32(a.out + o, h);
    if (a.out_pre) store_bf16x32(a.out_pre + o, z);
  } else if (EPI == CS_EPI_LINEAR_F32) {
    float *d = a.outf + o;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      uint32_t w[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) w[j] = __float_as_uint(valid ? v[8 * i + j] + bias[c0 + 8 * i + j] : 0.0f);
      st256(d + 8 * i, w);
    }
  } else {  // CS_EPI_BWD
    float r[32], zp[32];
    if (a.resid) load_bf16x32(a.resid + o, r);
    load_bf16x32(a.zprev + o, zp);
    __align__(32) __nv_bfloat16 g[32], dz[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      float gg = v[i];
      if (a.resid) gg += r[i];
      float d = gg * dsilu(zp[i]);
      if (!valid) {
        gg = 0.0f;
        d = 0.0f;
      }
      g[i] = __float2bfloat16(gg);
      dz[i] = __float2bfloat16(d);
    }
    store_bf16x32(a.out + o, dz);
    if (a.gout) store_bf16x32(a.gout + o, g);
  }
}

// ------------------------------------------------------------------ warp-specialised kernel
// 576 threads: warp 0 loads (TMA), warp 1 issues the MMAs, warps 2-17 drain
// TMEM: warp w reads TMEM lanes 32*(w%4).. (its 32 rows) and one 32-column
// slice, so four warps per scheduler share the epilogue's latency.  The weights of all taps stay in
// shared memory for the whole launch.  For a 5-tap convolution each 64-wide
// K block of A is one TMA box of BM+4 rows (the tile plus a 2-row halo on each
// side); tap t reads rows t..t+BM-1 of it through a descriptor whose base
// address is moved by t rows.  The accumulator is double-buffered in
// TMEM (2 x BN columns) so the epilogue of one tile overlaps the MMAs of the
// next.
constexpr int EPI_WARPS = 16;
constexpr int WS_THREADS = 64 + 32 * EPI_WARPS;
constexpr int WS_SMEM = 227 * 1024;

template <int BN, int EPI, int TAPS>
__global__ void __launch_bounds__(WS_THREADS, 1)
    conv_gemm_ws_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Args a,
                        int nst) {
  constexpr int HALO = TAPS == 5 ? 2 : 0;
  constexpr int BOXR = BM + 2 * HALO;                    // rows per A box
  constexpr int A_TILE = ((BOXR + 7) / 8) * 8 * 128;     // bytes, multiple of 1024
  constexpr int W_TILE = BN * 128;                        // one (tap, kb) tile of W
  constexpr uint32_t IDESC = tcg::idesc_bf16_f32(BM, BN);
  constexpr int TMEM_COLS = 2 * BN;                       // two accumulators
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int kb_n = a.kb_per_tap;
  uint8_t *wbase = smem;
  uint8_t *abase = smem + TAPS * kb_n * W_TILE;
  float *sbias = (float *)(abase + nst * A_TILE);  // BN floats
  uint64_t *bars = (uint64_t *)(abase + nst * A_TILE + 512);
  uint64_t *wfull = bars, *full = bars + 1, *empty = full + nst, *tfull = empty + nst, *tempty = tfull + 2;
  uint64_t *drain = tempty + 2;
  uint32_t *tmem_slot = (uint32_t *)(drain + 1);
  volatile int *abort_flag = (volatile int *)(tmem_slot + 1);
  volatile uint32_t *issued = (volatile uint32_t *)(tmem_slot + 2);   // A stages issued (producer)
  volatile uint32_t *consumed = (volatile uint32_t *)(tmem_slot + 3); // A stages consumed (MMA)

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntiles = (a.rows + BM - 1) / BM;
  if (tid == 0) {
    tcg::mbar_init(wfull, 1);
    for (int s = 0; s < nst; ++s) {
      tcg::mbar_init(&full[s], 1);
      tcg::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tcg::mbar_init(&tfull[b], 1);
      tcg::mbar_init(&tempty[b], EPI_WARPS);  // one arrival per epilogue warp
    }
    tcg::mbar_init(drain, 1);
    *abort_flag = 0;
    *issued = 0;
    *consumed = 0;
    tcg::mbar_fence_init();
    tcg::tma_prefetch_desc(&tmA);
    tcg::tma_prefetch_desc(&tmB);
  }
  if (warp == 1) {
    tcg::tmem_alloc(tmem_slot, TMEM_COLS);
    tcg::tmem_relinquish();
  }
  for (int c = tid; c < BN; c += blockDim.x) sbias[c] = a.bias ? a.bias[c] : 0.0f;
  tcg::tc_fence_before();
  __syncthreads();
  tcg::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- producer
    tcg::mbar_arrive_expect_tx(wfull, (uint32_t)(TAPS * kb_n * W_TILE));
    for (int t = 0; t < TAPS; ++t)
      for (int kb = 0; kb < kb_n; ++kb)
        tcg::tma_load_2d(wbase + (t * kb_n + kb) * W_TILE, &tmB, wfull, kb * BK, t * BN);
    uint32_t it = 0;
    for (int tile = blockIdx.x; tile < ntiles && !*abort_flag; tile += gridDim.x) {
      for (int kb = 0; kb < kb_n; ++kb) {
        const int s = it % nst;
        if (it >= (uint32_t)nst && !tcg::mbar_wait(&empty[s], ((it / nst) - 1) & 1)) {
          flag(a.err, 1u);
          *abort_flag = 1;
          break;
        }
        tcg::mbar_arrive_expect_tx(&full[s], BOXR * 128);
        tcg::tma_load_2d(abase + s * A_TILE, &tmA, &full[s], kb * BK, tile * BM - HALO);
        ++it;
        *issued = it;
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer
    bool ok = tcg::mbar_wait(wfull, 0);
    uint32_t it = 0, i = 0;
    for (int tile = blockIdx.x; ok && tile < ntiles && !*abort_flag; tile += gridDim.x, ++i) {
      const int buf = i & 1;
      if (i >= 2) ok = tcg::mbar_wait(&tempty[buf], ((i >> 1) - 1) & 1);
      if (!ok) break;
      tcg::tc_fence_after();
      const uint32_t acc = tmem + (uint32_t)(buf * BN);
      for (int kb = 0; kb < kb_n && ok; ++kb) {
        const int s = it % nst;
        ok = tcg::mbar_wait(&full[s], (it / nst) & 1);
        if (!ok) break;
        tcg::tc_fence_after();
        const uint32_t sa = tcg::smem_u32(abase + s * A_TILE);
#pragma unroll
        for (int t = 0; t < TAPS; ++t) {
          const uint64_t db = tcg::sdesc_k_sw128(tcg::smem_u32(wbase + (t * kb_n + kb) * W_TILE));
          const uint64_t da = tcg::sdesc_k_sw128_rows(sa, (uint32_t)t);
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk)
            tcg::mma_bf16(acc, da + 2 * kk, db + 2 * kk, IDESC, (kb > 0 || t > 0 || kk > 0) ? 1u : 0u);
        }
        tcg::mma_commit(&empty[s]);
        ++it;
        *consumed = it;
      }
      if (ok) tcg::mma_commit(&tfull[buf]);
    }
    if (!ok) {
      flag(a.err, 1u);
      *abort_flag = 1;
    }
  } else if (warp >= 2) {
    // ---------------- epilogue
    const int quarter = warp & 3;
    const int slice = (warp - 2) >> 2;   // 32-column slice of this warp
    const bool has_cols = slice * 32 < BN;
    uint32_t i = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
      const int buf = i & 1;
      // one lane waits; the whole warp follows its verdict (tcgen05.ld is
      // warp-collective)
      int ok = 1;
      if (lane == 0) ok = tcg::mbar_wait(&tfull[buf], (i >> 1) & 1) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        if (lane == 0) {
          flag(a.err, 2u);
          *abort_flag = 1;
        }
        break;
      }
      __syncwarp();
      tcg::tc_fence_after();
      if (has_cols) {
        const int c0 = slice * 32;
        const int row = tile * BM + quarter * 32 + lane;
        const int pos = a.lp > 0 ? row % a.lp : 2;
        const bool in_range = row < a.rows;
        const bool valid = in_range && (a.lp <= 0 || (pos >= 2 && pos < 2 + a.klev));
        float v[32];
        tcg::tmem_ld32(tmem + (uint32_t)(buf * BN) + ((uint32_t)(quarter * 32) << 16) + (uint32_t)c0, v);
        if (in_range) epilogue32<BN, EPI>(a, v, row, valid, c0, sbias);
      }
      tcg::tc_fence_before();
      __syncwarp();
      if (lane == 0) tcg::mbar_arrive(&tempty[buf]);
      if (__shfl_sync(0xffffffffu, lane == 0 ? *abort_flag : 0, 0)) break;
    }
  }
  __syncthreads();
  // On an abort, let every copy and MMA this CTA issued land before shared
  // memory and TMEM are released (bounded waits).
  if (tid == 0 && *abort_flag) {
    for (uint32_t q = *consumed; q < *issued; ++q) (void)tcg::mbar_wait(&full[q % nst], (q / nst) & 1);
  }
  if (tid == 32 && *abort_flag) {
    tcg::mma_commit(drain);
    (void)tcg::mbar_wait(drain, 0);
  }
  tcg::tc_fence_before();
  __syncthreads();
  if (warp == 1) tcg::tmem_dealloc(tmem, TMEM_COLS);
}

// ------------------------------------------------------------------ fused MLP layer + output head
// Inference only: h = SiLU(A W1^T + b1) (padding rows zero) and
// y = h W2^T + b2 (f32, padding rows zero) in one kernel, h never leaving
// the SM: the epilogue warps write it as bf16 into a shared-memory tile in
// the same 128-byte-swizzled K-major layout TMA writes, and the second
// layer's MMAs read it from there.  Warp 0 streams the 128-row tiles of A
// (a 3-stage ring; both weight matrices resident), warp 1 issues the MMAs
// (tile i's first layer, then tile i-1's second layer, so the tensor core
// works while the epilogue drains), warps 2-17 drain TMEM.  The first
// layer's accumulator and h are double-buffered; the arithmetic is the
// unfused epilogues' (SiLU then bf16; bias add), so y equals the two-kernel
// result bit for bit.
constexpr int MH_WARPS = 16;
constexpr int MH_THREADS = 64 + 32 * MH_WARPS;
template <int W>
struct MhLayout {
  static constexpr int KB = W / 64;
  static constexpr int NST = 3;
  static constexpr int TILE = KB * 16384;        // 128 rows x W bf16, KB blocks of 128 x 64
  static constexpr int W1_BYTES = KB * W * 128;   // W x W
  static constexpr int W2_BYTES = KB * 64 * 128;  // 64 x W
  static constexpr int OFF_W1 = 0;
  static constexpr int OFF_W2 = OFF_W1 + W1_BYTES;
  static constexpr int OFF_A = OFF_W2 + W2_BYTES;
  static constexpr int OFF_H = OFF_A + NST * TILE;
  static constexpr int OFF_BIAS = OFF_H + 2 * TILE;
  static constexpr int OFF_BAR = OFF_BIAS + (W + 64) * 4;
  static constexpr int SMEM = OFF_BAR + 256 + 1024;
  static constexpr int TMEM_COLS = 2 * W + 128 <= 256 ? 256 : 512;
};

template <int W>
__global__ void __launch_bounds__(MH_THREADS, 1)
    mlp_head_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmW1,
                    const __grid_constant__ CUtensorMap tmW2, const float *b1, const float *b2, int rows, int lp,
                    int klev, float *y, unsigned *err) {
  using L = MhLayout<W>;
  constexpr uint32_t ID1 = tcg::idesc_bf16_f32(BM, W), ID2 = tcg::idesc_bf16_f32(BM, 64);
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  float *sb1 = (float *)(smem + L::OFF_BIAS), *sb2 = sb1 + W;
  uint64_t *bars = (uint64_t *)(smem + L::OFF_BAR);
  uint64_t *wfull = bars, *full = bars + 1, *empty = full + L::NST;
  uint64_t *t1full = empty + L::NST, *t1empty = t1full + 2, *hfull = t1empty + 2, *t2full = hfull + 2,
           *t2empty = t2full + 2, *drain = t2empty + 2;
  uint32_t *tmem_slot = (uint32_t *)(drain + 1);
  volatile int *abort_flag = (volatile int *)(tmem_slot + 1);
  volatile uint32_t *issued = (volatile uint32_t *)(tmem_slot + 2);
  volatile uint32_t *consumed = (volatile uint32_t *)(tmem_slot + 3);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntiles = (rows + BM - 1) / BM;
  if (tid == 0) {
    tcg::mbar_init(wfull, 1);
    for (int s = 0; s < L::NST; ++s) {
      tcg::mbar_init(&full[s], 1);
      tcg::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tcg::mbar_init(&t1full[b], 1);
      tcg::mbar_init(&t1empty[b], MH_WARPS);
      tcg::mbar_init(&hfull[b], MH_WARPS);
      tcg::mbar_init(&t2full[b], 1);
      tcg::mbar_init(&t2empty[b], MH_WARPS);
    }
    tcg::mbar_init(drain, 1);
    *abort_flag = 0;
    *issued = 0;
    *consumed = 0;
    tcg::mbar_fence_init();
    tcg::tma_prefetch_desc(&tmA);
    tcg::tma_prefetch_desc(&tmW1);
    tcg::tma_prefetch_desc(&tmW2);
  }
  if (warp == 1) {
    tcg::tmem_alloc(tmem_slot, L::TMEM_COLS);
    tcg::tmem_relinquish();
  }
  for (int c = tid; c < W; c += blockDim.x) sb1[c] = b1 ? b1[c] : 0.0f;
  for (int c = tid; c < 64; c += blockDim.x) sb2[c] = b2 ? b2[c] : 0.0f;
  tcg::tc_fence_before();
  __syncthreads();
  tcg::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- producer
    tcg::mbar_arrive_expect_tx(wfull, (uint32_t)(L::W1_BYTES + L::W2_BYTES));
    for (int kb = 0; kb < L::KB; ++kb) tcg::tma_load_2d(smem + L::OFF_W1 + kb * W * 128, &tmW1, wfull, kb * BK, 0);
    for (int kb = 0; kb < L::KB; ++kb) tcg::tma_load_2d(smem + L::OFF_W2 + kb * 64 * 128, &tmW2, wfull, kb * BK, 0);
    uint32_t it = 0;
    for (int tile = blockIdx.x; tile < ntiles && !*abort_flag; tile += gridDim.x, ++it) {
      const int s = it % L::NST;
      if (it >= (uint32_t)L::NST && !tcg::mbar_wait(&empty[s], ((it / L::NST) - 1) & 1)) {
        flag(err, 1u);
        *abort_flag = 1;
        break;
      }
      tcg::mbar_arrive_expect_tx(&full[s], (uint32_t)L::TILE);
      for (int kb = 0; kb < L::KB; ++kb)
        tcg::tma_load_2d(smem + L::OFF_A + s * L::TILE + kb * 16384, &tmA, &full[s], kb * BK, tile * BM);
      *issued = it + 1;
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer
    // second layer of local tile j: h (shared memory) x W2^T into the second accumulator
    auto layer2 = [&](uint32_t j) -> bool {
      const int b = j & 1;
      if (!tcg::mbar_wait(&hfull[b], (j >> 1) & 1)) return false;
      if (j >= 2 && !tcg::mbar_wait(&t2empty[b], ((j >> 1) - 1) & 1)) return false;
      tcg::tc_fence_after();
      const uint32_t acc = tmem + (uint32_t)(2 * W + b * 64);
      const uint32_t sh = tcg::smem_u32(smem + L::OFF_H + b * L::TILE);
#pragma unroll
      for (int kb = 0; kb < L::KB; ++kb) {
        const uint64_t da = tcg::sdesc_k_sw128(sh + kb * 16384);
        const uint64_t db = tcg::sdesc_k_sw128(tcg::smem_u32(smem + L::OFF_W2 + kb * 64 * 128));
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk)
          tcg::mma_bf16(acc, da + 2 * kk, db + 2 * kk, ID2, (kb > 0 || kk > 0) ? 1u : 0u);
      }
      tcg::mma_commit(&t2full[b]);
      return true;
    };
    bool ok = tcg::mbar_wait(wfull, 0);
    uint32_t i = 0;
    for (int tile = blockIdx.x; ok && tile < ntiles && !*abort_flag; tile += gridDim.x, ++i) {
      const int b = i & 1, s = i % L::NST;
      if (i >= 2) ok = tcg::mbar_wait(&t1empty[b], ((i >> 1) - 1) & 1);
      if (ok) ok = tcg::mbar_wait(&full[s], (i / L::NST) & 1);
      if (!ok) break;
      tcg::tc_fence_after();
      const uint32_t acc = tmem + (uint32_t)(b * W);
      const uint32_t sa = tcg::smem_u32(smem + L::OFF_A + s * L::TILE);
#pragma unroll
      for (int kb = 0; kb < L::KB; ++kb) {
        const uint64_t da = tcg::sdesc_k_sw128(sa + kb * 16384);
        const uint64_t db = tcg::sdesc_k_sw128(tcg::smem_u32(smem + L::OFF_W1 + kb * W * 128));
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk)
          tcg::mma_bf16(acc, da + 2 * kk, db + 2 * kk, ID1, (kb > 0 || kk > 0) ? 1u : 0u);
      }
      tcg::mma_commit(&empty[s]);
      tcg::mma_commit(&t1full[b]);
      *consumed = i + 1;
      if (i >= 1 && !layer2(i - 1)) {
        ok = false;
        break;
      }
    }
    if (ok && i >= 1 && !*abort_flag) ok = layer2(i - 1);
    if (!ok) {
      flag(err, 1u);
      *abort_flag = 1;
    }
  } else if (warp >= 2) {
    // ---------------- epilogue, software-pipelined: the first layer of tile
    // i, then the output head of tile i-1 (its MMAs long finished), so no
    // warp waits for the second layer of the tile it has just handed over.
    // The head's 64 columns go to slices 0-1 at width 128 and to the slices
    // the first layer leaves idle (2-3) at width 64.
    const int quarter = warp & 3, slice = (warp - 2) >> 2;
    const int hslice = W == 64 ? slice - 2 : slice;  // head column slice of this warp, 0 or 1 if any
    // drain the output head of local tile j (rows of `tile`) into y
    auto head = [&](uint32_t j, int tile) -> bool {
      const int b = j & 1;
      int ok = 1;
      if (lane == 0) ok = tcg::mbar_wait(&t2full[b], (j >> 1) & 1) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) return false;
      __syncwarp();
      tcg::tc_fence_after();
      if (hslice >= 0 && hslice < 2) {
        const int row = tile * BM + quarter * 32 + lane;
        const int pos = lp > 0 ? row % lp : 2;
        const bool valid = row < rows && (lp <= 0 || (pos >= 2 && pos < 2 + klev));
        float v[32];
        tcg::tmem_ld32(tmem + (uint32_t)(2 * W + b * 64) + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(hslice * 32),
                       v);
        if (row < rows) {
          float *d = y + (size_t)row * 64 + hslice * 32;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            uint32_t w8[8];
#pragma unroll
            for (int jj = 0; jj < 8; ++jj)
              w8[jj] = __float_as_uint(valid ? v[8 * q + jj] + sb2[hslice * 32 + 8 * q + jj] : 0.0f);
            st256(d + 8 * q, w8);
          }
        }
      }
      tcg::tc_fence_before();
      __syncwarp();
      if (lane == 0) tcg::mbar_arrive(&t2empty[b]);
      return true;
    };
    uint32_t i = 0;
    bool ok_all = true;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++i) {
      const int b = i & 1;
      int ok = 1;
      if (lane == 0) ok = tcg::mbar_wait(&t1full[b], (i >> 1) & 1) ? 1 : 0;
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) {
        ok_all = false;
        break;
      }
      __syncwarp();
      tcg::tc_fence_after();
      if (slice * 32 < W) {
        const int rt = quarter * 32 + lane, row = tile * BM + rt;
        const int pos = lp > 0 ? row % lp : 2;
        const bool valid = row < rows && (lp <= 0 || (pos >= 2 && pos < 2 + klev));
        float v[32];
        tcg::tmem_ld32(tmem + (uint32_t)(b * W) + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(slice * 32), v);
        __align__(16) __nv_bfloat16 h[32];
#pragma unroll
        for (int q = 0; q < 32; ++q) {
          float hh = silu(v[q] + sb1[slice * 32 + q]);
          if (!valid) hh = 0.0f;
          h[q] = __float2bfloat16(hh);
        }
        uint8_t *hb = smem + L::OFF_H + b * L::TILE;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int chunk = slice * 4 + j, kb = chunk >> 3, c = chunk & 7;  // 16-byte chunk of the row
          *reinterpret_cast<uint4 *>(hb + kb * 16384 + rt * 128 + ((c ^ (rt & 7)) << 4)) =
              reinterpret_cast<const uint4 *>(h)[j];
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      }
      tcg::tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        tcg::mbar_arrive(&t1empty[b]);
        tcg::mbar_arrive(&hfull[b]);
      }
      if (i >= 1 && !head(i - 1, tile - (int)gridDim.x)) {
        ok_all = false;
        break;
      }
      if (__shfl_sync(0xffffffffu, lane == 0 ? *abort_flag : 0, 0)) {
        ok_all = false;
        break;
      }
    }
    if (ok_all && i >= 1 && !head(i - 1, blockIdx.x + (int)(i - 1) * (int)gridDim.x)) ok_all = false;
    if (!ok_all && lane == 0) {
      flag(err, 2u);
      *abort_flag = 1;
    }
  }
  __syncthreads();
  // On an abort, let every copy and MMA this CTA issued land before shared
  // memory and TMEM are released (bounded waits).
  if (tid == 0 && *abort_flag) {
    for (uint32_t q = *consumed; q < *issued; ++q) (void)tcg::mbar_wait(&full[q % L::NST], (q / L::NST) & 1);
  }
  if (tid == 32 && *abort_flag) {
    tcg::mma_commit(drain);
    (void)tcg::mbar_wait(drain, 0);
  }
  tcg::tc_fence_before();
  __syncthreads();
  if (warp == 1) tcg::tmem_dealloc(tmem, L::TMEM_COLS);
}

// ------------------------------------------------------------------ weight gradients
// dW[t][n][k] += sum_r dZ[r][n] * X[r + t - taps/2][k]: one GEMM per tap whose
// reduction runs over the rows, the outer dimension of both operands.  Both
// are therefore read MN-major: TMA fetches boxes of 64 features x 64 rows
// (128 bytes per row, 128-byte swizzle), a row per K index, and the
// descriptor walks them with 8-row groups 1024 bytes apart (SBO) and the
// second 64 features one box further (LBO).  M = 128 covers dZ's features
// (the upper half zero when n = 64), N = X's features (64 or 128).  Each CTA
// reduces one chunk of rows of one tap into a TMEM accumulator, then adds it
// to dW (f32 vector reductions).  Rows outside [0, rows) read as zero, as do
// X rows shifted past either end.
constexpr int WG_RK = 64;                    // rows (K) per stage
constexpr int WG_STAGES = 4;
constexpr int WG_HALF = WG_RK * 128;         // one box of 64 features: 8 KB
constexpr int WG_STAGE = 4 * WG_HALF;        // dZ (two halves) + X (two halves)
constexpr int WG_SMEM = WG_STAGES * WG_STAGE + 1024 + 256;

__device__ __forceinline__ uint64_t sdesc_mn_sw128(uint32_t saddr, uint32_t lbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu)          // start address / 16
         | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16)  // leading byte offset: the next 64 features
         | ((uint64_t)(1024 >> 4) << 32)             // stride byte offset: 8-row groups along K
         | ((uint64_t)1 << 46)                       // descriptor version
         | ((uint64_t)2 << 61);                      // swizzle: 128 B
}
__device__ __forceinline__ void red_add_v4(float *p, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b), "f"(c), "f"(d)
               : "memory");
}

template <int BN>
__global__ void __launch_bounds__(128, 1)
    wgrad_tc_kernel(const __grid_constant__ CUtensorMap tmD, const __grid_constant__ CUtensorMap tmX, int rows,
                    int chunk, int n, int taps, float *dw, unsigned *err) {
  // transpose bits 15 and 16: both operands MN-major
  constexpr uint32_t IDESC = tcg::idesc_bf16_f32(128, BN) | (1u << 15) | (1u << 16);
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *bars = (uint64_t *)(smem + WG_STAGES * WG_STAGE);
  uint64_t *full = bars, *empty = bars + WG_STAGES, *tfull = empty + WG_STAGES, *drain = tfull + 1;
  uint32_t *tmem_slot = (uint32_t *)(drain + 1);
  volatile int *abort_flag = (volatile int *)(tmem_slot + 1);
  volatile uint32_t *issued = (volatile uint32_t *)(tmem_slot + 2);
  volatile uint32_t *consumed = (volatile uint32_t *)(tmem_slot + 3);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int t = blockIdx.y, shift = t - taps / 2;
  const int r0 = blockIdx.x * chunk;
  const int r1 = min(rows, r0 + chunk);
  const int nkb = (r1 - r0 + WG_RK - 1) / WG_RK;
  const int nh = n / 64;
  constexpr int KH = BN / 64;
  // the dZ half TMA never writes (n = 64) stays zero: M is always 128
  if (nh == 1) {
    for (int i = tid; i < WG_STAGES * WG_HALF / 16; i += blockDim.x) {
      const int s = i / (WG_HALF / 16), j = i % (WG_HALF / 16);
      reinterpret_cast<uint4 *>(smem + s * WG_STAGE + WG_HALF)[j] = make_uint4(0u, 0u, 0u, 0u);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (tid == 0) {
    for (int s = 0; s < WG_STAGES; ++s) {
      tcg::mbar_init(&full[s], 1);
      tcg::mbar_init(&empty[s], 1);
    }
    tcg::mbar_init(tfull, 1);
    tcg::mbar_init(drain, 1);
    *abort_flag = 0;
    *issued = 0;
    *consumed = 0;
    tcg::mbar_fence_init();
    tcg::tma_prefetch_desc(&tmD);
    tcg::tma_prefetch_desc(&tmX);
  }
  if (warp == 1) {
    tcg::tmem_alloc(tmem_slot, BN);
    tcg::tmem_relinquish();
  }
  tcg::tc_fence_before();
  __syncthreads();
  tcg::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- producer
    for (int kb = 0; kb < nkb && !*abort_flag; ++kb) {
      const int s = kb % WG_STAGES;
      if (kb >= WG_STAGES && !tcg::mbar_wait(&empty[s], ((kb / WG_STAGES) - 1) & 1)) {
        flag(err, 1u);
        *abort_flag = 1;
        break;
      }
      uint8_t *st = smem + s * WG_STAGE;
      const int r = r0 + kb * WG_RK;
      tcg::mbar_arrive_expect_tx(&full[s], (uint32_t)((nh + KH) * WG_HALF));
      for (int h = 0; h < nh; ++h) tcg::tma_load_2d(st + h * WG_HALF, &tmD, &full[s], h * 64, r);
      for (int h = 0; h < KH; ++h) tcg::tma_load_2d(st + (2 + h) * WG_HALF, &tmX, &full[s], h * 64, r + shift);
      *issued = (uint32_t)(kb + 1);
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer
    bool ok = true;
    for (int kb = 0; kb < nkb && !*abort_flag; ++kb) {
      const int s = kb % WG_STAGES;
      ok = tcg::mbar_wait(&full[s], (kb / WG_STAGES) & 1);
      if (!ok) break;
      tcg::tc_fence_after();
      const uint32_t sa = tcg::smem_u32(smem + s * WG_STAGE);
      const uint64_t da = sdesc_mn_sw128(sa, WG_HALF);
      const uint64_t db = sdesc_mn_sw128(sa + 2 * WG_HALF, WG_HALF);
#pragma unroll
      for (int kk = 0; kk < WG_RK / 16; ++kk)  // 16 rows = two 1024-byte groups per instruction
        tcg::mma_bf16(tmem, da + (uint64_t)(kk * (2048 >> 4)), db + (uint64_t)(kk * (2048 >> 4)), IDESC,
                      (kb > 0 || kk > 0) ? 1u : 0u);
      tcg::mma_commit(&empty[s]);
      *consumed = (uint32_t)(kb + 1);
    }
    if (ok && !*abort_flag) {
      tcg::mma_commit(tfull);
    } else {
      flag(err, 1u);
      *abort_flag = 1;
    }
  }
  __syncwarp();
  // ---------------- epilogue: warp w holds TMEM lanes 32w.. = features n of dZ
  int ok = 1;
  if (lane == 0) ok = (!*abort_flag && tcg::mbar_wait(tfull, 0)) ? 1 : 0;
  ok = __shfl_sync(0xffffffffu, ok, 0);
  if (ok) {
    tcg::tc_fence_after();
    const int m0 = warp * 32;
    if (m0 < n) {
#pragma unroll
      for (int c0 = 0; c0 < BN; c0 += 32) {
        float v[32];
        tcg::tmem_ld32(tmem + ((uint32_t)m0 << 16) + (uint32_t)c0, v);
        float *d = dw + ((size_t)t * n + m0 + lane) * BN + c0;
#pragma unroll
        for (int i = 0; i < 32; i += 4) red_add_v4(d + i, v[i], v[i + 1], v[i + 2], v[i + 3]);
      }
    }
  } else if (lane == 0) {
    flag(err, 2u);
    *abort_flag = 1;
  }
  __syncthreads();
  // On an abort, let every copy and MMA this CTA issued land before shared
  // memory and TMEM are released (bounded waits).
  if (tid == 0 && *abort_flag) {
    for (uint32_t q = *consumed; q < *issued; ++q)
      (void)tcg::mbar_wait(&full[q % WG_STAGES], (q / WG_STAGES) & 1);
  }
  if (tid == 32 && *abort_flag) {
    tcg::mma_commit(drain);
    (void)tcg::mbar_wait(drain, 0);
  }
  tcg::tc_fence_before();
  __syncthreads();
  if (warp == 1) tcg::tmem_dealloc(tmem, BN);
}

// ------------------------------------------------------------------ host side
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  return fn;
}

// Row-major [rows][cols] bf16 matrix, boxes of 64 columns x box_rows rows,
// 128-byte swizzle; out-of-range rows read as zero.
bool make_map(CUtensorMap *m, const void *base, uint64_t rows, uint64_t cols, uint32_t box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {cols * 2};
  cuuint32_t box[2] = {64, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int BN, int EPI>
cudaError_t launch_t(const CUtensorMap &ma, const CUtensorMap &mb, const Args &a, int grid, cudaStream_t st) {
  const int smem = STAGES * (A_BYTES + BN * BK * 2) + 1024 + 256;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e =
        cudaFuncSetAttribute(conv_gemm_kernel<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  conv_gemm_kernel<BN, EPI><<<grid, 128, smem, st>>>(ma, mb, a);
  return cudaGetLastError();
}

template <int BN, int EPI, int TAPS>
cudaError_t launch_ws_t(const CUtensorMap &ma, const CUtensorMap &mb, const Args &a, int grid, int nst,
                        cudaStream_t st) {
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(conv_gemm_ws_kernel<BN, EPI, TAPS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, WS_SMEM);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  conv_gemm_ws_kernel<BN, EPI, TAPS><<<grid, WS_THREADS, WS_SMEM, st>>>(ma, mb, a, nst);
  return cudaGetLastError();
}

template <int BN>
cudaError_t launch_ws_n(const CUtensorMap &ma, const CUtensorMap &mb, const Args &a, int grid, int nst,
                        cudaStream_t st) {
  if (a.taps == 5) {
    if (a.epi == CS_EPI_SILU) return launch_ws_t<BN, CS_EPI_SILU, 5>(ma, mb, a, grid, nst, st);
    if (a.epi == CS_EPI_BWD) return launch_ws_t<BN, CS_EPI_BWD, 5>(ma, mb, a, grid, nst, st);
    return launch_ws_t<BN, CS_EPI_LINEAR_F32, 5>(ma, mb, a, grid, nst, st);
  }
  if (a.epi == CS_EPI_SILU) return launch_ws_t<BN, CS_EPI_SILU, 1>(ma, mb, a, grid, nst, st);
  if (a.epi == CS_EPI_BWD) return launch_ws_t<BN, CS_EPI_BWD, 1>(ma, mb, a, grid, nst, st);
  return launch_ws_t<BN, CS_EPI_LINEAR_F32, 1>(ma, mb, a, grid, nst, st);
}

template <int BN>
cudaError_t launch_wgrad_t(const CUtensorMap &md, const CUtensorMap &mx, int rows, int chunk, int nchunks, int n,
                           int taps, float *dw, unsigned *err, cudaStream_t st) {
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(wgrad_tc_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, WG_SMEM);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  wgrad_tc_kernel<BN><<<dim3(nchunks, taps), 128, WG_SMEM, st>>>(md, mx, rows, chunk, n, taps, dw, err);
  return cudaGetLastError();
}

template <int W>
cudaError_t launch_mh_t(const CUtensorMap &ma, const CUtensorMap &m1, const CUtensorMap &m2, const float *b1,
                        const float *b2, int rows, int lp, int klev, float *y, unsigned *err, int grid,
                        cudaStream_t st) {
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e =
        cudaFuncSetAttribute(mlp_head_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, MhLayout<W>::SMEM);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  mlp_head_kernel<W><<<grid, MH_THREADS, MhLayout<W>::SMEM, st>>>(ma, m1, m2, b1, b2, rows, lp, klev, y, err);
  return cudaGetLastError();
}
static_assert(MhLayout<128>::SMEM <= WS_SMEM, "the fused kernel fits in shared memory");

int g_impl = 0;  // 0: warp-specialised kernel, 1: the single-thread pipeline

}  // namespace sg

extern "C" int cs_set_gemm_impl(int32_t impl) {
  if (impl != 0 && impl != 1) return CS_E_ARG;
  sg::g_impl = impl;
  return CS_OK;
}

extern "C" int cs_conv_gemm(const cs_gemm_desc *g, void *stream) {
  using namespace sg;
  if (!g || !g->a || !g->w) return CS_E_ARG;
  if (g->k % 64 || g->k <= 0 || (g->n != 64 && g->n != 128) || (g->taps != 1 && g->taps != 5) ||
      g->rows <= 0)
    return CS_E_ARG;
  if (g->epi < CS_EPI_SILU || g->epi > CS_EPI_BWD) return CS_E_ARG;
  if (g->epi == CS_EPI_LINEAR_F32 ? !g->outf : !g->out) return CS_E_ARG;
  if (g->epi == CS_EPI_BWD && !g->zprev) return CS_E_ARG;
  // TMA operands on 16 bytes; the epilogue's 32-byte accesses need every
  // array it reads or writes on 32 bytes
  if (((uintptr_t)g->a | (uintptr_t)g->w) & 15) return CS_E_ARG;
  if (((uintptr_t)g->out | (uintptr_t)g->out_pre | (uintptr_t)g->gout | (uintptr_t)g->outf |
       (uintptr_t)g->resid | (uintptr_t)g->zprev) &
      31)
    return CS_E_ARG;
  // warp-specialised kernel: all weights resident in shared memory plus at
  // least two A stages of BM + halo rows
  const int halo = g->taps == 5 ? 2 : 0;
  const int a_tile = ((BM + 2 * halo + 7) / 8) * 8 * 128;
  const int w_bytes = g->taps * (g->k / 64) * g->n * 128;
  int nst = (WS_SMEM - 1024 - 1024 - w_bytes) / a_tile;
  if (nst > 8) nst = 8;
  const bool ws = g_impl == 0 && nst >= 2;
  CUtensorMap ma, mb;
  if (!make_map(&ma, g->a, (uint64_t)g->rows, (uint64_t)g->k, ws ? (uint32_t)(BM + 2 * halo) : (uint32_t)BM))
    return CS_E_CUDA;
  if (!make_map(&mb, g->w, (uint64_t)g->taps * g->n, (uint64_t)g->k, (uint32_t)g->n)) return CS_E_CUDA;
  Args a;
  memset(&a, 0, sizeof(a));
  a.rows = g->rows;
  a.kb_per_tap = g->k / 64;
  a.taps = g->taps;
  a.tap_origin = g->taps == 5 ? -2 : 0;
  a.lp = g->lp;
  a.klev = g->klev;
  a.epi = g->epi;
  a.bias = g->bias;
  a.out = (__nv_bfloat16 *)g->out;
  a.out_pre = (__nv_bfloat16 *)g->out_pre;
  a.resid = (const __nv_bfloat16 *)g->resid;
  a.zprev = (const __nv_bfloat16 *)g->zprev;
  a.gout = (__nv_bfloat16 *)g->gout;
  a.outf = g->outf;
  a.err = g->err;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = (g->rows + BM - 1) / BM;
  const int grid = ntiles < sms ? ntiles : sms;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (ws) {
    e = g->n == 128 ? launch_ws_n<128>(ma, mb, a, grid, nst, st) : launch_ws_n<64>(ma, mb, a, grid, nst, st);
    return e == cudaSuccess ? CS_OK : CS_E_CUDA;
  }
  if (g->n == 128) {
    if (g->epi == CS_EPI_SILU) e = launch_t<128, CS_EPI_SILU>(ma, mb, a, grid, st);
    else if (g->epi == CS_EPI_BWD) e = launch_t<128, CS_EPI_BWD>(ma, mb, a, grid, st);
    else e = launch_t<128, CS_EPI_LINEAR_F32>(ma, mb, a, grid, st);
  } else {
    if (g->epi == CS_EPI_SILU) e = launch_t<64, CS_EPI_SILU>(ma, mb, a, grid, st);
    else if (g->epi == CS_EPI_BWD) e = launch_t<64, CS_EPI_BWD>(ma, mb, a, grid, st);
    else e = launch_t<64, CS_EPI_LINEAR_F32>(ma, mb, a, grid, st);
  }
  return e == cudaSuccess ? CS_OK : CS_E_CUDA;
}

// dW[t][n][k] += sum over rows of dZ[r][n] X[r + t - taps/2][k] on the tensor
// cores (wgrad_tc_kernel): dZ [rows][n], X [rows][k] bf16 row-major, dW f32.
extern "C" int cs_wgrad_tc(const void *dz, const void *x, int32_t rows, int32_t n, int32_t k, int32_t taps,
                           float *dw, unsigned *err, void *stream) {
  using namespace sg;
  if (!dz || !x || !dw || rows <= 0 || (n != 64 && n != 128) || (k != 64 && k != 128) || (taps != 1 && taps != 5))
    return CS_E_ARG;
  if (((uintptr_t)dz | (uintptr_t)x | (uintptr_t)dw) & 15) return CS_E_ARG;
  CUtensorMap md, mx;
  if (!make_map(&md, dz, (uint64_t)rows, (uint64_t)n, (uint32_t)WG_RK)) return CS_E_CUDA;
  if (!make_map(&mx, x, (uint64_t)rows, (uint64_t)k, (uint32_t)WG_RK)) return CS_E_CUDA;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // about two CTAs per SM over all taps, chunks of at least 512 rows (each
  // chunk adds its n x k partial to dW)
  int nchunks = (2 * sms + taps - 1) / taps;
  const int maxchunks = (rows + 511) / 512;
  if (nchunks > maxchunks) nchunks = maxchunks;
  if (nchunks < 1) nchunks = 1;
  int chunk = (rows + nchunks - 1) / nchunks;
  chunk = (chunk + WG_RK - 1) / WG_RK * WG_RK;
  nchunks = (rows + chunk - 1) / chunk;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = k == 128 ? launch_wgrad_t<128>(md, mx, rows, chunk, nchunks, n, taps, dw, err, st)
                           : launch_wgrad_t<64>(md, mx, rows, chunk, nchunks, n, taps, dw, err, st);
  return e == cudaSuccess ? CS_OK : CS_E_CUDA;
}

// The network's MLP layer and output head in one kernel (inference):
// y = (SiLU(a w1^T + b1)) w2^T + b2, the hidden activation kept on chip
// (mlp_head_kernel).  a [rows][k] bf16, w1 [k][k], w2 [64][k] bf16, y f32
// [rows][64]; k 64 or 128; rows outside the levels of the lp/klev column
// layout written as zero.
extern "C" int cs_mlp_head(const void *a, const void *w1, const float *b1, const void *w2, const float *b2,
                           int32_t rows, int32_t k, int32_t lp, int32_t klev, float *y, unsigned *err,
                           void *stream) {
  using namespace sg;
  if (!a || !w1 || !w2 || !y || rows <= 0 || (k != 64 && k != 128)) return CS_E_ARG;
  if (((uintptr_t)a | (uintptr_t)w1 | (uintptr_t)w2) & 15) return CS_E_ARG;
  if ((uintptr_t)y & 31) return CS_E_ARG;
  CUtensorMap ma, m1, m2;
  if (!make_map(&ma, a, (uint64_t)rows, (uint64_t)k, (uint32_t)BM)) return CS_E_CUDA;
  if (!make_map(&m1, w1, (uint64_t)k, (uint64_t)k, (uint32_t)k)) return CS_E_CUDA;
  if (!make_map(&m2, w2, 64, (uint64_t)k, 64)) return CS_E_CUDA;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = (rows + BM - 1) / BM;
  const int grid = ntiles < sms ? ntiles : sms;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = k == 128 ? launch_mh_t<128>(ma, m1, m2, b1, b2, rows, lp, klev, y, err, grid, st)
                           : launch_mh_t<64>(ma, m1, m2, b1, b2, rows, lp, klev, y, err, grid, st);
  return e == cudaSuccess ? CS_OK : CS_E_CUDA;
}
