// CLOUDSC kernels for B200 (sm_100a): FP64 (the reference's double build) and
// FP32-mixed.  One thread walks one column through all levels; all NPROMA
// blocks are processed by one persistent launch (a grid-stride loop over
// column tiles).  See cloudsc_column.cuh for the numerical contract.
//
// Compiled with --fmad=false: no multiply-add contraction, so the FP64 kernel
// performs the reference's operations with one rounding each.
#include <cuda_runtime.h>
#include <cstdint>

#define CSC_DEV __device__ __forceinline__
#include "cloudsc_column.cuh"

#include "cloudsc_kparams.h"

namespace cloudsc {

__constant__ KParams<double> c_kpd;
__constant__ KParams<float> c_kpf;
__constant__ KParamsD c_kd;

template <typename Real>
__device__ __forceinline__ const KParams<Real> &KP();
template <>
__device__ __forceinline__ const KParams<double> &KP<double>() { return c_kpd; }
template <>
__device__ __forceinline__ const KParams<float> &KP<float>() { return c_kpf; }

template <typename T>
__device__ __forceinline__ T ld(const T *p) { return __ldg(p); }
__device__ __forceinline__ void atomic_add(uint32_t *p, uint32_t v) { atomicAdd(p, v); }
__device__ __forceinline__ double xabs(double x) { return fabs(x); }
__device__ __forceinline__ float xabs(float x) { return fabsf(x); }
__device__ __forceinline__ double xsign(double a, double b) { return copysign(a, b); }
__device__ __forceinline__ float xsign(float a, float b) { return copysignf(a, b); }

}  // namespace cloudsc

#include "cloudsc_body.cuh"

namespace cloudsc {

template <bool F32M, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) cloudsc_kernel(Fields F, Shape sh) {
  const int tpb = blockDim.x;
  const int tiles_per_blk = (sh.nproma + tpb - 1) / tpb;
  const int ntiles = sh.ngpblks * tiles_per_blk;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int ib = tile / tiles_per_blk;
    const int jl = (tile - ib * tiles_per_blk) * tpb + threadIdx.x;
    const int icend = min(sh.nproma, sh.ngptot - ib * sh.nproma);
    if (jl >= sh.kidia0 && jl < icend) cloudsc_column<double, F32M>(F, sh, ib, jl);
  }
}

}  // namespace cloudsc

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace cloudsc {

// Upload the parameters to this device's constant memory (all three blocks).
cudaError_t upload_params(const cloudsc_params &p, const Derived &d) {
  KParams<double> kd;
  KParams<float> kf;
  fill_kparams(p, d, kd);
  fill_kparams(p, d, kf);
  KParamsD dd;
  fill_kparams_d(p, dd);
  cudaError_t e = cudaMemcpyToSymbol(c_kpd, &kd, sizeof(kd));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_kpf, &kf, sizeof(kf));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_kd, &dd, sizeof(dd));
  return e;
}

// Register budget: __launch_bounds__(CLOUDSC_MAXT, CLOUDSC_MINB).  128 threads
// x 3 CTAs per SM caps the kernels at 168 registers (a few hundred bytes of
// spills): 12 warps per SM hide more FP64 latency than 8 warps at 255
// registers (measured 23.2 ms vs 28.6 ms for the FP64 kernel at 262,144
// columns).
// The FP32-mixed kernel is fastest with the full 255 registers (measured
// 22.6 ms vs 27.7 ms at 168).
#ifndef CLOUDSC_MAXT
#define CLOUDSC_MAXT 128
#endif
#ifndef CLOUDSC_MINB
#define CLOUDSC_MINB 3
#endif
#ifndef CLOUDSC_MIX_MAXT
#define CLOUDSC_MIX_MAXT 256
#endif
#ifndef CLOUDSC_MIX_MINB
#define CLOUDSC_MIX_MINB 1
#endif

// Largest CTA the kernel of `precision` was compiled for.
int max_threads(int precision) { return precision == 0 ? CLOUDSC_MAXT : CLOUDSC_MIX_MAXT; }

// Launch the kernel: precision 0 = FP64, 1 = FP32-mixed.
cudaError_t launch(int precision, const Fields &f, const Shape &sh, int threads, int grid,
                   cudaStream_t stream) {
  if (precision == 0) {
    if (threads > CLOUDSC_MAXT) return cudaErrorInvalidConfiguration;
    cloudsc_kernel<false, CLOUDSC_MAXT, CLOUDSC_MINB><<<grid, threads, 0, stream>>>(f, sh);
  } else {
    if (threads > CLOUDSC_MIX_MAXT) return cudaErrorInvalidConfiguration;
    cloudsc_kernel<true, CLOUDSC_MIX_MAXT, CLOUDSC_MIX_MINB><<<grid, threads, 0, stream>>>(f, sh);
  }
  return cudaGetLastError();
}

}  // namespace cloudsc

