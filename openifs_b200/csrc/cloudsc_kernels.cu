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
// plibm's exp/log tables are read from a shared-memory copy per CTA (filled
// at kernel start): the table lookups sit on the dependent path of every
// exp and pow, and shared-memory latency is below the L1 hit latency of a
// global load.  Measured at 262,144 columns, FP64: 15.75 ms vs 16.05 ms.
#define PLIBM_SMEM_TABLES 1
// Every column of a CTA meets the others at the end of each level, so all
// warps of the CTA run the same stretch of the (very long) level code at the
// same time and share the instruction cache.
#define CSC_LEVEL_SYNC() __syncthreads()
#include <type_traits>

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
#include "satadj_point.cuh"

namespace cloudsc {

// Columns are numbered g = ib * NPROMA + jl over all blocks and dealt to CTAs
// in tiles of blockDim.x consecutive columns (a warp reads 32 neighbouring
// columns: coalesced).  The tile loop is uniform over the CTA and every thread
// runs the level loop, so the per-level barrier is reached by all; a thread
// whose column is outside KIDIA..ICEND computes a valid stand-in column and
// stores nothing.
// FORM selects the arithmetic of the column body:
//   0  FP64, the reference's double build;
//   1  FP32-mixed: FP32 transcendentals, everything else in double;
//   3  FP64 with the cloud budget diagnostics (LCLDBUD*: PEXTRA written);
//   4  FP64 with the SPP perturbations and the cloud-inhomogeneity paths;
//   5  FP64 with both (3 and 4);
//   2  FP32 physics: the process rates in FP32 as well (Real = float); the
//      state, the sink limiters, the 5x5 solve, CLOUD_SUPERSATCHECK and the
//      tendency and flux budgets stay in double.  Float rounding of the rates
//      leaves residues above CLOUDSC's 1e-14 kg/kg thresholds that switch
//      precipitation processes on and off down the column, so this form is
//      faster but further from FP64 (measured tendency errors of 0.3-4 %).
// FT: Fields (the double-precision interface) or FieldsSP (float arrays,
// forms 0-2 only).  GEN: the parameter-exponent pows without their tests for
// the exponents 0.5, 1.5, 2 and 3 (the host launches it when the uploaded
// parameters have none of these, gen_exponents_ok).  FAST (KLEV <=
// kMaxLevFast): every column runs the fast pass (the branch-free division,
// fast_div); a column whose pass reported an operand outside that division's
// exact window is run again with IEEE division, so that the outputs are
// those of IEEE division for every input (with the budgets, the two passes
// split PEXTRA's levels between them: cloudsc_column, kbud).
template <int FORM, int MAXT, int MINB, typename FT = Fields, bool GEN = false, bool FAST = false>
__global__ void __launch_bounds__(MAXT, MINB) cloudsc_kernel(FT F, Shape sh) {
  // Let ptxas place part of the register spills in shared memory instead of
  // local memory (a PTX pragma; the spill slots it moves no longer go
  // through L1/L2).  With the shared-memory tables, FP64: 15.29 ms vs
  // 15.75 ms; FP32-mixed: 11.28 ms vs 11.72 ms.
  asm volatile(".pragma \"enable_smem_spilling\";");
  plibm_load_tables();
  const long long ncols = (long long)sh.ngpblks * sh.nproma;
  const long long ntiles = (ncols + blockDim.x - 1) / blockDim.x;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long g = tile * blockDim.x + threadIdx.x;
    int ib = (int)(g / sh.nproma);
    int jl = (int)(g - (long long)ib * sh.nproma);
    bool active = ib < sh.ngpblks;
    if (active) active = jl >= sh.kidia0 && jl < min(sh.nproma, sh.ngptot - ib * sh.nproma);
    if (!active) {
      ib = 0;
      jl = sh.kidia0;
    }
    if constexpr (FORM >= 3) {
      constexpr bool BUD = FORM == 3 || FORM == 5, OPT = FORM >= 4;
      if constexpr (FAST) {
        double plude_in[kMaxLevFast];
        bool bad = false;
        int kbud = sh.klev;
        cloudsc_column<double, false, BUD, OPT, FT, GEN, kPassFast>(F, sh, ib, jl, active, &bad, plude_in, &kbud);
        if (__syncthreads_or(bad))
          cloudsc_column<double, false, BUD, OPT, FT, GEN, kPassRedo>(F, sh, ib, jl, bad, nullptr, plude_in,
                                                                       &kbud);
      } else {
        cloudsc_column<double, false, BUD, OPT, FT, GEN>(F, sh, ib, jl, active);
      }
    } else if constexpr (FAST) {
      typedef std::conditional_t<FORM == 2, float, double> Real;
      double plude_in[kMaxLevFast];
      bool bad = false;
      cloudsc_column<Real, FORM != 0, false, false, FT, GEN, kPassFast>(F, sh, ib, jl, active, &bad, plude_in);
      // The rerun takes the whole CTA (the column code holds a CTA barrier
      // at every level); only the columns that reported store anything.
      if (__syncthreads_or(bad))
        cloudsc_column<Real, FORM != 0, false, false, FT, GEN, kPassRedo>(F, sh, ib, jl, bad, nullptr, plude_in);
    } else {
      typedef std::conditional_t<FORM == 2, float, double> Real;
      cloudsc_column<Real, FORM != 0, false, false, FT, GEN>(F, sh, ib, jl, active);
    }
  }
}

// CLOUD_SATADJ: one thread per (column, level) point, points numbered
// (ib * KLEV + jk) * NPROMA + jl -- the element offset of a level field -- so
// consecutive threads read consecutive columns of one level (coalesced).  A
// grid-stride loop covers all points of all blocks; levels above NCLDTOP get
// zero tendencies (cloud_satadj.F90:338-345).  256-thread CTAs at 64
// registers (4 CTAs, 32 warps per SM) and up to 64 CTAs per SM in the grid:
// 2.42 ms at 262,144 columns, against 2.55 ms at 80 registers with 16 CTAs
// per SM and 2.61 ms at 48 registers.
// INC: STATE_INCREMENT of the cumulative tendencies fused in
// (callpar.F90:1278-1280): each point writes CML + LOC back into the CML
// arrays it has just read (inc_* not NULL), one addition each, as the
// separate call does.
constexpr int kSatadjThreads = 256;
template <bool INC>
__global__ void __launch_bounds__(kSatadjThreads, 4) satadj_kernel(SatadjFields F, Shape sh) {
  plibm_load_tables();
  const KParams<double> &k = KP<double>();
  const double dt = sh.ptsphy;
  const double zqtmst = 1.0 / dt;
  const unsigned long long np = sh.nproma, kl = sh.klev;
  const unsigned long long npts = (unsigned long long)sh.ngpblks * kl * np;
  const int jktop = k.ncldtop - 1;  // first 0-based level with cloud processes
  int nwarn = 0;
  for (unsigned long long idx = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; idx < npts;
       idx += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long row = idx / np;
    const int jl = (int)(idx - row * np);
    const unsigned long long ib = row / kl;
    const int jk = (int)(row - ib * kl);
    const long long icend = (long long)sh.ngptot - (long long)ib * (long long)np;
    if (jl < sh.kidia0 || jl >= icend) continue;
    if (jk < jktop) {
      F.loc_t[idx] = 0.0;
      F.loc_q[idx] = 0.0;
      F.loc_a[idx] = 0.0;
      F.loc_l[idx] = 0.0;
      F.loc_i[idx] = 0.0;
      if constexpr (INC) {  // + 0.0 as STATE_INCREMENT adds it (turns -0 into +0)
        if (F.inc_t) F.inc_t[idx] = F.inc_t[idx] + 0.0;
        if (F.inc_q) F.inc_q[idx] = F.inc_q[idx] + 0.0;
        if (F.inc_a) F.inc_a[idx] = F.inc_a[idx] + 0.0;
        if (F.inc_l) F.inc_l[idx] = F.inc_l[idx] + 0.0;
        if (F.inc_i) F.inc_i[idx] = F.inc_i[idx] + 0.0;
      }
      continue;
    }
    const size_t oh = (size_t)(ib * (kl + 1) + jk) * np + jl;  // PAPH(jl, jk)
    const size_t o4 = (size_t)(ib * 4 * kl + jk) * np + jl;     // PLUDELI(jl, jk, 1)
    const size_t sl = (size_t)kl * np;                          // one PLUDELI component
    double lt, lq, la, ll, li;
    // the cumulative tendencies are read through the read-only path only
    // when this kernel does not write them back
    const double ct = INC ? F.cml_t[idx] : ld(F.cml_t + idx), cq = INC ? F.cml_q[idx] : ld(F.cml_q + idx),
                 ca = INC ? F.cml_a[idx] : ld(F.cml_a + idx), cl = INC ? F.cml_l[idx] : ld(F.cml_l + idx),
                 ci = INC ? F.cml_i[idx] : ld(F.cml_i + idx);
    satadj_point(k, dt, zqtmst, ld(F.pap + idx), ld(F.paph + oh), ld(F.paph + oh + np),
                 ld(F.paph + (size_t)(ib * (kl + 1) + kl) * np + jl), ld(F.pt + idx), ld(F.pq + idx),
                 ld(F.pa + idx), ld(F.pl + idx), ld(F.pi + idx), ct, cq, ca, cl, ci, ld(F.phrsw + idx),
                 ld(F.phrlw + idx), ld(F.vdf_t + idx), ld(F.vdf_q + idx), ld(F.pludeli + o4 + 2 * sl),
                 ld(F.pludeli + o4 + 3 * sl), ld(F.pvervel + idx), lt, lq, la, ll, li, nwarn);
    F.loc_t[idx] = lt;
    F.loc_q[idx] = lq;
    F.loc_a[idx] = la;
    F.loc_l[idx] = ll;
    F.loc_i[idx] = li;
    if constexpr (INC) {
      if (F.inc_t) F.inc_t[idx] = ct + lt;
      if (F.inc_q) F.inc_q[idx] = cq + lq;
      if (F.inc_a) F.inc_a[idx] = ca + la;
      if (F.inc_l) F.inc_l[idx] = cl + ll;
      if (F.inc_i) F.inc_i[idx] = ci + li;
    }
  }
  if (nwarn && F.ncounters) atomic_add(F.ncounters, (uint32_t)nwarn);
}

// SLTEND's supersaturation adjustment (sltend.F90:380-410): one thread per
// (column, level) point on levels NCLDTOP..KLEV, numbered like satadj_kernel;
// the tendencies are updated in place and the diagnostics written where
// their pointers are not NULL.
__global__ void __launch_bounds__(kSatadjThreads, 4) sltend_supersat_kernel(SltendFields F, Shape sh) {
  plibm_load_tables();
  const KParams<double> &k = KP<double>();
  const double tsphy = sh.ptsphy;
  const double zrtsphy = 1.0 / tsphy;
  const unsigned long long np = sh.nproma, kl = sh.klev;
  const unsigned long long npts = (unsigned long long)sh.ngpblks * kl * np;
  const int jktop = k.ncldtop - 1;
  for (unsigned long long idx = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; idx < npts;
       idx += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long row = idx / np;
    const int jl = (int)(idx - row * np);
    const unsigned long long ib = row / kl;
    const int jk = (int)(row - ib * kl);
    const long long icend = (long long)sh.ngptot - (long long)ib * (long long)np;
    if (jl < sh.kidia0 || jl >= icend || jk < jktop) continue;
    const size_t oc = (size_t)(ib * 5 * kl + jk) * np + jl;  // PTENCLD(jl, jk, NCLDQL)
    const size_t sl = (size_t)kl * np;
    const double tent = F.ptent[idx], tenq = F.ptenq[idx], tena = F.ptena[idx];
    const double zt = ld(F.pt + idx) + tsphy * (ld(F.pcent + idx) + tent);
    const double zq = ld(F.pq + idx) + tsphy * (ld(F.pcenq + idx) + tenq);
    const double za = ld(F.pa + idx) + tsphy * (ld(F.pcena + idx) + tena);
    double ta, qa, aa, la, ia;
    supersatcheck_kft1(k, zt, zq, za, ld(F.prsf1 + idx), ta, qa, aa, la, ia);
    F.ptent[idx] = tent + ta * zrtsphy;
    F.ptenq[idx] = tenq + qa * zrtsphy;
    F.ptena[idx] = tena + aa * zrtsphy;
    F.ptencld[oc] = F.ptencld[oc] + la * zrtsphy;
    F.ptencld[oc + sl] = F.ptencld[oc + sl] + ia * zrtsphy;
    if (F.padja) F.padja[idx] = aa * zrtsphy;
    if (F.padjl) F.padjl[idx] = la * zrtsphy;
    if (F.padji) F.padji[idx] = ia * zrtsphy;
  }
}

// STATE_INCREMENT (state_increment.F90:42-103): one thread per (column,
// level) point, numbered like satadj_kernel, adds each of the n increments
// to its state field (coalesced: a warp covers 32 neighbouring columns of
// one level of every field).
__global__ void __launch_bounds__(kSatadjThreads) state_increment_kernel(IncFields F, Shape sh) {
  const unsigned long long np = sh.nproma, kl = sh.klev;
  const unsigned long long npts = (unsigned long long)sh.ngpblks * kl * np;
  for (unsigned long long idx = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; idx < npts;
       idx += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long row = idx / np;
    const int jl = (int)(idx - row * np);
    const unsigned long long ib = row / kl;
    const unsigned long long within = idx - ib * kl * np;  // jk * NPROMA + jl
    const long long icend = (long long)sh.ngptot - (long long)ib * (long long)np;
    if (jl < sh.kidia0 || jl >= icend) continue;
    for (int f = 0; f < F.n; ++f) {
      double *d = F.dst[f] + ib * F.dst_bs[f] + within;
      *d = *d + ld(F.src[f] + ib * F.src_bs[f] + within);
    }
  }
}

// The column kernels' fast division on n operand pairs: q[i] = fast_div(a[i],
// b[i]) and bad[i] = 1 where an operand fell outside its exact window (a
// column kernel then reruns the column with IEEE division).  A self-check of
// the division alone.
__global__ void __launch_bounds__(kSatadjThreads) division_check_kernel(const double *a, const double *b,
                                                                       long long n, double *q, int *bad) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    DivCheck dc;
    q[i] = fast_div(a[i], b[i], dc);
    bad[i] = dc.bad() ? 1 : 0;
  }
}

// fast_rcp on n divisors: y[i] and the window report bad[i].
__global__ void __launch_bounds__(kSatadjThreads) reciprocal_check_kernel(const double *b, long long n, double *y,
                                                                         int *bad) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    DivCheck dc;
    y[i] = fast_rcp(b[i], dc);
    bad[i] = dc.bad() ? 1 : 0;
  }
}

}  // namespace cloudsc

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace cloudsc {

// Whether the parameters allow the GEN kernels (gen_exponents_ok).
bool params_allow_gen(const cloudsc_params &p, const Derived &d) {
  KParams<double> kd;
  fill_kparams(p, d, kd);
  return gen_exponents_ok(kd);
}

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

// Compiled launch variants: the __launch_bounds__(MAXT, MINB) pairs the
// kernels are built with.  MAXT x MINB threads share an SM's 65,536
// registers, so each pair fixes the register budget per thread (and with it
// the spills) and the CTA size it is meant for; the autotuner picks a
// variant, a CTA size up to its MAXT and the persistence at run time.
// 448 columns per CTA fill 148 SMs 3.96 times at 262,144 columns; the
// (448, 1) bound gives them 144 registers (0.8 % faster than the 128 of a
// (512, 1) bound, same bits).  Earlier measurements at 262,144 columns, FP64:
// 384 columns per CTA at 168 registers 17.77 ms against 15.98 ms at 448;
// three 128-thread CTAs per SM 21.7 ms.
struct Variant {
  int maxt, minb;
};
constexpr Variant kVariants[] = {{640, 1}, {448, 1}, {384, 1}, {256, 1}, {256, 2}, {128, 3}};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);
constexpr int kDefaultVariant = 1;  // (448, 1), run with 448 columns per CTA

int num_variants() { return kNumVariants; }
int default_variant() { return kDefaultVariant; }
void variant_bounds(int v, int *maxt, int *minb) {
  *maxt = kVariants[v].maxt;
  *minb = kVariants[v].minb;
}

template <int FORM, bool GEN, bool FAST>
static const void *kernel_ptr_form(int v) {
  switch (v) {
    case 0: return (const void *)cloudsc_kernel<FORM, kVariants[0].maxt, kVariants[0].minb, Fields, GEN, FAST>;
    case 1: return (const void *)cloudsc_kernel<FORM, kVariants[1].maxt, kVariants[1].minb, Fields, GEN, FAST>;
    case 2: return (const void *)cloudsc_kernel<FORM, kVariants[2].maxt, kVariants[2].minb, Fields, GEN, FAST>;
    case 3: return (const void *)cloudsc_kernel<FORM, kVariants[3].maxt, kVariants[3].minb, Fields, GEN, FAST>;
    case 4: return (const void *)cloudsc_kernel<FORM, kVariants[4].maxt, kVariants[4].minb, Fields, GEN, FAST>;
    case 5: return (const void *)cloudsc_kernel<FORM, kVariants[5].maxt, kVariants[5].minb, Fields, GEN, FAST>;
    default: return nullptr;
  }
}
static_assert(kNumVariants == 6, "kernel_ptr_form lists every variant");
// Forms 0-2 exist in every variant with GEN and FAST (the parameters of every
// known configuration allow GEN); for parameters that do not, in the (448, 1)
// variant with FAST only; for KLEV above kMaxLevFast, in the (448, 1) variant
// without either (`launch` then runs that one, at most 448 columns per CTA).
// Forms 3-5 (budgets, SPP, inhomogeneity, aerosols) exist in the (448, 1)
// variant only, in the same three builds; every variant maps to it.
template <int FORM>
static const void *kernel_ptr_opt_form(bool gen, bool fast) {
  if (!fast) return (const void *)cloudsc_kernel<FORM, 448, 1, Fields, false, false>;
  if (!gen) return (const void *)cloudsc_kernel<FORM, 448, 1, Fields, false, true>;
  return (const void *)cloudsc_kernel<FORM, 448, 1, Fields, true, true>;
}
static const void *kernel_ptr(int precision, int v, bool gen, bool fast) {
  if (precision <= 2 && !fast) {
    switch (precision) {
      case 0: return (const void *)cloudsc_kernel<0, 448, 1, Fields, false, false>;
      case 1: return (const void *)cloudsc_kernel<1, 448, 1, Fields, false, false>;
      case 2: return (const void *)cloudsc_kernel<2, 448, 1, Fields, false, false>;
    }
  }
  if (!gen && precision <= 2) {
    switch (precision) {
      case 0: return (const void *)cloudsc_kernel<0, 448, 1, Fields, false, true>;
      case 1: return (const void *)cloudsc_kernel<1, 448, 1, Fields, false, true>;
      case 2: return (const void *)cloudsc_kernel<2, 448, 1, Fields, false, true>;
    }
  }
  switch (precision) {
    case 0: return kernel_ptr_form<0, true, true>(v);
    case 1: return kernel_ptr_form<1, true, true>(v);
    case 2: return kernel_ptr_form<2, true, true>(v);
    case 3: return kernel_ptr_opt_form<3>(gen, fast);
    case 4: return kernel_ptr_opt_form<4>(gen, fast);
    case 5: return kernel_ptr_opt_form<5>(gen, fast);
    default: return nullptr;
  }
}

// The single-precision interface's kernels: forms 0-2 in the two variants
// the tuned schedules use, (640, 1) and (448, 1), with GEN and FAST; in the
// (448, 1) variant with FAST only, and without either for KLEV above
// kMaxLevFast.  Other variants map to the (448, 1) kernel (see launch_sp).
template <int FORM>
static const void *kernel_ptr_sp_form(int v, bool gen, bool fast) {
  if (!fast) return (const void *)cloudsc_kernel<FORM, 448, 1, FieldsSP, false, false>;
  if (!gen) return (const void *)cloudsc_kernel<FORM, 448, 1, FieldsSP, false, true>;
  if (v == 0) return (const void *)cloudsc_kernel<FORM, 640, 1, FieldsSP, true, true>;
  return (const void *)cloudsc_kernel<FORM, 448, 1, FieldsSP, true, true>;
}
static const void *kernel_ptr_sp(int precision, int v, bool gen, bool fast) {
  switch (precision) {
    case 0: return kernel_ptr_sp_form<0>(v, gen, fast);
    case 1: return kernel_ptr_sp_form<1>(v, gen, fast);
    case 2: return kernel_ptr_sp_form<2>(v, gen, fast);
    default: return nullptr;
  }
}

// Registers and local (spill) bytes per thread of variant v (needs a device).
cudaError_t variant_attributes(int precision, int v, int *regs, int *local_bytes) {
  const void *k = kernel_ptr(precision, v, true, true);
  if (!k) return cudaErrorInvalidValue;
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, k);
  if (e != cudaSuccess) return e;
  *regs = a.numRegs;
  *local_bytes = (int)a.localSizeBytes;
  return cudaSuccess;
}

// The largest local memory (stack frame) per thread of any column kernel:
// the spill slots and the fast pass's copy of the PLUDE inputs.
cudaError_t max_local_bytes(size_t *out) {
  size_t m = 0;
  auto see = [&](const void *k) -> cudaError_t {
    if (!k) return cudaSuccess;
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, k);
    if (e == cudaSuccess && a.localSizeBytes > m) m = a.localSizeBytes;
    return e;
  };
  for (int v = 0; v < kNumVariants; ++v)
    for (int g = 0; g < 2; ++g)
      for (int f = 0; f < 2; ++f) {
        for (int prec = 0; prec <= 5; ++prec) {
          cudaError_t e = see(kernel_ptr(prec, v, g != 0, f != 0));
          if (e != cudaSuccess) return e;
        }
        for (int prec = 0; prec <= 2; ++prec) {
          cudaError_t e = see(kernel_ptr_sp(prec, v, g != 0, f != 0));
          if (e != cudaSuccess) return e;
        }
      }
  *out = m;
  return cudaSuccess;
}

// Launch variant v of the kernel: precision 0 = FP64, 1 = FP32-mixed,
// 2 = FP32 physics, 3-5 the FP64 forms with budgets / SPP and inhomogeneity;
// gen: the parameters allow the GEN kernels (forms 0-2 otherwise run the
// (448, 1) kernel without GEN, at most 448 columns per CTA, as they do for
// KLEV above kMaxLevFast; forms 3-5 always run a (448, 1) kernel).
cudaError_t launch(int precision, int v, const Fields &f, const Shape &sh, int threads, int grid,
                   cudaStream_t stream, bool gen) {
  const bool fast = sh.klev <= kMaxLevFast;
  if (v < 0 || v >= kNumVariants || threads > kVariants[v].maxt) return cudaErrorInvalidConfiguration;
  if ((!gen || !fast || precision > 2) && threads > 448) return cudaErrorInvalidConfiguration;
  const void *k = kernel_ptr(precision, v, gen, fast);
  if (!k) return cudaErrorInvalidValue;
  Fields fa = f;
  Shape sa = sh;
  void *args[] = {&fa, &sa};
  return cudaLaunchKernel(k, dim3(grid), dim3(threads), args, 0, stream);
}

// Launch form `precision` (0-2) of the single-precision interface with the
// schedule of variant v: variant 0 keeps its (640, 1) kernel; every other
// variant runs the (448, 1) kernel with at most 448 columns per CTA.
cudaError_t launch_sp(int precision, int v, const FieldsSP &f, const Shape &sh, int threads, int grid,
                      cudaStream_t stream, bool gen) {
  const bool fast = sh.klev <= kMaxLevFast;
  if (v < 0 || v >= kNumVariants || threads > kVariants[v].maxt) return cudaErrorInvalidConfiguration;
  if ((v != 0 || !gen || !fast) && threads > 448) return cudaErrorInvalidConfiguration;
  const void *k = kernel_ptr_sp(precision, v, gen, fast);
  if (!k) return cudaErrorInvalidValue;
  FieldsSP fa = f;
  Shape sa = sh;
  void *args[] = {&fa, &sa};
  return cudaLaunchKernel(k, dim3(grid), dim3(threads), args, 0, stream);
}

// Launch CLOUD_SATADJ over every point of the batched arrays: a grid of
// 256-thread CTAs, at most 64 per SM, striding over the points.
// With any inc_* pointer set, the form with the fused STATE_INCREMENT runs.
cudaError_t launch_satadj(const SatadjFields &f, const Shape &sh, cudaStream_t stream) {
  const unsigned long long npts = (unsigned long long)sh.ngpblks * sh.klev * sh.nproma;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  unsigned long long blocks = (npts + kSatadjThreads - 1) / kSatadjThreads;
  const unsigned long long cap = (unsigned long long)sms * 64;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  if (f.inc_t || f.inc_q || f.inc_a || f.inc_l || f.inc_i)
    satadj_kernel<true><<<(unsigned)blocks, kSatadjThreads, 0, stream>>>(f, sh);
  else
    satadj_kernel<false><<<(unsigned)blocks, kSatadjThreads, 0, stream>>>(f, sh);
  return cudaGetLastError();
}

// STATE_INCREMENT over every point: a grid of 256-thread CTAs, at most 16
// per SM, striding over the points.
cudaError_t launch_state_increment(const IncFields &f, const Shape &sh, cudaStream_t stream) {
  const unsigned long long npts = (unsigned long long)sh.ngpblks * sh.klev * sh.nproma;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  unsigned long long blocks = (npts + kSatadjThreads - 1) / kSatadjThreads;
  const unsigned long long cap = (unsigned long long)sms * 16;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  state_increment_kernel<<<(unsigned)blocks, kSatadjThreads, 0, stream>>>(f, sh);
  return cudaGetLastError();
}

cudaError_t launch_sltend_supersat(const SltendFields &f, const Shape &sh, cudaStream_t stream) {
  const unsigned long long npts = (unsigned long long)sh.ngpblks * sh.klev * sh.nproma;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  unsigned long long blocks = (npts + kSatadjThreads - 1) / kSatadjThreads;
  const unsigned long long cap = (unsigned long long)sms * 64;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  sltend_supersat_kernel<<<(unsigned)blocks, kSatadjThreads, 0, stream>>>(f, sh);
  return cudaGetLastError();
}

cudaError_t launch_division_check(const double *a, const double *b, long long n, double *q, int *bad,
                                  cudaStream_t stream) {
  long long blocks = (n + kSatadjThreads - 1) / kSatadjThreads;
  if (blocks > 148LL * 16) blocks = 148LL * 16;
  if (blocks < 1) blocks = 1;
  division_check_kernel<<<(unsigned)blocks, kSatadjThreads, 0, stream>>>(a, b, n, q, bad);
  return cudaGetLastError();
}

cudaError_t launch_reciprocal_check(const double *b, long long n, double *y, int *bad, cudaStream_t stream) {
  long long blocks = (n + kSatadjThreads - 1) / kSatadjThreads;
  if (blocks > 148LL * 16) blocks = 148LL * 16;
  if (blocks < 1) blocks = 1;
  reciprocal_check_kernel<<<(unsigned)blocks, kSatadjThreads, 0, stream>>>(b, n, y, bad);
  return cudaGetLastError();
}

}  // namespace cloudsc
