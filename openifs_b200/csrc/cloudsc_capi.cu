// C ABI of the B200 CLOUDSC implementation (declared in include/cloudsc_b200.h).
//
// Host-side responsibilities: the reference's constant set-up for standalone
// use (cloudsc_b200_params_default), parameter validation and upload to
// constant memory, argument checking with CLOUDSC's error conventions, and the
// three launch paths:
//   cloudsc_b200_batched       device pointers, one persistent launch;
//   cloudsc_b200_batched_host  host pointers, block chunks pipelined through
//                              H2D / compute / D2H on three streams;
//   cloudsc_b200_block         the per-NPROMA-block drop-in with host pointers;
// and the same two forms (device-pointer batched, per-block host) of
// CLOUD_SATADJ, the saturation adjustment that runs before CLOUDSC.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <mutex>
#include <string>
#include <vector>
#include "cloudsc_common.cuh"
#include "plibm.h"

namespace cloudsc {
cudaError_t upload_params(const cloudsc_params &p, const Derived &d);
int num_variants();
int default_variant();
void variant_bounds(int v, int *maxt, int *minb);
cudaError_t variant_attributes(int precision, int v, int *regs, int *local_bytes);
cudaError_t max_local_bytes(size_t *out);
cudaError_t launch(int precision, int v, const Fields &f, const Shape &sh, int threads, int grid,
                   cudaStream_t stream, bool gen);
bool params_allow_gen(const cloudsc_params &p, const Derived &d);
cudaError_t launch_satadj(const SatadjFields &f, const Shape &sh, cudaStream_t stream);
cudaError_t launch_sltend_supersat(const SltendFields &f, const Shape &sh, cudaStream_t stream);
cudaError_t launch_state_increment(const IncFields &f, const Shape &sh, cudaStream_t stream);
cudaError_t launch_division_check(const double *a, const double *b, long long n, double *q, int *bad,
                                  cudaStream_t stream);
cudaError_t launch_reciprocal_check(const double *b, long long n, double *y, int *bad, cudaStream_t stream);
cudaError_t launch_sp(int precision, int v, const FieldsSP &f, const Shape &sh, int threads, int grid,
                      cudaStream_t stream, bool gen);
}  // namespace cloudsc

using namespace cloudsc;

namespace {

thread_local std::string t_last_error;

std::mutex g_mu;
cloudsc_params g_params;
bool g_have_params = false;
bool g_gen = true;  // the uploaded parameters allow the GEN kernels
unsigned long long g_gen_count = 0;  // parameter uploads so far
constexpr int kMaxDev = 64;
unsigned long long g_dev_gen[kMaxDev] = {0};
// Launch schedule per precision (0 FP64, 1 FP32-mixed, 2 FP32 physics): compiled variant,
// columns per CTA, persistent CTAs per SM (0: one CTA per column tile).
struct Schedule {
  int variant, threads, ctas_per_sm;
};
Schedule g_sched[3] = {{default_variant(), 448, 0}, {default_variant(), 448, 0}, {default_variant(), 448, 0}};

// The fixed device array of cloudsc_b200_block_noalloc (see that entry).  It
// is the only device object of this file, so this file's device module --
// and with it the array's 16 MiB -- is loaded on a device when something
// first asks for the array's address.  ensure_params() does that when it
// uploads the parameters to a device, so the array is reserved at
// cloudsc_b200_setup (or at the first call on another device), not at the
// first cloudsc_b200_block_noalloc call.
constexpr size_t kNoAllocBytes = size_t(16) << 20;  // 16 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

int fail(int code, const char *what, cudaError_t e = cudaSuccess) {
  t_last_error = what;
  if (e != cudaSuccess) {
    t_last_error += ": ";
    t_last_error += cudaGetErrorString(e);
  }
  return code;
}

// After an error in an entry point that has queued copies or kernels on
// `streams`: wait for them, so that nothing still reads or writes the
// caller's host arrays once the call has returned.  Returns `rc`.
int drained(int rc, std::initializer_list<cudaStream_t> streams) {
  for (cudaStream_t st : streams) cudaStreamSynchronize(st);
  return rc;
}

// SPP, a cloud-inhomogeneity path or an aerosol switch that acts is on: the
// FP64 form with them runs.  (LAERLIQAUTOLSP and LAERLIQCOLL act only under
// IWARMRAIN = 1, cloudsc.F90:1985-1989, 2020-2023; IWARMRAIN is 3, :727, so
// those two change nothing and need no form of their own.)
bool opt_on(const cloudsc_params &p) {
  return p.lspp || p.lcloud_inhomog || p.lrad_cloud_inhomog || p.laericesed || p.laericeauto;
}

// Inputs of the SPP / inhomogeneity form: PGP2DSPP (KLON, NRFTOTAL) when a
// perturbation is on (its MP, and MP+1 for CLOUDINHOM, within NRFTOTAL),
// PGAW with an inhomogeneity path, PFSD with LRAD_CLOUD_INHOMOG.
int opt_args_ok(const cloudsc_params &p, const void *pgaw, const void *pgp2dspp, const void *pfsd,
                const void *pre_ice, const void *picrit_aer, const void *pnice) {
  if (p.laericesed && !pre_ice) return fail(CLOUDSC_E_NULL, "LAERICESED is on: PRE_ICE is required");
  if (p.laericeauto && (!picrit_aer || !pnice))
    return fail(CLOUDSC_E_NULL, "LAERICEAUTO is on: PICRIT_AER and PNICE are required");
  if (p.lspp)
    for (int n = 0; n < 8; ++n) {
      if (!p.spp_on[n]) continue;
      if (!pgp2dspp) return fail(CLOUDSC_E_NULL, "an SPP perturbation is on: PGP2DSPP is required");
      if (p.spp_mp[n] < 1 || p.spp_mp[n] + (n == CLOUDSC_SPP_CLOUDINHOM ? 1 : 0) > p.spp_nrftotal)
        return fail(CLOUDSC_E_SHAPE, "an SPP field pointer MP is outside 1..NRFTOTAL");
    }
  if ((p.lcloud_inhomog || p.lrad_cloud_inhomog) && !pgaw)
    return fail(CLOUDSC_E_NULL, "the cloud-inhomogeneity paths need PGAW");
  if (p.lrad_cloud_inhomog && !pfsd) return fail(CLOUDSC_E_NULL, "LRAD_CLOUD_INHOMOG writes PFSD");
  return CLOUDSC_OK;
}

// The cloud budget diagnostics (LCLDBUD*, cloudsc.F90:3832-4110) are on: the
// FP64 kernel form that writes PEXTRA runs.
bool budgets_on(const cloudsc_params &p) {
  return p.lcldbudc || p.lcldbudl || p.lcldbudi || p.lcldbudt || p.lcldbud_vertint;
}

// Arguments of the budget form, checked as the reference does (it ABORTs when
// KFLDX is too small, cloudsc.F90:3945-4106, or KLEV < 60 with the vertical
// integral, :3851, which writes level slots up to 83); an input a section
// that is on reads must not be NULL.
int budget_args_ok(const cloudsc_params &p, int klev, int kfldx, const void *pextra, const void *pvfa,
                   const void *pdyna, const void *pdynl, const void *pdyni, const void *pdyns,
                   const void *phrsw, const void *phrlw, const void *kctop, const void *kpbltype) {
  const int need = (p.lbud23 ? 26 : 0) + (p.lcldbud_vertint ? 1 : 0) + (p.lcldbudc ? 12 : 0) +
                   (p.lcldbudl ? 22 : 0) + (p.lcldbudi ? 20 : 0) + (p.lcldbudt ? 13 : 0);
  if (!pextra || kfldx < need)
    return fail(CLOUDSC_E_SHAPE, "the budget diagnostics need PEXTRA with enough fields (KFLDX)");
  if (p.lcldbud_vertint && klev < 84)
    return fail(CLOUDSC_E_SHAPE, "the vertical-integral budget writes PEXTRA levels up to 83");
  const bool ok = !((p.lcldbudc || p.lcldbud_vertint) && (!pvfa || !pdyna)) &&
                  !((p.lcldbudl || p.lcldbud_vertint) && !pdynl) &&
                  !((p.lcldbudi || p.lcldbud_vertint) && !pdyni) && !(p.lcldbud_vertint && !pdyns) &&
                  !(p.lcldbudt && (!phrsw || !phrlw)) && !(p.lcldbud_vertint && (!kctop || !kpbltype));
  if (!ok) return fail(CLOUDSC_E_NULL, "an input the budget diagnostics read is NULL");
  return CLOUDSC_OK;
}

Derived make_derived(const cloudsc_params &p) {
  Derived d;
  // ZCONST**RCL_KKBAUN (cloudsc.F90:2179-2181) takes one of two values; it is
  // evaluated once here with the kernels' own pow.
  d.zconst_pow_land = plibm_pow(p.rcl_kk_cloud_num_land, p.rcl_kkbaun);
  d.zconst_pow_sea = plibm_pow(p.rcl_kk_cloud_num_sea, p.rcl_kkbaun);
  d.flt_0p4 = (double)0.4f;
  d.flt_0p8 = (double)0.8f;
  return d;
}

// Make sure the current device holds the latest uploaded parameters.
int ensure_params(int *dev_out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "cudaGetDevice", e);
  if (dev < 0 || dev >= kMaxDev) return fail(CLOUDSC_E_CUDA, "device index out of range");
  if (dev_out) *dev_out = dev;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_have_params) return fail(CLOUDSC_E_PARAMS, "cloudsc_b200_setup has not been called");
  if (g_dev_gen[dev] != g_gen_count) {
    e = upload_params(g_params, make_derived(g_params));
    if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "parameter upload", e);
    // load this file's module (the no-allocation entry's fixed array) now
    void *scratch = nullptr;
    e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
    if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "cudaGetSymbolAddress(no-allocation array)", e);
    // Reserve the column kernels' local memory now, not at their first
    // launch: the driver sizes it as the per-thread stack times the threads
    // the device can hold (about half a GB on a B200 for a 2.6 KB frame), so
    // raise the stack limit to the largest kernel's frame (never lower it).
    size_t need = 0, cur = 0;
    e = max_local_bytes(&need);
    if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "cudaFuncGetAttributes(column kernels)", e);
    e = cudaDeviceGetLimit(&cur, cudaLimitStackSize);
    if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "cudaDeviceGetLimit(stack size)", e);
    if (cur < need) {
      e = cudaDeviceSetLimit(cudaLimitStackSize, need);
      if (e != cudaSuccess)
        return fail(CLOUDSC_E_CUDA, "reserving the column kernels' local memory (cudaDeviceSetLimit, stack size)", e);
    }
    g_dev_gen[dev] = g_gen_count;
  }
  return CLOUDSC_OK;
}

int check_params_match(const cloudsc_params *p) {
  if (!p) return fail(CLOUDSC_E_NULL, "params is NULL");
  if (p->magic != CLOUDSC_PARAMS_MAGIC) return fail(CLOUDSC_E_PARAMS, "bad params magic");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_have_params) return fail(CLOUDSC_E_PARAMS, "cloudsc_b200_setup has not been called");
  if (std::memcmp(p, &g_params, sizeof(cloudsc_params)) != 0)
    return fail(CLOUDSC_E_PARAMS, "params differ from the ones passed to cloudsc_b200_setup");
  return CLOUDSC_OK;
}

int grid_for(int ctas, int tiles) {
  if (ctas <= 0) return tiles;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int g = sms * ctas;
  return g < tiles ? g : tiles;
}

}  // namespace

extern "C" {

const char *cloudsc_b200_last_error(void) { return t_last_error.c_str(); }

const char *cloudsc_b200_version(void) { return "cloudsc_b200 1.0 (sm_100a)"; }

size_t cloudsc_b200_params_size(void) { return sizeof(cloudsc_params); }

// Restatement of the reference defaults (SUCLDP, SUPHEC, YOMCST, SUCUMF,
// SUECRAD, SU0PHY); see the header for the citations.  Gamma-function values
// use FCGENERALIZED_GAMMA's binary32 Lanczos coefficients
// (fcgeneralized_gamma.F90:69-126), as the reference does.
static double lanczos_gamma_f32coef(double px) {
  const float coef[6] = {76.18009172947146f, -86.50532032941677f, 24.01409824083091f,
                         -1.231739572450155f, 0.1208650973866179E-2f, -0.5395239384953E-5f};
  const double stp = (double)2.5066282746310005f;
  const double sercst = (double)1.000000000190015f;
  const double pi = 2.0 * std::asin(1.0);
  double w = px >= 0.0 ? 1.0 : 0.0;
  double x = (1.0 - px) * (1.0 - w) + px * w;
  double tt = x + 5.5;
  double lead = (x + 0.5) * std::log(tt) - tt;
  double ser = sercst;
  for (int j = 0; j < 6; ++j) ser = ser + (double)coef[j] / ((double)(j + 1) + x);
  double g = std::exp(lead + std::log(stp * ser / x));
  return g * w + (pi / std::sin(pi * px) / g) * (1.0 - w);
}

int cloudsc_b200_params_default(double tsphy, int32_t ncldtop, cloudsc_params *p) {
  if (!p) return fail(CLOUDSC_E_NULL, "params is NULL");
  if (!(tsphy > 0.0)) return fail(CLOUDSC_E_SHAPE, "tsphy must be positive");
  std::memset(p, 0, sizeof(*p));
  p->magic = CLOUDSC_PARAMS_MAGIC;
  p->version = 1;
  const double plrg = 1.0, pldare = 1.0, plradi = 1.0;  // sudyncore.F90:86-90
  const double pi = 2.0 * std::asin(1.0);
  // YOMCST
  const double rgas = 6.0221367E+23 * 1.380658E-23;  // RNAVO*RKBOL
  p->rpi = pi;
  p->ra = 6371229. * plradi;
  p->rg = 9.80665;
  p->rd = 1000. * rgas / 28.9644;
  p->rv = 1000. * rgas / 18.0153;
  p->rcpd = 3.5 * p->rd;
  p->retv = p->rv / p->rd - 1.0;
  p->rtt = 273.16;
  p->rlvtt = 2.5008E+6;
  p->rlstt = 2.8345E+6;
  p->rlmlt = p->rlstt - p->rlvtt;
  // YOETHF
  p->r2es = 611.21 * p->rd / p->rv;
  p->r3les = 17.502;
  p->r3ies = 22.587;
  p->r4les = 32.19;
  p->r4ies = -0.7;
  p->r5les = p->r3les * (p->rtt - p->r4les);
  p->r5ies = p->r3ies * (p->rtt - p->r4ies);
  p->r5alvcp = p->r5les * p->rlvtt / p->rcpd;
  p->r5alscp = p->r5ies * p->rlstt / p->rcpd;
  p->ralvdcp = p->rlvtt / p->rcpd;
  p->ralsdcp = p->rlstt / p->rcpd;
  p->ralfdcp = p->rlmlt / p->rcpd;
  p->rtwat = p->rtt;
  p->rtice = p->rtt - 23.;
  p->rticecu = p->rtt - 23.;
  p->rtwat_rtice_r = 1.0 / (p->rtwat - p->rtice);
  p->rtwat_rticecu_r = 1.0 / (p->rtwat - p->rticecu);
  p->rkoop1 = 2.583;
  p->rkoop2 = 0.48116E-2;
  // TECLDP scalars
  const double vplrg = pldare * std::sqrt(plrg);
  p->ramid = 0.8;
  p->rprc1 = 100.;
  p->ramin = 1.E-8;
  p->rlmin = 1.E-8;
  p->rcldiff = 6.0E-6 * plrg * pldare;
  p->rcldiff_convi = 10.0;
  p->rclcrit_sea = 2.5E-4;
  p->rclcrit_land = 5.5E-4;
  p->rkconv = plrg * pldare / 6000.;
  p->rcl_inhomogaut = 1.5;
  p->rcl_inhomogacc = 3.0;
  p->rsnowlin1 = plrg * pldare / 1000.;
  p->rsnowlin2 = 0.030;
  p->rlcritsnow = 2.0E-5;
  p->rvice = 0.13 * vplrg;
  p->rvrain = 4.0 * vplrg;
  p->rvsnow = 1.0 * vplrg;
  p->rxfallspeedrain = 1.0;
  p->rxfallspeedice = 1.0;
  p->ricehi1 = 1.0 / 30000.;
  p->ricehi2 = 1.0 / 233.;
  p->rnice = 0.027;
  p->rccn = 125.0;
  p->rcldtopcf = 0.01;
  p->rdepliqrefrate = 0.5;
  p->rdepliqrefdepth = 500.0 / plrg;
  p->rcl_overlapliqice = 0.65;
  p->rcl_effrime = 1.0;
  p->riceinit = 1.E-12;
  p->rthomo = p->rtt - 38.0;
  p->rprecrhmax = 0.7;
  p->rpecons = 5.44E-4 * plrg * pldare / p->rg;
  p->rvrfactor = 5.09E-3 * vplrg;
  p->rcovpmin = 0.1;
  p->rtaumel = 2.0 * 3.6E3 / (plrg * pldare);
  p->rkooptau = 3.0 * 3.6E3 / (plrg * pldare);
  p->rdenswat = 1000.0;
  p->rdensref = 1.0;
  // rain particle size distribution and process constants
  const double cr = 386.8 * vplrg, ar = p->rdenswat * pi / 6., br = 3.0, x4r = 0.0;
  const double fzrbb = 2.E2, schmidt = 0.6, dynvisc = 1.717E-5;
  p->rcl_dr = 0.67;
  p->rcl_x1r = 0.22;
  p->rcl_x2r = 2.20;
  p->rcl_lam1r = ar * p->rcl_x1r * lanczos_gamma_f32coef(br + 1. + x4r);
  p->rcl_lam2r = 1.0 / (br + 1. + x4r - p->rcl_x2r);
  p->rcl_cdenom1 = 5.57E11;
  p->rcl_cdenom2 = 1.03E8;
  p->rcl_cdenom3 = 2.04E2;
  p->rcl_ka273 = 2.4E-2;
  const double g1r = lanczos_gamma_f32coef((p->rcl_dr + 5.) / 2.);
  const double g3r = lanczos_gamma_f32coef(br + 1.0 + x4r);
  const double g4r = lanczos_gamma_f32coef(p->rcl_dr + br + 1.0 + x4r);
  const double g5r = lanczos_gamma_f32coef(3.0 + p->rcl_dr + x4r);
  const double g6r = lanczos_gamma_f32coef(4.0 + br + x4r);
  p->rcl_const1r = 2. * pi * p->rcl_x1r * plrg * pldare;
  p->rcl_const2r = 0.31 * std::pow(schmidt, 0.3333) * g1r * std::pow(cr / dynvisc, 0.5);
  p->rcl_const3r = (p->rcl_dr + 5.) / 2. - p->rcl_x2r;
  p->rcl_const4r = 2. - p->rcl_x2r;
  p->rcl_const7r = cr * g4r / g3r;
  p->rcl_const8r = 0.0;
  p->rcl_const9r = pi * 0.25 * p->rcl_x1r * cr * g5r;
  p->rcl_const10r = 3.0 + p->rcl_dr - p->rcl_x2r;
  p->rcl_eff_racw = 0.7;
  p->rcl_kkaac = 67.;
  p->rcl_kkbac = 1.15;
  p->rcl_kkaau = 1350.;
  p->rcl_kkbauq = 2.47;
  p->rcl_kkbaun = -1.79;
  p->rcl_kk_cloud_num_sea = 50.;
  p->rcl_kk_cloud_num_land = 300.;
  p->rcl_fzrab = -0.66;
  p->rcl_const5r = pi / (6.) * fzrbb * ar * p->rcl_x1r * g6r;
  p->rcl_const6r = -1. * (4. + br + x4r - p->rcl_x2r);
  // cloud ice (RCL_CI/RCL_DI are the Morrison-Gettelman overrides, sucldp.F90:456-457)
  const double ai = 0.069, bi = 2.0, ci = 100., di = 1.0, x1i = 2.0E6, x2i = 0.0, x4i = 0.0;
  const double g1i = lanczos_gamma_f32coef(bi + 1.0 + x4i);
  const double g2i = lanczos_gamma_f32coef(x4i + 2.0);
  const double g3i = lanczos_gamma_f32coef((di + 5.0 + 2.0 * x4i) / 2.0);
  const double g4i = lanczos_gamma_f32coef(di + bi + 1.0 + x4i);
  p->rcl_const1i = 1.0 / (ai * x1i * g1i);
  p->rcl_const2i = 1.0 * pi * x1i;
  p->rcl_const3i = 0.44 * std::pow(0.6, 1.0 / 3.0) * std::pow(ci, 0.5) * g3i / std::pow(1.717E-5, 0.5);
  p->rcl_const4i = (2.0 + x4i - x2i) / (bi + 1.0 + x4i - x2i);
  p->rcl_const5i = (5.0 + di + 2.0 * x4i - 2.0 * x2i) / (2.0 * (bi + 1. + x4i - x2i));
  p->rcl_const6i = g2i;
  p->rcl_const7i = ci * g4i / g1i;
  p->rcl_apb1 = 7.14E11;
  p->rcl_apb2 = 1.16E8;
  p->rcl_apb3 = 2.416E2;
  // snow
  const double as = 0.069, bs = 2.0, cs = 16.8 * vplrg, ds = 0.527, x2s = 0.0, x4s = 0.0;
  p->rcl_x1s = 2.0E6;
  const double g1s = lanczos_gamma_f32coef(bs + 1.0 + x4s);
  const double g2s = lanczos_gamma_f32coef(3.0 + ds + x4s);
  const double g3s = lanczos_gamma_f32coef((ds + 5.0 + 2.0 * x4s) / 2.0);
  const double g4s = lanczos_gamma_f32coef(x4s + 2.0);
  p->rcl_lam1s = as * p->rcl_x1s * lanczos_gamma_f32coef(bs + 1.0 + x4s);
  p->rcl_lam2s = 1.0 / (bs + 1. + x4s - x2s);
  p->rcl_const1s = 1.0 / (as * p->rcl_x1s * g1s);
  p->rcl_const2s = 1.0 * pi * p->rcl_x1s;
  p->rcl_const3s = 0.44 * std::pow(0.6, 1.0 / 3.0) * std::pow(cs, 0.5) * g3s / std::pow(1.717E-5, 0.5);
  p->rcl_const4s = (2.0 + x4s - x2s) / (bs + 1.0 + x4s - x2s);
  p->rcl_const5s = (5.0 + ds + 2.0 * x4s - 2.0 * x2s) / (2.0 * (bs + 1. + x4s - x2s));
  p->rcl_const6s = g4s;
  p->rcl_const7s = pi * 0.25 * p->rcl_x1s * cs * g2s;
  p->rcl_const8s = (3.0 + ds + x4s - x2s) / (bs + 1.0 + x4s - x2s);
  // switches and the remaining derived types
  p->ncldtop = ncldtop;
  p->lcldbud_timeint = 1;
  p->rssicefactor = std::fmin(tsphy / p->rkooptau, 1.0);
  p->lmfdsnow = 1;
  p->rmfadvw = 0.0;
  p->rmfadvwdd = 0.0;
  p->rcloud_frac_std = 1.0;
  return CLOUDSC_OK;
}

int32_t cloudsc_b200_ncldtop(int32_t klev, const double *stpre, double rcldtopp) {
  if (!stpre || klev < 2) return -1;
  int32_t nc = 2;
  for (int32_t jlev = klev; jlev >= 2; --jlev)
    if (stpre[jlev - 1] > rcldtopp) nc = jlev;
  return nc;
}

int cloudsc_b200_setup(const cloudsc_params *p) {
  if (!p) return fail(CLOUDSC_E_NULL, "params is NULL");
  if (p->magic != CLOUDSC_PARAMS_MAGIC || p->version != 1)
    return fail(CLOUDSC_E_PARAMS, "bad params magic or version");
  if (p->ncldtop < 2) return fail(CLOUDSC_E_SHAPE, "ncldtop must be >= 2");
  const bool gen = params_allow_gen(*p, make_derived(*p));
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_params = *p;
    g_have_params = true;
    g_gen = gen;
    ++g_gen_count;
  }
  return ensure_params(nullptr);
}

int cloudsc_b200_num_variants(void) { return num_variants(); }

int cloudsc_b200_variant_info(int32_t precision, int32_t variant, int32_t *max_threads, int32_t *min_ctas,
                              int32_t *regs, int32_t *local_bytes) {
  if (precision < 0 || precision > 2) return fail(CLOUDSC_E_SHAPE, "precision must be 0, 1 or 2");
  if (variant < 0 || variant >= num_variants()) return fail(CLOUDSC_E_SHAPE, "no such variant");
  int mt = 0, mb = 0, r = -1, l = -1;
  variant_bounds(variant, &mt, &mb);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0) {
    cudaError_t e = variant_attributes(precision, variant, &r, &l);
    if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "cudaFuncGetAttributes", e);
  } else {
    cudaGetLastError();  // no device: registers and local bytes stay -1
  }
  if (max_threads) *max_threads = mt;
  if (min_ctas) *min_ctas = mb;
  if (regs) *regs = r;
  if (local_bytes) *local_bytes = l;
  return CLOUDSC_OK;
}

int cloudsc_b200_set_schedule(int32_t precision, int32_t variant, int32_t threads_per_cta,
                              int32_t ctas_per_sm) {
  if (precision < 0 || precision > 2) return fail(CLOUDSC_E_SHAPE, "precision must be 0, 1 or 2");
  if (variant < 0 || variant >= num_variants()) return fail(CLOUDSC_E_SHAPE, "no such variant");
  int mt = 0, mb = 0;
  variant_bounds(variant, &mt, &mb);
  if (threads_per_cta < 32 || threads_per_cta > mt || threads_per_cta % 32)
    return fail(CLOUDSC_E_SHAPE, "threads_per_cta must be a multiple of 32, at least 32 and at most "
                                 "the variant's compiled limit");
  if (ctas_per_sm < 0 || ctas_per_sm > 32) return fail(CLOUDSC_E_SHAPE, "ctas_per_sm must be in [0,32]");
  std::lock_guard<std::mutex> lk(g_mu);
  g_sched[precision] = {variant, threads_per_cta, ctas_per_sm};
  return CLOUDSC_OK;
}

int cloudsc_b200_get_schedule(int32_t precision, int32_t *variant, int32_t *threads_per_cta,
                              int32_t *ctas_per_sm) {
  if (precision < 0 || precision > 2) return fail(CLOUDSC_E_SHAPE, "precision must be 0, 1 or 2");
  std::lock_guard<std::mutex> lk(g_mu);
  const Schedule sc = g_sched[precision];
  if (variant) *variant = sc.variant;
  if (threads_per_cta) *threads_per_cta = sc.threads;
  if (ctas_per_sm) *ctas_per_sm = sc.ctas_per_sm;
  return CLOUDSC_OK;
}

// The variant with the most registers per thread that still holds a CTA of
// threads_per_cta: the smallest compiled limit >= threads_per_cta among the
// one-CTA-per-SM variants.
int cloudsc_b200_set_launch(int32_t precision, int32_t threads_per_cta, int32_t ctas_per_sm) {
  if (precision < 0 || precision > 2) return fail(CLOUDSC_E_SHAPE, "precision must be 0, 1 or 2");
  int best = -1, best_mt = 1 << 30;
  for (int v = 0; v < num_variants(); ++v) {
    int mt = 0, mb = 0;
    variant_bounds(v, &mt, &mb);
    if (mb == 1 && mt >= threads_per_cta && mt < best_mt) {
      best = v;
      best_mt = mt;
    }
  }
  if (best < 0 || threads_per_cta < 32 || threads_per_cta % 32)
    return fail(CLOUDSC_E_SHAPE, "threads_per_cta must be a multiple of 32, at least 32 and at most "
                                 "the largest compiled limit");
  return cloudsc_b200_set_schedule(precision, best, threads_per_cta, ctas_per_sm);
}

// With the budget diagnostics on, the FP64 form that writes PEXTRA (kernel
// form 3, launched with the FP64 schedule) runs instead of the plain one.
static int launch_checked(int precision, const Fields &f, const Shape &sh, cudaStream_t stream) {
  // One snapshot of the schedule and the switches: the kernel form is chosen
  // from the same parameters whose arrays are checked here, even if another
  // thread calls cloudsc_b200_setup meanwhile.
  Schedule sc;
  bool bud = false, opt = false, need_gaw = false, need_spp = false, need_fsd = false, gen = true;
  bool need_re = false, need_icrit = false;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    sc = g_sched[precision];
    gen = g_gen;
    if (g_have_params) {
      bud = budgets_on(g_params);
      opt = opt_on(g_params);
      need_gaw = g_params.lcloud_inhomog || g_params.lrad_cloud_inhomog;
      need_fsd = g_params.lrad_cloud_inhomog;
      need_re = g_params.laericesed;
      need_icrit = g_params.laericeauto;
      if (g_params.lspp)
        for (int n = 0; n < 8; ++n) need_spp = need_spp || g_params.spp_on[n];
    }
  }
  int form = precision;
  if (bud || opt) {
    if (precision != 0)
      return fail(CLOUDSC_E_UNSUPPORTED,
                  "the budget diagnostics, SPP, the inhomogeneity paths and the aerosol switches are FP64 only");
    if (bud && !f.pextra)
      return fail(CLOUDSC_E_UNSUPPORTED, "the budget diagnostics need PEXTRA: use cloudsc_b200_batched_diag "
                                         "or cloudsc_b200_block");
    if ((need_gaw && !f.pgaw) || (need_spp && !f.pgp2dspp) || (need_fsd && !f.pfsd) || (need_re && !f.pre_ice) ||
        (need_icrit && (!f.picrit_aer || !f.pnice)))
      return fail(CLOUDSC_E_UNSUPPORTED, "SPP, the inhomogeneity paths and the aerosol switches need their "
                                         "arrays: use cloudsc_b200_batched_diag or cloudsc_b200_block");
    form = bud && opt ? 5 : (opt ? 4 : 3);
  }
  // parameters that rule out the GEN kernels, more than kMaxLevFast levels
  // and forms 3-5: a (448, 1) kernel, at most 448 columns per CTA
  const bool small = !gen || sh.klev > kMaxLevFast || form > 2;
  const int threads = (small && sc.threads > 448) ? 448 : sc.threads;
  const int tiles = (int)(((long long)sh.ngpblks * sh.nproma + threads - 1) / threads);
  const int grid = grid_for(sc.ctas_per_sm, tiles);
  cudaError_t e = launch(form, sc.variant, f, sh, threads, grid, stream, gen);
  if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "kernel launch", e);
  return CLOUDSC_OK;
}

int cloudsc_b200_batched(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot,
    double ptsphy, const double *pt, const double *pq, const double *ptendency_cml_t,
    const double *ptendency_cml_q, const double *ptendency_cml_a, const double *ptendency_cml_cld,
    double *ptendency_loc_t, double *ptendency_loc_q, double *ptendency_loc_a,
    double *ptendency_loc_cld, const double *pvfl, const double *pvfi, const double *pap,
    const double *paph, const double *plsm, const int32_t *ldcum, const int32_t *ktype,
    const double *peis, const double *plu, double *plude, const double *pludeli,
    const double *psnde, const double *pmfu, const double *pmfd, const double *pa,
    const double *pclv, double *pcovptot, double *prainfrac_toprfz, double *pfsqlf,
    double *pfsqif, double *pfcqnng, double *pfcqlng, double *pfsqrf, double *pfsqsf,
    double *pfcqrng, double *pfcqsng, double *pfsqltur, double *pfsqitur, double *pfplsl,
    double *pfplsn, double *pfhpsl, double *pfhpsn, uint32_t *ncounters, int32_t precision,
    void *stream) {
  int rc = check_params_match(p);
  if (rc) return rc;
  if (precision < 0 || precision > 2) return fail(CLOUDSC_E_SHAPE, "precision must be 0, 1 or 2");
  if (budgets_on(*p) || opt_on(*p))
    return fail(CLOUDSC_E_UNSUPPORTED, "budgets, SPP, the inhomogeneity paths and the aerosol switches: use cloudsc_b200_batched_diag "
                                       "or cloudsc_b200_block");
  if (nproma < 1 || klev < 2 || ngpblks < 1 || ngptot < 1 ||
      (long long)ngptot > (long long)nproma * ngpblks || ngptot <= (long long)nproma * (ngpblks - 1))
    return fail(CLOUDSC_E_SHAPE, "inconsistent NPROMA/KLEV/NGPBLKS/NGPTOT");
  if (p->ncldtop > klev) return fail(CLOUDSC_E_SHAPE, "NCLDTOP > KLEV");
  if (!(ptsphy > 0.0)) return fail(CLOUDSC_E_SHAPE, "PTSPHY must be positive");
  const void *req[] = {pt, pq, ptendency_cml_t, ptendency_cml_q, ptendency_cml_a, ptendency_cml_cld,
                       ptendency_loc_t, ptendency_loc_q, ptendency_loc_a, ptendency_loc_cld, pvfl,
                       pvfi, pap, paph, plsm, ldcum, ktype, peis, plu, plude, pludeli, psnde, pmfu,
                       pmfd, pa, pclv, pcovptot, prainfrac_toprfz, pfsqlf, pfsqif, pfcqnng, pfcqlng,
                       pfsqrf, pfsqsf, pfcqrng, pfcqsng, pfsqltur, pfsqitur, pfplsl, pfplsn, pfhpsl,
                       pfhpsn};
  for (const void *q : req)
    if (!q) return fail(CLOUDSC_E_NULL, "a required array pointer is NULL");
  rc = ensure_params(nullptr);
  if (rc) return rc;
  Fields f = {pt, pq, ptendency_cml_t, ptendency_cml_q, ptendency_cml_a, ptendency_cml_cld,
              ptendency_loc_t, ptendency_loc_q, ptendency_loc_a, ptendency_loc_cld, pvfl, pvfi,
              pap, paph, plsm, ldcum, ktype, peis, plu, plude, pludeli, psnde, pmfu, pmfd, pa,
              pclv, pcovptot, prainfrac_toprfz, pfsqlf, pfsqif, pfcqnng, pfcqlng, pfsqrf, pfsqsf,
              pfcqrng, pfcqsng, pfsqltur, pfsqitur, pfplsl, pfplsn, pfhpsl, pfhpsn, ncounters};
  Shape sh = {nproma, klev, ngpblks, ngptot, 0, ptsphy};
  return launch_checked(precision, f, sh, (cudaStream_t)stream);
}

int cloudsc_b200_batched_diag(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot,
    double ptsphy, const double *pt, const double *pq, const double *ptendency_cml_t,
    const double *ptendency_cml_q, const double *ptendency_cml_a, const double *ptendency_cml_cld,
    double *ptendency_loc_t, double *ptendency_loc_q, double *ptendency_loc_a,
    double *ptendency_loc_cld, const double *pvfl, const double *pvfi, const double *pap,
    const double *paph, const double *plsm, const int32_t *ldcum, const int32_t *ktype,
    const double *peis, const double *plu, double *plude, const double *pludeli,
    const double *psnde, const double *pmfu, const double *pmfd, const double *pa,
    const double *pclv, double *pcovptot, double *prainfrac_toprfz, double *pfsqlf,
    double *pfsqif, double *pfcqnng, double *pfcqlng, double *pfsqrf, double *pfsqsf,
    double *pfcqrng, double *pfcqsng, double *pfsqltur, double *pfsqitur, double *pfplsl,
    double *pfplsn, double *pfhpsl, double *pfhpsn, const double *pvfa, const double *pdyna,
    const double *pdynl, const double *pdyni, const double *pdyns, const double *phrsw,
    const double *phrlw, const double *pgaw, const int32_t *kctop, const int32_t *kpbltype,
    const double *pgp2dspp, const double *pre_ice, const double *picrit_aer, const double *pnice,
    double *pfsd, double *pextra, int32_t kfldx, uint32_t *ncounters, void *stream) {
  int rc = check_params_match(p);
  if (rc) return rc;
  if (nproma < 1 || klev < 2 || ngpblks < 1 || ngptot < 1 ||
      (long long)ngptot > (long long)nproma * ngpblks || ngptot <= (long long)nproma * (ngpblks - 1))
    return fail(CLOUDSC_E_SHAPE, "inconsistent NPROMA/KLEV/NGPBLKS/NGPTOT");
  if (p->ncldtop > klev) return fail(CLOUDSC_E_SHAPE, "NCLDTOP > KLEV");
  if (!(ptsphy > 0.0)) return fail(CLOUDSC_E_SHAPE, "PTSPHY must be positive");
  const void *req[] = {pt, pq, ptendency_cml_t, ptendency_cml_q, ptendency_cml_a, ptendency_cml_cld,
                       ptendency_loc_t, ptendency_loc_q, ptendency_loc_a, ptendency_loc_cld, pvfl,
                       pvfi, pap, paph, plsm, ldcum, ktype, peis, plu, plude, pludeli, psnde, pmfu,
                       pmfd, pa, pclv, pcovptot, prainfrac_toprfz, pfsqlf, pfsqif, pfcqnng, pfcqlng,
                       pfsqrf, pfsqsf, pfcqrng, pfcqsng, pfsqltur, pfsqitur, pfplsl, pfplsn, pfhpsl,
                       pfhpsn};
  for (const void *q : req)
    if (!q) return fail(CLOUDSC_E_NULL, "a required array pointer is NULL");
  if (budgets_on(*p)) {
    rc = budget_args_ok(*p, klev, kfldx, pextra, pvfa, pdyna, pdynl, pdyni, pdyns, phrsw, phrlw, kctop,
                        kpbltype);
    if (rc) return rc;
  }
  if (opt_on(*p)) {
    rc = opt_args_ok(*p, pgaw, pgp2dspp, pfsd, pre_ice, picrit_aer, pnice);
    if (rc) return rc;
  }
  rc = ensure_params(nullptr);
  if (rc) return rc;
  Fields f = {pt, pq, ptendency_cml_t, ptendency_cml_q, ptendency_cml_a, ptendency_cml_cld,
              ptendency_loc_t, ptendency_loc_q, ptendency_loc_a, ptendency_loc_cld, pvfl, pvfi,
              pap, paph, plsm, ldcum, ktype, peis, plu, plude, pludeli, psnde, pmfu, pmfd, pa,
              pclv, pcovptot, prainfrac_toprfz, pfsqlf, pfsqif, pfcqnng, pfcqlng, pfsqrf, pfsqsf,
              pfcqrng, pfcqsng, pfsqltur, pfsqitur, pfplsl, pfplsn, pfhpsl, pfhpsn, ncounters,
              pvfa, pdyna, pdynl, pdyni, pdyns, phrsw, phrlw, kctop, kpbltype, pextra, kfldx,
              pgaw, pgp2dspp, pfsd, p->spp_nrftotal, pre_ice, picrit_aer, pnice};
  Shape sh = {nproma, klev, ngpblks, ngptot, 0, ptsphy};
  return launch_checked(0, f, sh, (cudaStream_t)stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Host-pointer paths.  Device memory comes from a per-thread workspace that is
// grown on demand and kept until the thread exits, so repeated calls from the
// same OpenMP thread (EC_PHYS_DRV calls CLOUDSC once per block) allocate once.
// ---------------------------------------------------------------------------
namespace {

// Per-block sizes (in elements) of every array the kernel touches, in the
// order of the Fields struct.
struct Layout {
  size_t s1, s2, s2h;
  size_t n_in2 = 0;
};

enum Kind { K2, K3_5, K3_4, K3_2, KH, K1 };
struct Arr {
  Kind kind;
  bool in, out;  // copied to / from the device
};
// Fields order: pt, pq, cml_t, cml_q, cml_a, cml_cld, loc_t, loc_q, loc_a, loc_cld,
// pvfl, pvfi, pap, paph, plsm, ldcum, ktype, peis, plu, plude, pludeli, psnde, pmfu,
// pmfd, pa, pclv, pcovptot, prainfrac, 14 fluxes
const Arr kArrs[42] = {
    {K2, 1, 0},   {K2, 1, 0},   {K2, 1, 0},   {K2, 1, 0},   {K2, 1, 0},   {K3_5, 1, 0},
    {K2, 0, 1},   {K2, 0, 1},   {K2, 0, 1},   {K3_5, 0, 1}, {K2, 1, 0},   {K2, 1, 0},
    {K2, 1, 0},   {KH, 1, 0},   {K1, 1, 0},   {K1, 1, 0},   {K1, 1, 0},   {K1, 1, 0},
    {K2, 1, 0},   {K2, 1, 1},   {K3_4, 1, 0}, {K3_2, 1, 0}, {K2, 1, 0},   {K2, 1, 0},
    {K2, 1, 0},   {K3_5, 1, 0}, {K2, 0, 1},   {K1, 0, 1},   {KH, 0, 1},   {KH, 0, 1},
    {KH, 0, 1},   {KH, 0, 1},   {KH, 0, 1},   {KH, 0, 1},   {KH, 0, 1},   {KH, 0, 1},
    {KH, 0, 1},   {KH, 0, 1},   {KH, 0, 1},   {KH, 0, 1},   {KH, 0, 1},   {KH, 0, 1}};

size_t elems(Kind k, size_t np, size_t klev) {
  switch (k) {
    case K2: return np * klev;
    case K3_5: return np * klev * 5;
    case K3_4: return np * klev * 4;
    case K3_2: return np * klev * 2;
    case KH: return np * (klev + 1);
    default: return np;
  }
}
// rows of nproma elements per block (for strided column-range copies)
size_t rows(Kind k, size_t klev) { return elems(k, 1, klev); }
// Rows of array i that a call returns to the caller.  PTENDENCY_LOC_CLD's
// last species (NCLV) is never written by the reference (cloudsc.F90:971
// loops to NCLV-1) nor by the kernels, so only its first NCLV-1 species rows
// are copied back and the caller's NCLV slice is left as it was.
constexpr int kLocCld = 9;
size_t out_rows(int i, size_t klev) { return i == kLocCld ? 4 * klev : rows(kArrs[i].kind, klev); }
// Rows of input array i that the kernels read, from the start of each block's
// slab.  The species arrays are read only in part at the default
// configuration: PTENDENCY_CML_CLD and PCLV for species 1..NCLV-1
// (cloudsc.F90:995-999, vapour comes from PQ), PLUDELI for its first two
// components (liquid and ice detrainment, :1372-1373, :4265, :4280).  Only these rows cross
// PCIe; the device rows after them are never read.
constexpr int kCmlCld = 5, kPludeli = 20, kPclv = 25;
size_t in_rows(int i, size_t klev) {
  if (i == kCmlCld || i == kPclv) return 4 * klev;
  if (i == kPludeli) return 2 * klev;
  return rows(kArrs[i].kind, klev);
}
// Bytes of an element of array i: the integer arrays (LDCUM, KTYPE) 4, the
// real ones fb (8 in the double-precision interface, 4 in the single one).
size_t elem_size(int i, size_t fb = 8) { return (i == 15 || i == 16) ? 4 : fb; }
// Host-to-device copy of blocks b0 .. b0+nb-1 of input array i (the rows the
// kernels read) into a device slab of nb blocks.
cudaError_t copy_in(void *dst, const void *host, int i, size_t np, size_t kl, size_t b0, size_t nb,
                    cudaStream_t s, size_t fb = 8) {
  const size_t esz = elem_size(i, fb);
  const size_t per = elems(kArrs[i].kind, np, kl) * esz;  // one block's slab
  const size_t used = in_rows(i, kl) * np * esz;
  const char *src = (const char *)host + b0 * per;
  if (used == per) return cudaMemcpyAsync(dst, src, per * nb, cudaMemcpyHostToDevice, s);
  return cudaMemcpy2DAsync(dst, per, src, per, used, nb, cudaMemcpyHostToDevice, s);
}

struct Workspace {
  int dev = -1;
  char *buf = nullptr;
  size_t cap = 0;
  cudaStream_t st[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t ev_in[4], ev_done[4], ev_out[4];
  bool events = false;
  uint32_t *counter = nullptr;
  void release() {
    if (buf) cudaFree(buf);
    if (counter) cudaFree(counter);
    for (auto &s : st)
      if (s) cudaStreamDestroy(s);
    if (events)
      for (int i = 0; i < 4; ++i) {
        cudaEventDestroy(ev_in[i]);
        cudaEventDestroy(ev_done[i]);
        cudaEventDestroy(ev_out[i]);
      }
    buf = nullptr;
    counter = nullptr;
    cap = 0;
    for (auto &s : st) s = nullptr;
    events = false;
  }
  // Thread exit: release without touching a torn-down context.
  ~Workspace() { release(); }
  int prepare(int device, size_t bytes) {
    cudaError_t e;
    if (dev != device) {
      // a different device: release what this thread owns on the old one
      // (with the old device current), then start over on the new one
      if (dev >= 0) {
        cudaSetDevice(dev);
        release();
        cudaSetDevice(device);
      }
      dev = device;
    }
    if (!st[0])
      for (auto &s : st) {
        e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "cudaStreamCreate", e);
      }
    if (!events) {
      for (int i = 0; i < 4; ++i) {
        cudaEventCreateWithFlags(&ev_in[i], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&ev_done[i], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&ev_out[i], cudaEventDisableTiming);
      }
      events = true;
    }
    if (!counter) {
      e = cudaMalloc(&counter, 64);
      if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "cudaMalloc(counter)", e);
    }
    if (bytes > cap) {
      if (buf) cudaFree(buf);
      buf = nullptr;
      e = cudaMalloc(&buf, bytes);
      if (e != cudaSuccess) {
        cap = 0;
        return fail(CLOUDSC_E_CUDA, "cudaMalloc(workspace)", e);
      }
      cap = bytes;
    }
    return CLOUDSC_OK;
  }
};

thread_local Workspace t_ws;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Carve the device arrays of `nblk` blocks out of `base`; returns bytes used.
size_t carve(char *base, size_t np, size_t klev, size_t nblk, void *dptr[42], size_t fb = 8) {
  size_t off = 0;
  for (int i = 0; i < 42; ++i) {
    size_t esz = elem_size(i, fb);
    size_t n = elems(kArrs[i].kind, np, klev) * nblk * esz;
    if (dptr) dptr[i] = base ? base + off : nullptr;
    off += align256(n);
  }
  return off;
}

Fields fields_from(void *d[42], uint32_t *counter) {
  Fields f{};
  f.pt = (const double *)d[0]; f.pq = (const double *)d[1]; f.cml_t = (const double *)d[2];
  f.cml_q = (const double *)d[3]; f.cml_a = (const double *)d[4]; f.cml_cld = (const double *)d[5];
  f.loc_t = (double *)d[6]; f.loc_q = (double *)d[7]; f.loc_a = (double *)d[8]; f.loc_cld = (double *)d[9];
  f.pvfl = (const double *)d[10]; f.pvfi = (const double *)d[11]; f.pap = (const double *)d[12];
  f.paph = (const double *)d[13]; f.plsm = (const double *)d[14]; f.ldcum = (const int32_t *)d[15];
  f.ktype = (const int32_t *)d[16]; f.peis = (const double *)d[17]; f.plu = (const double *)d[18];
  f.plude = (double *)d[19]; f.pludeli = (const double *)d[20]; f.psnde = (const double *)d[21];
  f.pmfu = (const double *)d[22]; f.pmfd = (const double *)d[23]; f.pa = (const double *)d[24];
  f.pclv = (const double *)d[25]; f.pcovptot = (double *)d[26]; f.prainfrac_toprfz = (double *)d[27];
  f.pfsqlf = (double *)d[28]; f.pfsqif = (double *)d[29]; f.pfcqnng = (double *)d[30];
  f.pfcqlng = (double *)d[31]; f.pfsqrf = (double *)d[32]; f.pfsqsf = (double *)d[33];
  f.pfcqrng = (double *)d[34]; f.pfcqsng = (double *)d[35]; f.pfsqltur = (double *)d[36];
  f.pfsqitur = (double *)d[37]; f.pfplsl = (double *)d[38]; f.pfplsn = (double *)d[39];
  f.pfhpsl = (double *)d[40]; f.pfhpsn = (double *)d[41];
  f.ncounters = counter;
  return f;
}

FieldsSP fields_sp_from(void *d[42], uint32_t *counter) {
  FieldsSP f{};
  f.pt = (const float *)d[0]; f.pq = (const float *)d[1]; f.cml_t = (const float *)d[2];
  f.cml_q = (const float *)d[3]; f.cml_a = (const float *)d[4]; f.cml_cld = (const float *)d[5];
  f.loc_t = (float *)d[6]; f.loc_q = (float *)d[7]; f.loc_a = (float *)d[8]; f.loc_cld = (float *)d[9];
  f.pvfl = (const float *)d[10]; f.pvfi = (const float *)d[11]; f.pap = (const float *)d[12];
  f.paph = (const float *)d[13]; f.plsm = (const float *)d[14]; f.ldcum = (const int32_t *)d[15];
  f.ktype = (const int32_t *)d[16]; f.peis = (const float *)d[17]; f.plu = (const float *)d[18];
  f.plude = (float *)d[19]; f.pludeli = (const float *)d[20]; f.psnde = (const float *)d[21];
  f.pmfu = (const float *)d[22]; f.pmfd = (const float *)d[23]; f.pa = (const float *)d[24];
  f.pclv = (const float *)d[25]; f.pcovptot = (float *)d[26]; f.prainfrac_toprfz = (float *)d[27];
  f.pfsqlf = (float *)d[28]; f.pfsqif = (float *)d[29]; f.pfcqnng = (float *)d[30];
  f.pfcqlng = (float *)d[31]; f.pfsqrf = (float *)d[32]; f.pfsqsf = (float *)d[33];
  f.pfcqrng = (float *)d[34]; f.pfcqsng = (float *)d[35]; f.pfsqltur = (float *)d[36];
  f.pfsqitur = (float *)d[37]; f.pfplsl = (float *)d[38]; f.pfplsn = (float *)d[39];
  f.pfhpsl = (float *)d[40]; f.pfhpsn = (float *)d[41];
  f.ncounters = counter;
  return f;
}

// Launch the single-precision interface's kernel of `precision` with that
// precision's schedule.
int launch_sp_checked(int precision, const FieldsSP &f, const Shape &sh, cudaStream_t stream) {
  Schedule sc;
  bool gen = true;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    sc = g_sched[precision];
    gen = g_gen;
  }
  int threads = sc.threads;
  if ((sc.variant != 0 || !gen || sh.klev > kMaxLevFast) && threads > 448) threads = 448;
  const int tiles = (int)(((long long)sh.ngpblks * sh.nproma + threads - 1) / threads);
  const int grid = grid_for(sc.ctas_per_sm, tiles);
  cudaError_t e = launch_sp(precision, sc.variant, f, sh, threads, grid, stream, gen);
  if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "kernel launch", e);
  return CLOUDSC_OK;
}

// The host-pointer pipeline of cloudsc_b200_batched_host(_sp): chunks of
// blocks through three device slots, H2D on stream 0, the kernel on stream 1,
// D2H on stream 2; fb = bytes of a real element (8 or 4); `launch_fn(d, sh,
// stream)` launches the kernel on the slot's arrays d.
template <typename LaunchFn>
int host_pipeline(const void *host[42], int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot,
                  double ptsphy, int32_t chunk_blocks, size_t fb, LaunchFn launch_fn) {
  int dev = 0;
  int rc = ensure_params(&dev);
  if (rc) return rc;
  const size_t np = nproma, kl = klev;
  int cb = chunk_blocks > 0 ? chunk_blocks : 64;
  if (cb > ngpblks) cb = ngpblks;
  const int nslot = 3;
  const size_t slot_bytes = carve(nullptr, np, kl, cb, nullptr, fb);
  rc = t_ws.prepare(dev, slot_bytes * nslot);
  if (rc) return rc;
  cudaError_t e = cudaMemsetAsync(t_ws.counter, 0, sizeof(uint32_t), t_ws.st[1]);
  if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "cudaMemsetAsync", e);
  const int nchunk = (ngpblks + cb - 1) / cb;
  for (int c = 0; c < nchunk && e == cudaSuccess; ++c) {
    const int slot = c % nslot;
    const int b0 = c * cb, nb = (b0 + cb <= ngpblks) ? cb : ngpblks - b0;
    void *d[42];
    carve(t_ws.buf + slot * slot_bytes, np, kl, cb, d, fb);
    // the slot is free once its previous D2H has finished
    if (c >= nslot) e = cudaStreamWaitEvent(t_ws.st[0], t_ws.ev_out[slot], 0);
    for (int i = 0; i < 42 && e == cudaSuccess; ++i)
      if (kArrs[i].in) e = copy_in(d[i], host[i], i, np, kl, b0, nb, t_ws.st[0], fb);
    if (e == cudaSuccess) e = cudaEventRecord(t_ws.ev_in[slot], t_ws.st[0]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(t_ws.st[1], t_ws.ev_in[slot], 0);
    if (e != cudaSuccess) break;
    int ngptot_c = ngptot - b0 * nproma;
    if (ngptot_c > nb * nproma) ngptot_c = nb * nproma;
    Shape sh = {nproma, klev, nb, ngptot_c, 0, ptsphy};
    rc = launch_fn(d, sh, t_ws.st[1]);
    if (rc) return drained(rc, {t_ws.st[0], t_ws.st[1], t_ws.st[2]});
    e = cudaEventRecord(t_ws.ev_done[slot], t_ws.st[1]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(t_ws.st[2], t_ws.ev_done[slot], 0);
    // Whole blocks are copied back in one piece; a partial last block (columns
    // beyond NGPTOT) returns only its computed columns, leaving the padding
    // of the caller's array untouched as the reference does.
    const int icend_last = ngptot_c - (nb - 1) * nproma;
    const int nfull = (icend_last == nproma) ? nb : nb - 1;
    for (int i = 0; i < 42 && e == cudaSuccess; ++i) {
      if (!kArrs[i].out) continue;
      const size_t esz = elem_size(i, fb);
      size_t per = elems(kArrs[i].kind, np, kl) * esz;
      char *hb = (char *)host[i] + (size_t)b0 * per;
      if (nfull > 0 && i == kLocCld)
        e = cudaMemcpy2DAsync(hb, per, d[i], per, out_rows(i, kl) * np * esz, nfull, cudaMemcpyDeviceToHost,
                              t_ws.st[2]);
      else if (nfull > 0)
        e = cudaMemcpyAsync(hb, d[i], per * nfull, cudaMemcpyDeviceToHost, t_ws.st[2]);
      if (e == cudaSuccess && nfull < nb)
        e = cudaMemcpy2DAsync(hb + per * nfull, np * esz, (char *)d[i] + per * nfull, np * esz,
                              (size_t)icend_last * esz, out_rows(i, kl), cudaMemcpyDeviceToHost, t_ws.st[2]);
    }
    if (e == cudaSuccess) e = cudaEventRecord(t_ws.ev_out[slot], t_ws.st[2]);
  }
  uint32_t nwarn = 0;
  if (e == cudaSuccess) e = cudaStreamWaitEvent(t_ws.st[2], t_ws.ev_done[(nchunk - 1) % nslot], 0);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&nwarn, t_ws.counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, t_ws.st[2]);
  if (e == cudaSuccess) e = cudaStreamSynchronize(t_ws.st[2]);
  if (e != cudaSuccess)
    return drained(fail(CLOUDSC_E_CUDA, "pipelined host path", e), {t_ws.st[0], t_ws.st[1], t_ws.st[2]});
  return (int)nwarn;
}

// Argument checks shared by the batched entries of both interfaces.
int batched_args_ok(const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot,
                    double ptsphy, int32_t precision) {
  int rc = check_params_match(p);
  if (rc) return rc;
  if (precision < 0 || precision > 2) return fail(CLOUDSC_E_SHAPE, "precision must be 0, 1 or 2");
  if (budgets_on(*p) || opt_on(*p))
    return fail(CLOUDSC_E_UNSUPPORTED, "budgets, SPP, the inhomogeneity paths and the aerosol switches: use cloudsc_b200_block "
                                       "or cloudsc_b200_batched_diag");
  if (nproma < 1 || klev < 2 || ngpblks < 1 || ngptot < 1 ||
      (long long)ngptot > (long long)nproma * ngpblks || ngptot <= (long long)nproma * (ngpblks - 1))
    return fail(CLOUDSC_E_SHAPE, "inconsistent NPROMA/KLEV/NGPBLKS/NGPTOT");
  if (p->ncldtop > klev) return fail(CLOUDSC_E_SHAPE, "NCLDTOP > KLEV");
  if (!(ptsphy > 0.0)) return fail(CLOUDSC_E_SHAPE, "PTSPHY must be positive");
  return CLOUDSC_OK;
}

}  // namespace

extern "C" {

int cloudsc_b200_block(
    const cloudsc_params *p, int32_t kidia, int32_t kfdia, int32_t klon, int32_t klev,
    int32_t lddiag, double ptsphy, const double *pt, const double *pq,
    const double *ptendency_cml_t, const double *ptendency_cml_q, const double *ptendency_cml_a,
    const double *ptendency_cml_cld, double *ptendency_loc_t, double *ptendency_loc_q,
    double *ptendency_loc_a, double *ptendency_loc_cld, const double *pvfa, const double *pvfl,
    const double *pvfi, const double *pdyna, const double *pdynl, const double *pdyni,
    const double *pdynr, const double *pdyns, const double *phrsw, const double *phrlw,
    const double *pvervel, const double *pap, const double *paph, const double *pgeom,
    const double *plsm, const double *pgaw, const int32_t *ldcum, const int32_t *kctop,
    const int32_t *ktype, const int32_t *kpbltype, double *peis, const double *plu, double *plude,
    const double *pludeli, const double *psnde, const double *pmfu, const double *pmfd,
    const double *pgp2dspp, int32_t ldslphy, const double *pa, const double *pclv,
    const double *plcrit_aer, const double *picrit_aer, const double *pre_ice, const double *pccn,
    const double *pnice, double *pcovptot, double *pfsd, double *prainfrac_toprfz, double *pfsqlf,
    double *pfsqif, double *pfcqnng, double *pfcqlng, double *pfsqrf, double *pfsqsf,
    double *pfcqrng, double *pfcqsng, double *pfsqltur, double *pfsqitur, double *pfplsl,
    double *pfplsn, double *pfhpsl, double *pfhpsn, double *pextra, int32_t kfldx) {
  // PLCRIT_AER and PCCN are read only under IWARMRAIN = 1 (see opt_on)
  (void)lddiag; (void)pdynr; (void)pvervel; (void)pgeom; (void)ldslphy; (void)plcrit_aer; (void)pccn;
  int rc = check_params_match(p);
  if (rc) return rc;
  if (klon < 1 || klev < 2 || kidia < 1 || kfdia > klon || kidia > kfdia)
    return fail(CLOUDSC_E_SHAPE, "inconsistent KIDIA/KFDIA/KLON/KLEV");
  if (p->ncldtop > klev) return fail(CLOUDSC_E_SHAPE, "NCLDTOP > KLEV");
  if (!(ptsphy > 0.0)) return fail(CLOUDSC_E_SHAPE, "PTSPHY must be positive");
  const void *host[42] = {pt, pq, ptendency_cml_t, ptendency_cml_q, ptendency_cml_a, ptendency_cml_cld,
                          ptendency_loc_t, ptendency_loc_q, ptendency_loc_a, ptendency_loc_cld, pvfl,
                          pvfi, pap, paph, plsm, ldcum, ktype, peis, plu, plude, pludeli, psnde, pmfu,
                          pmfd, pa, pclv, pcovptot, prainfrac_toprfz, pfsqlf, pfsqif, pfcqnng, pfcqlng,
                          pfsqrf, pfsqsf, pfcqrng, pfcqsng, pfsqltur, pfsqitur, pfplsl, pfplsn, pfhpsl,
                          pfhpsn};
  for (const void *q : host)
    if (!q) return fail(CLOUDSC_E_NULL, "a required array pointer is NULL");
  const bool bud = budgets_on(*p), opt = opt_on(*p);
  if (bud) {
    rc = budget_args_ok(*p, klev, kfldx, pextra, pvfa, pdyna, pdynl, pdyni, pdyns, phrsw, phrlw, kctop,
                        kpbltype);
    if (rc) return rc;
  }
  if (opt) {
    rc = opt_args_ok(*p, pgaw, pgp2dspp, pfsd, pre_ice, picrit_aer, pnice);
    if (rc) return rc;
  }
  int dev = 0;
  rc = ensure_params(&dev);
  if (rc) return rc;
  const size_t np = klon, kl = klev;
  const size_t bytes = carve(nullptr, np, kl, 1, nullptr);
  // with the budget diagnostics: 7 level fields, 2 int columns and PEXTRA after the arrays
  const size_t s2b = np * kl * 8, nx = bud ? (size_t)kfldx : 0;
  const size_t base = (bytes + 255) / 256 * 256;
  const size_t extra = bud ? 7 * s2b + 2 * ((np * 4 + 255) / 256 * 256) + nx * s2b : 0;
  // with SPP / inhomogeneity / aerosol: PGAW, PGP2DSPP (KLON, NRFTOTAL),
  // PFSD, then PRE_ICE, PICRIT_AER, PNICE after that
  const size_t nrf = opt && p->lspp ? (size_t)p->spp_nrftotal : 0;
  const size_t gawb = (np * 8 + 255) / 256 * 256, sppb = (np * nrf * 8 + 255) / 256 * 256;
  const size_t extra2 = opt ? gawb + sppb + s2b + 3 * s2b : 0;
  rc = t_ws.prepare(dev, base + extra + extra2);
  if (rc) return rc;
  void *d[42];
  carve(t_ws.buf, np, kl, 1, d);
  cudaStream_t s = t_ws.st[0];
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 42 && e == cudaSuccess; ++i)
    if (kArrs[i].in) e = copy_in(d[i], host[i], i, np, kl, 0, 1, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(t_ws.counter, 0, sizeof(uint32_t), s);
  if (e != cudaSuccess) return drained(fail(CLOUDSC_E_CUDA, "host-to-device copy", e), {s});
  Fields f = fields_from(d, t_ws.counter);
  double *dx = nullptr;
  if (bud) {
    char *b = t_ws.buf + base;
    const double *lv[7] = {pvfa, pdyna, pdynl, pdyni, pdyns, phrsw, phrlw};
    const double **dst[7] = {&f.pvfa, &f.pdyna, &f.pdynl, &f.pdyni, &f.pdyns, &f.phrsw, &f.phrlw};
    for (int i = 0; i < 7 && e == cudaSuccess; ++i, b += s2b) {
      *dst[i] = lv[i] ? (const double *)b : nullptr;
      if (lv[i]) e = cudaMemcpyAsync(b, lv[i], s2b, cudaMemcpyHostToDevice, s);
    }
    const int32_t *iv[2] = {kctop, kpbltype};
    const int32_t **idst[2] = {&f.kctop, &f.kpbltype};
    for (int i = 0; i < 2 && e == cudaSuccess; ++i, b += (np * 4 + 255) / 256 * 256) {
      *idst[i] = iv[i] ? (const int32_t *)b : nullptr;
      if (iv[i]) e = cudaMemcpyAsync(b, iv[i], np * 4, cudaMemcpyHostToDevice, s);
    }
    dx = (double *)b;
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, pextra, nx * s2b, cudaMemcpyHostToDevice, s);
    f.pextra = dx;
    f.kfldx = kfldx;
    if (e != cudaSuccess) return drained(fail(CLOUDSC_E_CUDA, "host-to-device copy", e), {s});
  }
  double *dfsd = nullptr;
  if (opt) {
    char *b = t_ws.buf + base + extra;
    f.pgaw = pgaw ? (const double *)b : nullptr;
    if (pgaw) e = cudaMemcpyAsync(b, pgaw, np * 8, cudaMemcpyHostToDevice, s);
    b += gawb;
    f.pgp2dspp = (pgp2dspp && nrf) ? (const double *)b : nullptr;
    if (e == cudaSuccess && pgp2dspp && nrf) e = cudaMemcpyAsync(b, pgp2dspp, np * nrf * 8, cudaMemcpyHostToDevice, s);
    b += sppb;
    dfsd = pfsd ? (double *)b : nullptr;
    f.pfsd = dfsd;
    f.nrftotal = p->spp_nrftotal;
    b += s2b;
    const double *av[3] = {pre_ice, picrit_aer, pnice};
    const double **adst[3] = {&f.pre_ice, &f.picrit_aer, &f.pnice};
    for (int i = 0; i < 3 && e == cudaSuccess; ++i, b += s2b) {
      *adst[i] = av[i] ? (const double *)b : nullptr;
      if (av[i]) e = cudaMemcpyAsync(b, av[i], s2b, cudaMemcpyHostToDevice, s);
    }
    if (e != cudaSuccess) return drained(fail(CLOUDSC_E_CUDA, "host-to-device copy", e), {s});
  }
  Shape sh = {klon, klev, 1, kfdia, kidia - 1, ptsphy};
  rc = launch_checked(0, f, sh, s);
  if (rc) return drained(rc, {s});
  // copy back only columns KIDIA..KFDIA of every output row
  const size_t c0 = kidia - 1, ncol = kfdia - kidia + 1;
  for (int i = 0; i < 42 && e == cudaSuccess; ++i) {
    if (!kArrs[i].out) continue;
    size_t nrow = out_rows(i, kl);
    e = cudaMemcpy2DAsync((double *)host[i] + c0, np * 8, (double *)d[i] + c0, np * 8, ncol * 8, nrow,
                          cudaMemcpyDeviceToHost, s);
  }
  if (bud && e == cudaSuccess)  // PEXTRA(KIDIA:KFDIA, :, :)
    e = cudaMemcpy2DAsync(pextra + c0, np * 8, dx + c0, np * 8, ncol * 8, kl * nx, cudaMemcpyDeviceToHost, s);
  if (dfsd && e == cudaSuccess)  // PFSD(KIDIA:KFDIA, :)
    e = cudaMemcpy2DAsync(pfsd + c0, np * 8, dfsd + c0, np * 8, ncol * 8, kl, cudaMemcpyDeviceToHost, s);
  uint32_t nwarn = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&nwarn, t_ws.counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return drained(fail(CLOUDSC_E_CUDA, "device-to-host copy", e), {s});
  return (int)nwarn;
}

int cloudsc_b200_batched_host(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot,
    double ptsphy, const double *pt, const double *pq, const double *ptendency_cml_t,
    const double *ptendency_cml_q, const double *ptendency_cml_a, const double *ptendency_cml_cld,
    double *ptendency_loc_t, double *ptendency_loc_q, double *ptendency_loc_a,
    double *ptendency_loc_cld, const double *pvfl, const double *pvfi, const double *pap,
    const double *paph, const double *plsm, const int32_t *ldcum, const int32_t *ktype,
    const double *peis, const double *plu, double *plude, const double *pludeli,
    const double *psnde, const double *pmfu, const double *pmfd, const double *pa,
    const double *pclv, double *pcovptot, double *prainfrac_toprfz, double *pfsqlf,
    double *pfsqif, double *pfcqnng, double *pfcqlng, double *pfsqrf, double *pfsqsf,
    double *pfcqrng, double *pfcqsng, double *pfsqltur, double *pfsqitur, double *pfplsl,
    double *pfplsn, double *pfhpsl, double *pfhpsn, int32_t precision, int32_t chunk_blocks) {
  int rc = batched_args_ok(p, nproma, klev, ngpblks, ngptot, ptsphy, precision);
  if (rc) return rc;
  const void *host[42] = {pt, pq, ptendency_cml_t, ptendency_cml_q, ptendency_cml_a, ptendency_cml_cld,
                          ptendency_loc_t, ptendency_loc_q, ptendency_loc_a, ptendency_loc_cld, pvfl,
                          pvfi, pap, paph, plsm, ldcum, ktype, peis, plu, plude, pludeli, psnde, pmfu,
                          pmfd, pa, pclv, pcovptot, prainfrac_toprfz, pfsqlf, pfsqif, pfcqnng, pfcqlng,
                          pfsqrf, pfsqsf, pfcqrng, pfcqsng, pfsqltur, pfsqitur, pfplsl, pfplsn, pfhpsl,
                          pfhpsn};
  for (const void *q : host)
    if (!q) return fail(CLOUDSC_E_NULL, "a required array pointer is NULL");
  return host_pipeline(host, nproma, klev, ngpblks, ngptot, ptsphy, chunk_blocks, 8,
                       [&](void *d[42], const Shape &sh, cudaStream_t st) {
                         return launch_checked(precision, fields_from(d, t_ws.counter), sh, st);
                       });
}

// The single-precision interface (JPRB = REAL(4)), device pointers.
int cloudsc_b200_batched_sp(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot, float ptsphy,
    const float *pt, const float *pq, const float *ptendency_cml_t, const float *ptendency_cml_q,
    const float *ptendency_cml_a, const float *ptendency_cml_cld, float *ptendency_loc_t,
    float *ptendency_loc_q, float *ptendency_loc_a, float *ptendency_loc_cld, const float *pvfl,
    const float *pvfi, const float *pap, const float *paph, const float *plsm, const int32_t *ldcum,
    const int32_t *ktype, const float *peis, const float *plu, float *plude, const float *pludeli,
    const float *psnde, const float *pmfu, const float *pmfd, const float *pa, const float *pclv,
    float *pcovptot, float *prainfrac_toprfz, float *pfsqlf, float *pfsqif, float *pfcqnng, float *pfcqlng,
    float *pfsqrf, float *pfsqsf, float *pfcqrng, float *pfcqsng, float *pfsqltur, float *pfsqitur,
    float *pfplsl, float *pfplsn, float *pfhpsl, float *pfhpsn, uint32_t *ncounters, int32_t precision,
    void *stream) {
  int rc = batched_args_ok(p, nproma, klev, ngpblks, ngptot, ptsphy, precision);
  if (rc) return rc;
  void *d[42] = {(void *)pt, (void *)pq, (void *)ptendency_cml_t, (void *)ptendency_cml_q,
                 (void *)ptendency_cml_a, (void *)ptendency_cml_cld, ptendency_loc_t, ptendency_loc_q,
                 ptendency_loc_a, ptendency_loc_cld, (void *)pvfl, (void *)pvfi, (void *)pap, (void *)paph,
                 (void *)plsm, (void *)ldcum, (void *)ktype, (void *)peis, (void *)plu, plude,
                 (void *)pludeli, (void *)psnde, (void *)pmfu, (void *)pmfd, (void *)pa, (void *)pclv,
                 pcovptot, prainfrac_toprfz, pfsqlf, pfsqif, pfcqnng, pfcqlng, pfsqrf, pfsqsf, pfcqrng,
                 pfcqsng, pfsqltur, pfsqitur, pfplsl, pfplsn, pfhpsl, pfhpsn};
  for (void *q : d)
    if (!q) return fail(CLOUDSC_E_NULL, "a required array pointer is NULL");
  rc = ensure_params(nullptr);
  if (rc) return rc;
  Shape sh = {nproma, klev, ngpblks, ngptot, 0, (double)ptsphy};
  return launch_sp_checked(precision, fields_sp_from(d, ncounters), sh, (cudaStream_t)stream);
}

// The single-precision interface, host pointers, pipelined like
// cloudsc_b200_batched_host (half the bytes cross PCIe).
int cloudsc_b200_batched_host_sp(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot, float ptsphy,
    const float *pt, const float *pq, const float *ptendency_cml_t, const float *ptendency_cml_q,
    const float *ptendency_cml_a, const float *ptendency_cml_cld, float *ptendency_loc_t,
    float *ptendency_loc_q, float *ptendency_loc_a, float *ptendency_loc_cld, const float *pvfl,
    const float *pvfi, const float *pap, const float *paph, const float *plsm, const int32_t *ldcum,
    const int32_t *ktype, const float *peis, const float *plu, float *plude, const float *pludeli,
    const float *psnde, const float *pmfu, const float *pmfd, const float *pa, const float *pclv,
    float *pcovptot, float *prainfrac_toprfz, float *pfsqlf, float *pfsqif, float *pfcqnng, float *pfcqlng,
    float *pfsqrf, float *pfsqsf, float *pfcqrng, float *pfcqsng, float *pfsqltur, float *pfsqitur,
    float *pfplsl, float *pfplsn, float *pfhpsl, float *pfhpsn, int32_t precision, int32_t chunk_blocks) {
  int rc = batched_args_ok(p, nproma, klev, ngpblks, ngptot, ptsphy, precision);
  if (rc) return rc;
  const void *host[42] = {pt, pq, ptendency_cml_t, ptendency_cml_q, ptendency_cml_a, ptendency_cml_cld,
                          ptendency_loc_t, ptendency_loc_q, ptendency_loc_a, ptendency_loc_cld, pvfl,
                          pvfi, pap, paph, plsm, ldcum, ktype, peis, plu, plude, pludeli, psnde, pmfu,
                          pmfd, pa, pclv, pcovptot, prainfrac_toprfz, pfsqlf, pfsqif, pfcqnng, pfcqlng,
                          pfsqrf, pfsqsf, pfcqrng, pfcqsng, pfsqltur, pfsqitur, pfplsl, pfplsn, pfhpsl,
                          pfhpsn};
  for (const void *q : host)
    if (!q) return fail(CLOUDSC_E_NULL, "a required array pointer is NULL");
  return host_pipeline(host, nproma, klev, ngpblks, ngptot, (double)ptsphy, chunk_blocks, 4,
                       [&](void *d[42], const Shape &sh, cudaStream_t st) {
                         return launch_sp_checked(precision, fields_sp_from(d, t_ws.counter), sh, st);
                       });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// cloudsc_b200_block_noalloc: the per-block drop-in without any device
// allocation.  Its device memory is one file-scope array, g_noalloc_scratch,
// of kNoAllocBytes, shared by every call in the process.  The array is
// reserved on a device when cloudsc_b200_setup (or the first call of any
// entry on that device) uploads the parameters there; every call looks its
// device address up again with cudaGetSymbolAddress (cheap, and never stale
// after a context reset).  Calls are serialised by g_noalloc_mu (the array
// holds one block at a time).  After a call returns, the array still holds
// that call's inputs and outputs until the next call overwrites them.
// ---------------------------------------------------------------------------
namespace {

std::mutex g_noalloc_mu;

}  // namespace

extern "C" {

size_t cloudsc_b200_block_noalloc_capacity(void) { return kNoAllocBytes; }

int cloudsc_b200_block_noalloc(
    const cloudsc_params *p, int32_t kidia, int32_t kfdia, int32_t klon, int32_t klev,
    double ptsphy, const double *pt, const double *pq, const double *ptendency_cml_t,
    const double *ptendency_cml_q, const double *ptendency_cml_a, const double *ptendency_cml_cld,
    double *ptendency_loc_t, double *ptendency_loc_q, double *ptendency_loc_a,
    double *ptendency_loc_cld, const double *pvfl, const double *pvfi, const double *pap,
    const double *paph, const double *plsm, const int32_t *ldcum, const int32_t *ktype,
    const double *peis, const double *plu, double *plude, const double *pludeli,
    const double *psnde, const double *pmfu, const double *pmfd, const double *pa,
    const double *pclv, double *pcovptot, double *prainfrac_toprfz, double *pfsqlf,
    double *pfsqif, double *pfcqnng, double *pfcqlng, double *pfsqrf, double *pfsqsf,
    double *pfcqrng, double *pfcqsng, double *pfsqltur, double *pfsqitur, double *pfplsl,
    double *pfplsn, double *pfhpsl, double *pfhpsn, void *stream) {
  int rc = check_params_match(p);
  if (rc) return rc;
  if (budgets_on(*p) || opt_on(*p))
    return fail(CLOUDSC_E_UNSUPPORTED, "budgets, SPP, the inhomogeneity paths and the aerosol switches: use cloudsc_b200_block "
                                       "or cloudsc_b200_batched_diag");
  if (klon < 1 || klev < 2 || kidia < 1 || kfdia > klon || kidia > kfdia)
    return fail(CLOUDSC_E_SHAPE, "inconsistent KIDIA/KFDIA/KLON/KLEV");
  if (p->ncldtop > klev) return fail(CLOUDSC_E_SHAPE, "NCLDTOP > KLEV");
  if (!(ptsphy > 0.0)) return fail(CLOUDSC_E_SHAPE, "PTSPHY must be positive");
  const void *host[42] = {pt, pq, ptendency_cml_t, ptendency_cml_q, ptendency_cml_a, ptendency_cml_cld,
                          ptendency_loc_t, ptendency_loc_q, ptendency_loc_a, ptendency_loc_cld, pvfl,
                          pvfi, pap, paph, plsm, ldcum, ktype, peis, plu, plude, pludeli, psnde, pmfu,
                          pmfd, pa, pclv, pcovptot, prainfrac_toprfz, pfsqlf, pfsqif, pfcqnng, pfcqlng,
                          pfsqrf, pfsqsf, pfcqrng, pfcqsng, pfsqltur, pfsqitur, pfplsl, pfplsn, pfhpsl,
                          pfhpsn};
  for (const void *q : host)
    if (!q) return fail(CLOUDSC_E_NULL, "a required array pointer is NULL");
  const size_t np = klon, kl = klev;
  // the first 256 bytes hold the warning counter, the arrays follow
  const size_t need = 256 + carve(nullptr, np, kl, 1, nullptr);
  if (need > kNoAllocBytes) {
    t_last_error = "cloudsc_b200_block_noalloc: this block needs " + std::to_string(need) +
                   " bytes of device scratch, the fixed array holds " + std::to_string(kNoAllocBytes) +
                   " (reduce KLON or use cloudsc_b200_block)";
    return CLOUDSC_E_TOO_LARGE;
  }
  rc = ensure_params(nullptr);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  void *scratch = nullptr;
  {
    cudaError_t e = cudaGetSymbolAddress(&scratch, g_noalloc_scratch);
    if (e != cudaSuccess || !scratch) return fail(CLOUDSC_E_CUDA, "cudaGetSymbolAddress(scratch)", e);
  }
  char *base = (char *)scratch;
  uint32_t *counter = (uint32_t *)base;
  void *d[42];
  carve(base + 256, np, kl, 1, d);
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 42 && e == cudaSuccess; ++i)
    if (kArrs[i].in) e = copy_in(d[i], host[i], i, np, kl, 0, 1, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
  if (e != cudaSuccess) return drained(fail(CLOUDSC_E_CUDA, "host-to-device copy", e), {s});
  Fields f = fields_from(d, counter);
  Shape sh = {klon, klev, 1, kfdia, kidia - 1, ptsphy};
  rc = launch_checked(0, f, sh, s);
  if (rc) return drained(rc, {s});
  const size_t c0 = kidia - 1, ncol = kfdia - kidia + 1;
  for (int i = 0; i < 42 && e == cudaSuccess; ++i) {
    if (!kArrs[i].out) continue;
    size_t nrow = out_rows(i, kl);
    e = cudaMemcpy2DAsync((double *)host[i] + c0, np * 8, (double *)d[i] + c0, np * 8, ncol * 8, nrow,
                          cudaMemcpyDeviceToHost, s);
  }
  uint32_t nwarn = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&nwarn, counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return drained(fail(CLOUDSC_E_CUDA, "device-to-host copy", e), {s});
  return (int)nwarn;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// CLOUD_SATADJ entry points (cloud_satadj.F90:13-26).
// ---------------------------------------------------------------------------
namespace {

int satadj_shape_ok(const cloudsc_params *p, double ptsphy) {
  int rc = check_params_match(p);
  if (rc) return rc;
  if (!(ptsphy > 0.0)) return fail(CLOUDSC_E_SHAPE, "PTSPHY must be positive");
  return CLOUDSC_OK;
}

}  // namespace

extern "C" {

int cloudsc_b200_satadj_batched(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot, double ptsphy,
    const double *pap, const double *paph, const double *pt, const double *pq, const double *pa,
    const double *pl, const double *pi, const double *ptendency_cml_t, const double *ptendency_cml_q,
    const double *ptendency_cml_a, const double *ptendency_cml_l, const double *ptendency_cml_i,
    const double *phrsw, const double *phrlw, const double *ptendency_vdf_t,
    const double *ptendency_vdf_q, const double *pludeli, const double *pvervel,
    double *ptendency_loc_t, double *ptendency_loc_q, double *ptendency_loc_a,
    double *ptendency_loc_l, double *ptendency_loc_i, uint32_t *ncounters, void *stream) {
  int rc = satadj_shape_ok(p, ptsphy);
  if (rc) return rc;
  if (nproma < 1 || klev < 2 || ngpblks < 1 || ngptot < 1 ||
      (long long)ngptot > (long long)nproma * ngpblks || ngptot <= (long long)nproma * (ngpblks - 1))
    return fail(CLOUDSC_E_SHAPE, "inconsistent NPROMA/KLEV/NGPBLKS/NGPTOT");
  if (p->ncldtop > klev) return fail(CLOUDSC_E_SHAPE, "NCLDTOP > KLEV");
  const void *req[] = {pap, paph, pt, pq, pa, pl, pi, ptendency_cml_t, ptendency_cml_q, ptendency_cml_a,
                       ptendency_cml_l, ptendency_cml_i, phrsw, phrlw, ptendency_vdf_t, ptendency_vdf_q,
                       pludeli, pvervel, ptendency_loc_t, ptendency_loc_q, ptendency_loc_a,
                       ptendency_loc_l, ptendency_loc_i};
  for (const void *q : req)
    if (!q) return fail(CLOUDSC_E_NULL, "a required array pointer is NULL");
  rc = ensure_params(nullptr);
  if (rc) return rc;
  SatadjFields f = {pap, paph, pt, pq, pa, pl, pi, ptendency_cml_t, ptendency_cml_q, ptendency_cml_a,
                    ptendency_cml_l, ptendency_cml_i, phrsw, phrlw, ptendency_vdf_t, ptendency_vdf_q,
                    pludeli, pvervel, ptendency_loc_t, ptendency_loc_q, ptendency_loc_a, ptendency_loc_l,
                    ptendency_loc_i, ncounters};
  Shape sh = {nproma, klev, ngpblks, ngptot, 0, ptsphy};
  cudaError_t e = launch_satadj(f, sh, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "kernel launch", e);
  return CLOUDSC_OK;
}

int cloudsc_b200_satadj_block(
    const cloudsc_params *p, int32_t kidia, int32_t kfdia, int32_t klon, int32_t klev, const int32_t *ktype,
    int32_t lddiag, double ptsphy, const double *pap, const double *paph, const double *pt,
    const double *pq, const double *pa, const double *pl, const double *pi,
    const double *ptendency_cml_t, const double *ptendency_cml_q, const double *ptendency_cml_a,
    const double *ptendency_cml_l, const double *ptendency_cml_i, const double *phrsw,
    const double *phrlw, const double *ptendency_vdf_t, const double *ptendency_vdf_q,
    const double *pmfu, const double *pmfd, const double *pludeli, const double *pvervel,
    const double *pgp2dspp, double *ptendency_loc_t, double *ptendency_loc_q,
    double *ptendency_loc_a, double *ptendency_loc_l, double *ptendency_loc_i, double *pextra,
    int32_t kfldx) {
  (void)ktype; (void)lddiag; (void)pmfu; (void)pmfd; (void)pgp2dspp; (void)pextra; (void)kfldx;
  int rc = satadj_shape_ok(p, ptsphy);
  if (rc) return rc;
  if (klon < 1 || klev < 2 || kidia < 1 || kfdia > klon || kidia > kfdia)
    return fail(CLOUDSC_E_SHAPE, "inconsistent KIDIA/KFDIA/KLON/KLEV");
  if (p->ncldtop > klev) return fail(CLOUDSC_E_SHAPE, "NCLDTOP > KLEV");
  // inputs in the order of SatadjFields; PLUDELI is copied for its components
  // 3 and 4 only (the ones the scheme reads, :407, :411)
  const double *in[18] = {pap, paph, pt, pq, pa, pl, pi, ptendency_cml_t, ptendency_cml_q,
                          ptendency_cml_a, ptendency_cml_l, ptendency_cml_i, phrsw, phrlw,
                          ptendency_vdf_t, ptendency_vdf_q, pludeli, pvervel};
  double *out[5] = {ptendency_loc_t, ptendency_loc_q, ptendency_loc_a, ptendency_loc_l, ptendency_loc_i};
  for (const double *q : in)
    if (!q) return fail(CLOUDSC_E_NULL, "a required array pointer is NULL");
  for (double *q : out)
    if (!q) return fail(CLOUDSC_E_NULL, "a required array pointer is NULL");
  int dev = 0;
  rc = ensure_params(&dev);
  if (rc) return rc;
  const size_t s2 = (size_t)klon * klev, s2h = (size_t)klon * (klev + 1);
  auto elems_of = [&](int i) { return i == 1 ? s2h : (i == 16 ? 4 * s2 : s2); };
  size_t total = 0;
  for (int i = 0; i < 18; ++i) total += elems_of(i);
  total += 5 * s2;
  rc = t_ws.prepare(dev, total * sizeof(double));
  if (rc) return rc;
  double *d_in[18], *d_out[5];
  double *cur = (double *)t_ws.buf;
  for (int i = 0; i < 18; ++i) {
    d_in[i] = cur;
    cur += elems_of(i);
  }
  for (int i = 0; i < 5; ++i) {
    d_out[i] = cur;
    cur += s2;
  }
  cudaStream_t s = t_ws.st[0];
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < 18 && e == cudaSuccess; ++i) {
    if (i == 16)
      e = cudaMemcpyAsync(d_in[i] + 2 * s2, in[i] + 2 * s2, 2 * s2 * sizeof(double), cudaMemcpyHostToDevice, s);
    else
      e = cudaMemcpyAsync(d_in[i], in[i], elems_of(i) * sizeof(double), cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(t_ws.counter, 0, sizeof(uint32_t), s);
  if (e != cudaSuccess) return drained(fail(CLOUDSC_E_CUDA, "host-to-device copy", e), {s});
  SatadjFields f = {d_in[0], d_in[1], d_in[2], d_in[3], d_in[4], d_in[5], d_in[6], d_in[7], d_in[8],
                    d_in[9], d_in[10], d_in[11], d_in[12], d_in[13], d_in[14], d_in[15], d_in[16], d_in[17],
                    d_out[0], d_out[1], d_out[2], d_out[3], d_out[4], t_ws.counter};
  Shape sh = {klon, klev, 1, kfdia, kidia - 1, ptsphy};
  e = launch_satadj(f, sh, s);
  if (e != cudaSuccess) return drained(fail(CLOUDSC_E_CUDA, "kernel launch", e), {s});
  // copy back columns KIDIA..KFDIA of every level
  const size_t c0 = kidia - 1, ncol = kfdia - kidia + 1;
  for (int i = 0; i < 5 && e == cudaSuccess; ++i)
    e = cudaMemcpy2DAsync(out[i] + c0, klon * sizeof(double), d_out[i] + c0, klon * sizeof(double),
                          ncol * sizeof(double), klev, cudaMemcpyDeviceToHost, s);
  uint32_t nwarn = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&nwarn, t_ws.counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return drained(fail(CLOUDSC_E_CUDA, "device-to-host copy", e), {s});
  return (int)nwarn;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// SLTEND's supersaturation adjustment (sltend.F90:380-410), the reuse of
// CLOUD_SUPERSATCHECK after the cloud scheme.
// ---------------------------------------------------------------------------
extern "C" {

int cloudsc_b200_sltend_supersat_batched(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot, double tsphy,
    const double *pt, const double *pq, const double *pa, const double *prsf1, const double *prs1,
    const double *pcent, const double *pcenq, const double *pcena, double *ptent, double *ptenq,
    double *ptena, double *ptencld, double *padja, double *padjl, double *padji, void *stream) {
  int rc = satadj_shape_ok(p, tsphy);
  if (rc) return rc;
  if (nproma < 1 || klev < 2 || ngpblks < 1 || ngptot < 1 ||
      (long long)ngptot > (long long)nproma * ngpblks || ngptot <= (long long)nproma * (ngpblks - 1))
    return fail(CLOUDSC_E_SHAPE, "inconsistent NPROMA/KLEV/NGPBLKS/NGPTOT");
  if (p->ncldtop > klev) return fail(CLOUDSC_E_SHAPE, "NCLDTOP > KLEV");
  const void *req[] = {pt, pq, pa, prsf1, prs1, pcent, pcenq, pcena, ptent, ptenq, ptena, ptencld};
  for (const void *q : req)
    if (!q) return fail(CLOUDSC_E_NULL, "a required array pointer is NULL");
  rc = ensure_params(nullptr);
  if (rc) return rc;
  SltendFields f = {pt, pq, pa, prsf1, prs1, pcent, pcenq, pcena, ptent, ptenq, ptena, ptencld,
                    padja, padjl, padji};
  Shape sh = {nproma, klev, ngpblks, ngptot, 0, tsphy};
  cudaError_t e = launch_sltend_supersat(f, sh, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "kernel launch", e);
  return CLOUDSC_OK;
}

// STATE_INCREMENT (state_increment.F90:9-105), batched.
int cloudsc_b200_state_increment_batched(int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot,
                                         int32_t kidia, const cloudsc_state *st, const cloudsc_increments *inc,
                                         void *stream) {
  if (!st || !inc) return fail(CLOUDSC_E_NULL, "postate or the increments are NULL");
  if (nproma < 1 || klev < 1 || ngpblks < 1 || ngptot < 1 || kidia < 1 || kidia > nproma ||
      (long long)ngptot > (long long)nproma * ngpblks || ngptot <= (long long)nproma * (ngpblks - 1))
    return fail(CLOUDSC_E_SHAPE, "inconsistent NPROMA/KLEV/NGPBLKS/NGPTOT/KIDIA");
  const bool any_cld = inc->pa_ql || inc->pa_qi || inc->pa_qr || inc->pa_qs;
  if (any_cld && st->nclv < 4) return fail(CLOUDSC_E_SHAPE, "NCLV of the state's CLD must be at least 4");
  if (inc->nclv_pa < 0 || (any_cld && inc->nclv_pa > 0 && inc->nclv_pa < 4))
    return fail(CLOUDSC_E_SHAPE, "the increments' NCLV must be 0 or at least 4");
  const unsigned long long s2 = (unsigned long long)nproma * klev;
  const unsigned long long cs = (unsigned long long)(st->nclv > 0 ? st->nclv : 0) * s2;
  const unsigned long long ps = inc->nclv_pa > 0 ? (unsigned long long)inc->nclv_pa * s2 : s2;
  // (state field, its KEYMASK bit or 0 for always, increment, strides), in
  // the reference's order (state_increment.F90:42-103)
  struct Pair {
    double *dst;
    uint32_t key;
    const double *src;
    unsigned long long dbs, sbs;
  };
  const Pair pairs[11] = {
      {st->u, 0, inc->pa_u, s2, s2},
      {st->v, 0, inc->pa_v, s2, s2},
      {st->t, 0, inc->pa_t, s2, s2},
      {st->q, CLOUDSC_KEY_Q, inc->pa_q, s2, s2},
      {st->o3, CLOUDSC_KEY_O3, inc->pa_o3, s2, s2},
      {st->a, CLOUDSC_KEY_A, inc->pa_a, s2, s2},
      {st->tke, CLOUDSC_KEY_TKE, inc->pa_tke, s2, s2},
      {st->cld ? st->cld + 0 * s2 : nullptr, CLOUDSC_KEY_QL, inc->pa_ql, cs, ps},
      {st->cld ? st->cld + 1 * s2 : nullptr, CLOUDSC_KEY_QI, inc->pa_qi, cs, ps},
      {st->cld ? st->cld + 2 * s2 : nullptr, CLOUDSC_KEY_QR, inc->pa_qr, cs, ps},
      {st->cld ? st->cld + 3 * s2 : nullptr, CLOUDSC_KEY_QS, inc->pa_qs, cs, ps}};
  IncFields f{};
  for (const Pair &q : pairs) {
    if (!q.src) continue;                              // PRESENT(PA_X) false
    if (q.key && !(st->keymask & q.key)) continue;     // KEYMASK off
    if (!q.dst) return fail(CLOUDSC_E_NULL, "an increment is given for a field the state does not carry");
    f.dst[f.n] = q.dst;
    f.src[f.n] = q.src;
    f.dst_bs[f.n] = q.dbs;
    f.src_bs[f.n] = q.sbs;
    ++f.n;
  }
  if (f.n == 0) return CLOUDSC_OK;
  Shape sh = {nproma, klev, ngpblks, ngptot, kidia - 1, 0.0};
  cudaError_t e = launch_state_increment(f, sh, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "kernel launch", e);
  return CLOUDSC_OK;
}

// CLOUD_SATADJ + STATE_INCREMENT of its tendencies (callpar.F90:1253-1280).
int cloudsc_b200_satadj_increment_batched(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot, double ptsphy,
    const double *pap, const double *paph, const double *pt, const double *pq, const double *pa,
    const double *pl, const double *pi, double *ptendency_cml_t, double *ptendency_cml_q,
    double *ptendency_cml_a, double *ptendency_cml_l, double *ptendency_cml_i, const double *phrsw,
    const double *phrlw, const double *ptendency_vdf_t, const double *ptendency_vdf_q, const double *pludeli,
    const double *pvervel, double *ptendency_loc_t, double *ptendency_loc_q, double *ptendency_loc_a,
    double *ptendency_loc_l, double *ptendency_loc_i, uint32_t keymask, uint32_t *ncounters,
    void *stream) {
  int rc = satadj_shape_ok(p, ptsphy);
  if (rc) return rc;
  if (nproma < 1 || klev < 2 || ngpblks < 1 || ngptot < 1 ||
      (long long)ngptot > (long long)nproma * ngpblks || ngptot <= (long long)nproma * (ngpblks - 1))
    return fail(CLOUDSC_E_SHAPE, "inconsistent NPROMA/KLEV/NGPBLKS/NGPTOT");
  if (p->ncldtop > klev) return fail(CLOUDSC_E_SHAPE, "NCLDTOP > KLEV");
  const void *req[] = {pap, paph, pt, pq, pa, pl, pi, ptendency_cml_t, ptendency_cml_q, ptendency_cml_a,
                       ptendency_cml_l, ptendency_cml_i, phrsw, phrlw, ptendency_vdf_t, ptendency_vdf_q,
                       pludeli, pvervel, ptendency_loc_t, ptendency_loc_q, ptendency_loc_a,
                       ptendency_loc_l, ptendency_loc_i};
  for (const void *q : req)
    if (!q) return fail(CLOUDSC_E_NULL, "a required array pointer is NULL");
  rc = ensure_params(nullptr);
  if (rc) return rc;
  SatadjFields f = {pap, paph, pt, pq, pa, pl, pi, ptendency_cml_t, ptendency_cml_q, ptendency_cml_a,
                    ptendency_cml_l, ptendency_cml_i, phrsw, phrlw, ptendency_vdf_t, ptendency_vdf_q,
                    pludeli, pvervel, ptendency_loc_t, ptendency_loc_q, ptendency_loc_a, ptendency_loc_l,
                    ptendency_loc_i, ncounters};
  f.inc_t = ptendency_cml_t;  // T is incremented whatever the mask
  f.inc_q = (keymask & CLOUDSC_KEY_Q) ? ptendency_cml_q : nullptr;
  f.inc_a = (keymask & CLOUDSC_KEY_A) ? ptendency_cml_a : nullptr;
  f.inc_l = (keymask & CLOUDSC_KEY_QL) ? ptendency_cml_l : nullptr;
  f.inc_i = (keymask & CLOUDSC_KEY_QI) ? ptendency_cml_i : nullptr;
  Shape sh = {nproma, klev, ngpblks, ngptot, 0, ptsphy};
  cudaError_t e = launch_satadj(f, sh, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "kernel launch", e);
  return CLOUDSC_OK;
}

int cloudsc_b200_division_check(const double *a, const double *b, int64_t n, double *q, int32_t *bad,
                                void *stream) {
  if (n < 0) return fail(CLOUDSC_E_SHAPE, "n < 0");
  if (n == 0) return CLOUDSC_OK;
  if (!a || !b || !q || !bad) return fail(CLOUDSC_E_NULL, "a required array pointer is NULL");
  cudaError_t e = launch_division_check(a, b, (long long)n, q, bad, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "kernel launch", e);
  return CLOUDSC_OK;
}

int cloudsc_b200_reciprocal_check(const double *b, int64_t n, double *y, int32_t *bad, void *stream) {
  if (n < 0) return fail(CLOUDSC_E_SHAPE, "n < 0");
  if (n == 0) return CLOUDSC_OK;
  if (!b || !y || !bad) return fail(CLOUDSC_E_NULL, "a required array pointer is NULL");
  cudaError_t e = launch_reciprocal_check(b, (long long)n, y, bad, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail(CLOUDSC_E_CUDA, "kernel launch", e);
  return CLOUDSC_OK;
}

}  // extern "C"
