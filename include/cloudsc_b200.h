/*
 * cloudsc_b200.h -- C ABI of the B200 (sm_100a) implementation of the OpenIFS
 * prognostic cloud scheme CLOUDSC.
 *
 * The entry points keep the argument list of the reference subroutine
 *   ifs-source/arpifs/phys_ec/cloudsc.F90:14-44   (SUBROUTINE CLOUDSC)
 * in the same order, with the seven derived-type arguments (YDECLDP, YDECUMF,
 * YDEPHLI, YDERAD, YDEPHY, YDVDF, YDSPP_CONFIG) collapsed into one POD struct,
 * cloudsc_params, that the caller fills once (from the model's own YDECLDP and
 * friends, or with cloudsc_b200_params_default).
 *
 * Conventions (identical to the Fortran reference):
 *   - every array is column-major Fortran storage: element (jl,jk) of a
 *     (KLON,KLEV) array is at (jk-1)*KLON + (jl-1); element (jl,jk,jm) of a
 *     (KLON,KLEV,N) array is at ((jm-1)*KLEV + (jk-1))*KLON + (jl-1);
 *     half-level arrays are (KLON,KLEV+1);
 *   - KIDIA/KFDIA are 1-based; only columns KIDIA..KFDIA are written;
 *   - LOGICAL arguments are 4-byte integers (non-zero = .TRUE.);
 *   - REAL(KIND=JPRB) is double (the double-precision OpenIFS build);
 *   - outputs the reference leaves undefined: PTENDENCY_LOC_CLD(:,:,NCLV) is
 *     never written (cloudsc.F90:971 loops to NCLV-1), PCOVPTOT(:,1:NCLDTOP-1)
 *     is written as 0.
 *
 * Return codes: 0 = success; > 0 = number of negative-condensate warning events
 * (the reference WRITEs a warning to NULOUT for each, cloudsc.F90:3794,3802);
 * < 0 = one of the CLOUDSC_E_* errors below.  Nothing traps or aborts on the
 * device.
 */
#ifndef CLOUDSC_B200_H
#define CLOUDSC_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CLOUDSC_NCLV 5 /* yoecldp.F90:102 NCLV; species index order below */
#define CLOUDSC_NCLDQL 1
#define CLOUDSC_NCLDQI 2
#define CLOUDSC_NCLDQR 3
#define CLOUDSC_NCLDQS 4
#define CLOUDSC_NCLDQV 5

#define CLOUDSC_OK 0
#define CLOUDSC_E_NULL (-1)        /* a required array pointer is NULL          */
#define CLOUDSC_E_SHAPE (-2)       /* KIDIA/KFDIA/KLON/KLEV/NCLDTOP inconsistent */
#define CLOUDSC_E_UNSUPPORTED (-3) /* a parameter switch this build lacks is on  */
#define CLOUDSC_E_CUDA (-4)        /* a CUDA runtime call failed                */
#define CLOUDSC_E_PARAMS (-5)      /* no parameters uploaded / bad param struct */
#define CLOUDSC_E_TOO_LARGE (-6)   /* request exceeds a fixed capacity          */

#define CLOUDSC_PARAMS_MAGIC 0x434c4453u /* 'CLDS' */

/*
 * Every scalar CLOUDSC reads through its ASSOCIATE block (cloudsc.F90:612-682)
 * plus the YOMCST/YOETHF constants of fcttre.func.h.  Field names are the
 * reference names in lower case.  Integers are int32; logicals are int32.
 */
typedef struct cloudsc_params {
  uint32_t magic;   /* CLOUDSC_PARAMS_MAGIC */
  int32_t version;  /* 1 */
  /* ---- YOMCST (yomcst.F90) ---- */
  double rg, rd, rv, rcpd, retv, rtt, rlvtt, rlstt, rlmlt, rpi, ra;
  /* ---- YOETHF (suphec.F90:231-254) ---- */
  double r2es, r3les, r3ies, r4les, r4ies, r5les, r5ies, r5alvcp, r5alscp;
  double ralvdcp, ralsdcp, ralfdcp, rtwat, rtice, rticecu;
  double rtwat_rtice_r, rtwat_rticecu_r, rkoop1, rkoop2;
  /* ---- TECLDP (yoecldp.F90, defaults from sucldp.F90:243-530) ---- */
  double ramid, ramin, rlmin, rcldiff, rcldiff_convi, rclcrit_sea, rclcrit_land;
  double rkconv, rprc1, rpecons, rprecrhmax, rvrfactor, rcovpmin, rtaumel;
  double rkooptau, rssicefactor, rsnowlin1, rsnowlin2, rlcritsnow, rthomo;
  double rvice, rvrain, rvsnow, rxfallspeedrain, rxfallspeedice, rnice, rccn;
  double rcldtopcf, rdepliqrefrate, rdepliqrefdepth, riceinit, rdensref, rdenswat;
  double rcl_overlapliqice, rcl_effrime, rcl_inhomogaut, rcl_inhomogacc;
  double rcl_kkaac, rcl_kkbac, rcl_kkaau, rcl_kkbauq, rcl_kkbaun;
  double rcl_kk_cloud_num_sea, rcl_kk_cloud_num_land, rcl_eff_racw;
  double rcl_dr, rcl_x1r, rcl_x2r, rcl_lam1r, rcl_lam2r;
  double rcl_const1r, rcl_const2r, rcl_const3r, rcl_const4r, rcl_const5r;
  double rcl_const6r, rcl_const7r, rcl_const8r, rcl_const9r, rcl_const10r;
  double rcl_cdenom1, rcl_cdenom2, rcl_cdenom3, rcl_ka273, rcl_fzrab;
  double rcl_x1s, rcl_lam1s, rcl_lam2s;
  double rcl_const1s, rcl_const2s, rcl_const3s, rcl_const4s, rcl_const5s;
  double rcl_const6s, rcl_const7s, rcl_const8s;
  double rcl_const1i, rcl_const2i, rcl_const3i, rcl_const4i, rcl_const5i;
  double rcl_const6i, rcl_const7i;
  double rcl_apb1, rcl_apb2, rcl_apb3;
  double ricehi1, ricehi2;
  int32_t ncldtop;
  /* switches that select code paths; the values the B200 kernels implement
   * are the reference defaults noted beside each (others -> CLOUDSC_E_UNSUPPORTED) */
  int32_t laericeauto, laericesed, laerliqautolsp, laerliqcoll; /* any: LAERICESED, LAERICEAUTO FP64 (their
                                                                  arrays required); LAERLIQAUTOLSP and
                                                                  LAERLIQCOLL act only under IWARMRAIN = 1
                                                                  (cloudsc.F90:1985,2020), which the
                                                                  reference fixes at 3 (:727): no effect */
  int32_t lcloud_inhomog;                                       /* any (FP64) */
  int32_t lcldbudc, lcldbudl, lcldbudi, lcldbudt, lcldbud_vertint; /* any: budgets to PEXTRA, FP64 */
  int32_t lcldbud_timeint;                                      /* any */
  int32_t lcldbudget, lscmec;                                   /* 0 (diagnostic only) */
  /* ---- TECUMF (sucumf.F90:203,228-229) ---- */
  int32_t lmfdsnow;                                             /* any (default 1) */
  double rmfadvw, rmfadvwdd;                                    /* any (default 0) */
  /* ---- TERAD / TEPHY / TVDF / TSPP_CONFIG ---- */
  double rcloud_frac_std;                                       /* suecrad.F90:745 */
  int32_t lrad_cloud_inhomog;                                   /* any (FP64): PFSD */
  int32_t lbud23;                                               /* any (budgets off) */
  double reisthsc;                                              /* unused when budgets off */
  int32_t lspp;                                                 /* any */
  int32_t pad_;
  /* ---- SPP perturbations (YDSPP_CONFIG, cloudsc.F90:850-939), read when
   * lspp: perturbation n of RAMID, RCLDIFF, RCLCRIT, RLCRITSNOW, RAINEVAP,
   * SNOWSUBLIM, FALLSPEED, CLOUDINHOM (n = 0..7, CLOUDSC_SPP_* below) is on
   * when its pointer YDSPP_CONFIG%PPTR%x > 0; spp_mp[n] is its PN%MP (the
   * 1-based PGP2DSPP field; CLOUDINHOM also uses MP+1), spp_mu[2n+i] and
   * spp_xmag[2n+i] its PN%MU(i+1) and PN%XMAG(i+1).  A parameter X becomes
   * X*EXP(MU + XMAG*PGP2DSPP(JL,MP)). ---- */
  int32_t spp_on[8];
  int32_t spp_mp[8];
  double spp_mu[16];
  double spp_xmag[16];
  int32_t spp_lramidlimit1;                                     /* YDSPP_CONFIG%LRAMIDLIMIT1 */
  int32_t spp_nrftotal;                                         /* fields of PGP2DSPP (SM%NRFTOTAL) */
} cloudsc_params;

#define CLOUDSC_SPP_RAMID 0
#define CLOUDSC_SPP_RCLDIFF 1
#define CLOUDSC_SPP_RCLCRIT 2
#define CLOUDSC_SPP_RLCRITSNOW 3
#define CLOUDSC_SPP_RAINEVAP 4
#define CLOUDSC_SPP_SNOWSUBLIM 5
#define CLOUDSC_SPP_FALLSPEED 6
#define CLOUDSC_SPP_CLOUDINHOM 7

/*
 * Fill *p with the reference defaults of SUCLDP/SUPHEC/YOMCST/SUCUMF/SUECRAD
 * for physics time step tsphy (RSSICEFACTOR = MIN(TSPHY/RKOOPTAU,1),
 * sucldp.F90:655) and cloud-top level ncldtop (sucldp.F90:631-634).
 * Replaces: the SUCLDP call chain (ifs-source/arpifs/phys_ec/sucldp.F90:243-655).
 */
int cloudsc_b200_params_default(double tsphy, int32_t ncldtop, cloudsc_params *p);

/*
 * NCLDTOP from the standard-atmosphere full-level pressures stpre[0..klev-1]
 * (Pa) and RCLDTOPP (su0phy.F90:1343, 100 Pa): the smallest level >= 2 whose
 * pressure exceeds rcldtopp.  Replaces sucldp.F90:631-634.
 */
int32_t cloudsc_b200_ncldtop(int32_t klev, const double *stpre, double rcldtopp);

/*
 * Upload *p to every device this process uses (constant memory).  Must be
 * called once before the first CLOUDSC call and again whenever the parameters
 * change.  Thread-safe.  Replaces the derived-type arguments YDECLDP..YDSPP_CONFIG.
 */
int cloudsc_b200_setup(const cloudsc_params *p);

/*
 * Per-block drop-in: the full CLOUDSC argument list with HOST pointers.
 * Replaces the call at ifs-source/arpifs/phys_ec/cloud_layer.F90:169-201
 * (SUBROUTINE CLOUDSC, ifs-source/arpifs/phys_ec/cloudsc.F90:14-44).
 * Copies the block to the GPU, runs the FP64 kernel, copies results back.
 * Safe to call concurrently from several host threads (one stream and one
 * device workspace per calling thread), as EC_PHYS_DRV does under OpenMP
 * (ec_phys_drv.F90:438).  Arrays the default configuration does not read may be NULL:
 * pvfa, pdyna..pdyns, phrsw, phrlw, pvervel, pgeom, pgaw, kctop, kpbltype,
 * pgp2dspp, plcrit_aer, picrit_aer, pre_ice, pccn, pnice, pfsd, pextra.  With
 * a cloud budget switch on (LCLDBUD*), the budget diagnostics are added to
 * PEXTRA(KIDIA:KFDIA,:,1:KFLDX) and the inputs the sections that are on read
 * are required (see cloudsc_b200_batched_diag); likewise PRE_ICE with
 * LAERICESED and PICRIT_AER, PNICE with LAERICEAUTO (PLCRIT_AER and PCCN are
 * never read: see the aerosol switches in cloudsc_params).
 */
int cloudsc_b200_block(
    const cloudsc_params *p, int32_t kidia, int32_t kfdia, int32_t klon, int32_t klev,
    int32_t lddiag, double ptsphy, const double *pt, const double *pq,
    const double *ptendency_cml_t, const double *ptendency_cml_q,
    const double *ptendency_cml_a, const double *ptendency_cml_cld,
    double *ptendency_loc_t, double *ptendency_loc_q, double *ptendency_loc_a,
    double *ptendency_loc_cld, const double *pvfa, const double *pvfl,
    const double *pvfi, const double *pdyna, const double *pdynl,
    const double *pdyni, const double *pdynr, const double *pdyns,
    const double *phrsw, const double *phrlw, const double *pvervel,
    const double *pap, const double *paph, const double *pgeom, const double *plsm,
    const double *pgaw, const int32_t *ldcum, const int32_t *kctop,
    const int32_t *ktype, const int32_t *kpbltype, double *peis, const double *plu,
    double *plude, const double *pludeli, const double *psnde, const double *pmfu,
    const double *pmfd, const double *pgp2dspp, int32_t ldslphy, const double *pa,
    const double *pclv, const double *plcrit_aer, const double *picrit_aer,
    const double *pre_ice, const double *pccn, const double *pnice,
    double *pcovptot, double *pfsd, double *prainfrac_toprfz, double *pfsqlf,
    double *pfsqif, double *pfcqnng, double *pfcqlng, double *pfsqrf,
    double *pfsqsf, double *pfcqrng, double *pfcqsng, double *pfsqltur,
    double *pfsqitur, double *pfplsl, double *pfplsn, double *pfhpsl,
    double *pfhpsn, double *pextra, int32_t kfldx);

/*
 * Batched persistent launch: DEVICE pointers to arrays stored as
 * (NPROMA, <dims>, NGPBLKS), the EC_PHYS_DRV storage (ec_phys_drv.F90:145-185);
 * block ib (0-based) of an array with per-block size S starts at ib*S.
 * Block ib covers columns 1..MIN(NPROMA, NGPTOT-ib*NPROMA) (ec_phys_drv.F90:441).
 * One kernel launch processes every block on `stream` (a cudaStream_t, or
 * NULL for the default stream); the call returns without synchronising.
 * Argument order is that of CLOUDSC with KIDIA/KFDIA/KLON replaced by
 * NPROMA/NGPBLKS/NGPTOT.  The optional `ncounters` device buffer (may be NULL)
 * receives the number of negative-condensate warning events (uint32, added to).
 * `precision` selects the arithmetic: 0 = FP64 (the reference's double
 * build); 1 = FP32-mixed (the exponentials and powers of the microphysics and
 * of the level's saturation values in FP32, everything else in FP64);
 * 2 = FP32 physics (the process rates in FP32 as well; the state, the sink
 * limiters, the 5x5 solve, the saturation adjustment and the tendency and
 * flux budgets in FP64).
 */
int cloudsc_b200_batched(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks,
    int32_t ngptot, double ptsphy, const double *pt, const double *pq,
    const double *ptendency_cml_t, const double *ptendency_cml_q,
    const double *ptendency_cml_a, const double *ptendency_cml_cld,
    double *ptendency_loc_t, double *ptendency_loc_q, double *ptendency_loc_a,
    double *ptendency_loc_cld, const double *pvfl, const double *pvfi,
    const double *pap, const double *paph, const double *plsm,
    const int32_t *ldcum, const int32_t *ktype, const double *peis,
    const double *plu, double *plude, const double *pludeli, const double *psnde,
    const double *pmfu, const double *pmfd, const double *pa, const double *pclv,
    double *pcovptot, double *prainfrac_toprfz, double *pfsqlf, double *pfsqif,
    double *pfcqnng, double *pfcqlng, double *pfsqrf, double *pfsqsf,
    double *pfcqrng, double *pfcqsng, double *pfsqltur, double *pfsqitur,
    double *pfplsl, double *pfplsn, double *pfhpsl, double *pfhpsn,
    uint32_t *ncounters, int32_t precision, void *stream);

/*
 * Batched call with HOST pointers (same arrays and order as
 * cloudsc_b200_batched): blocks are processed in chunks of chunk_blocks
 * (<= 0 selects 64), each chunk's host-to-device copy, kernel and
 * device-to-host copy pipelined on three streams over three device buffers,
 * so transfers overlap compute.  Host arrays should be page-locked for the
 * copies to run asynchronously.  Synchronous: returns when all outputs are
 * back in host memory.  Columns beyond NGPTOT in the last block are left
 * untouched.  Replaces the whole EC_PHYS_DRV block loop over CLOUDSC
 * (ec_phys_drv.F90:430-442) for callers that keep the state on the host.
 */
int cloudsc_b200_batched_host(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks,
    int32_t ngptot, double ptsphy, const double *pt, const double *pq,
    const double *ptendency_cml_t, const double *ptendency_cml_q,
    const double *ptendency_cml_a, const double *ptendency_cml_cld,
    double *ptendency_loc_t, double *ptendency_loc_q, double *ptendency_loc_a,
    double *ptendency_loc_cld, const double *pvfl, const double *pvfi,
    const double *pap, const double *paph, const double *plsm,
    const int32_t *ldcum, const int32_t *ktype, const double *peis,
    const double *plu, double *plude, const double *pludeli, const double *psnde,
    const double *pmfu, const double *pmfd, const double *pa, const double *pclv,
    double *pcovptot, double *prainfrac_toprfz, double *pfsqlf, double *pfsqif,
    double *pfcqnng, double *pfcqlng, double *pfsqrf, double *pfsqsf,
    double *pfcqrng, double *pfcqsng, double *pfsqltur, double *pfsqitur,
    double *pfplsl, double *pfplsn, double *pfhpsl, double *pfhpsn,
    int32_t precision, int32_t chunk_blocks);

/*
 * The single-precision interface: the OpenIFS single-precision build
 * (JPRB = REAL(4); contrib/fiat/src/parkind/parkind1.F90:41-44, bundle.yml's
 * single-precision option) passes every REAL array of CLOUDSC's argument
 * list as float.  These two entries take the arrays of cloudsc_b200_batched /
 * cloudsc_b200_batched_host in float (LDCUM and KTYPE stay int32, the
 * parameters stay the double cloudsc_params, filled from the build's float
 * constants) and run the same kernels: each float input is widened to double
 * when it is read and each output rounded to float when it is written, so
 * `precision` 0 gives exactly the FP64 kernel's results on the widened
 * inputs, rounded to float; 1 and 2 select the FP32-mixed and FP32-physics
 * arithmetic.  Half the bytes of the double interface cross HBM and PCIe.
 * No reference counterpart beyond CLOUDSC itself in that build.
 */
int cloudsc_b200_batched_sp(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks,
    int32_t ngptot, float ptsphy, const float *pt, const float *pq,
    const float *ptendency_cml_t, const float *ptendency_cml_q,
    const float *ptendency_cml_a, const float *ptendency_cml_cld,
    float *ptendency_loc_t, float *ptendency_loc_q, float *ptendency_loc_a,
    float *ptendency_loc_cld, const float *pvfl, const float *pvfi,
    const float *pap, const float *paph, const float *plsm,
    const int32_t *ldcum, const int32_t *ktype, const float *peis,
    const float *plu, float *plude, const float *pludeli, const float *psnde,
    const float *pmfu, const float *pmfd, const float *pa, const float *pclv,
    float *pcovptot, float *prainfrac_toprfz, float *pfsqlf, float *pfsqif,
    float *pfcqnng, float *pfcqlng, float *pfsqrf, float *pfsqsf,
    float *pfcqrng, float *pfcqsng, float *pfsqltur, float *pfsqitur,
    float *pfplsl, float *pfplsn, float *pfhpsl, float *pfhpsn,
    uint32_t *ncounters, int32_t precision, void *stream);

/* The single-precision interface with host pointers, pipelined like
 * cloudsc_b200_batched_host. */
int cloudsc_b200_batched_host_sp(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks,
    int32_t ngptot, float ptsphy, const float *pt, const float *pq,
    const float *ptendency_cml_t, const float *ptendency_cml_q,
    const float *ptendency_cml_a, const float *ptendency_cml_cld,
    float *ptendency_loc_t, float *ptendency_loc_q, float *ptendency_loc_a,
    float *ptendency_loc_cld, const float *pvfl, const float *pvfi,
    const float *pap, const float *paph, const float *plsm,
    const int32_t *ldcum, const int32_t *ktype, const float *peis,
    const float *plu, float *plude, const float *pludeli, const float *psnde,
    const float *pmfu, const float *pmfd, const float *pa, const float *pclv,
    float *pcovptot, float *prainfrac_toprfz, float *pfsqlf, float *pfsqif,
    float *pfcqnng, float *pfcqlng, float *pfsqrf, float *pfsqsf,
    float *pfcqrng, float *pfcqsng, float *pfsqltur, float *pfsqitur,
    float *pfplsl, float *pfplsn, float *pfhpsl, float *pfhpsn,
    int32_t precision, int32_t chunk_blocks);

/*
 * Per-block call that allocates no device memory.  No reference counterpart:
 * the reference has no device memory at all.  This entry is for callers that
 * cannot call cudaMalloc: a model run whose GPU memory is fully reserved up
 * front by its own pool or arena, where a later allocation fails or would
 * fragment it, and drivers that must not allocate between time steps.  Same
 * computation and results as cloudsc_b200_block (FP64),
 * host pointers, the arrays the default configuration reads and writes, in
 * cloudsc_b200_batched's order, plus `stream` (a cudaStream_t, NULL = the
 * default stream) on which the copies and the kernel run; the call returns
 * after the stream has finished them.
 *
 * Device memory: one fixed array inside the library of
 * cloudsc_b200_block_noalloc_capacity() bytes (16 MiB), shared by every call
 * in the process: 256 bytes + the block's arrays must fit, i.e. KLON <= 288
 * at KLEV = 137; larger blocks return CLOUDSC_E_TOO_LARGE (use
 * cloudsc_b200_block).  Two calls whose GPU work overlapped would race on
 * the shared array; to prevent that, calls are serialised by a lock inside
 * the library and each returns only after its stream has finished.  After a
 * call the array keeps that call's inputs and outputs until the next call
 * (the warning counter is cleared at the start of each call).  The array's
 * 16 MiB are reserved on a device when cloudsc_b200_setup uploads the
 * parameters there (for another device: at the first call of any entry on
 * it), so a caller that reserves its own GPU memory pool should call
 * cloudsc_b200_setup first and leave room for them.  The same set-up also
 * reserves the kernels' per-thread local memory (it raises the CUDA stack
 * size limit to the largest kernel's frame, about 3 KB, never lowering
 * it): the driver holds that for every thread the device can run, which it
 * would otherwise take at the first launch (measured on a B200 with a 2.6 KB
 * frame: set-up took 542 MiB with the fixed array, and the first call then
 * none).
 */
int cloudsc_b200_block_noalloc(
    const cloudsc_params *p, int32_t kidia, int32_t kfdia, int32_t klon, int32_t klev,
    double ptsphy, const double *pt, const double *pq, const double *ptendency_cml_t,
    const double *ptendency_cml_q, const double *ptendency_cml_a,
    const double *ptendency_cml_cld, double *ptendency_loc_t, double *ptendency_loc_q,
    double *ptendency_loc_a, double *ptendency_loc_cld, const double *pvfl,
    const double *pvfi, const double *pap, const double *paph, const double *plsm,
    const int32_t *ldcum, const int32_t *ktype, const double *peis,
    const double *plu, double *plude, const double *pludeli, const double *psnde,
    const double *pmfu, const double *pmfd, const double *pa, const double *pclv,
    double *pcovptot, double *prainfrac_toprfz, double *pfsqlf, double *pfsqif,
    double *pfcqnng, double *pfcqlng, double *pfsqrf, double *pfsqsf,
    double *pfcqrng, double *pfcqsng, double *pfsqltur, double *pfsqitur,
    double *pfplsl, double *pfplsn, double *pfhpsl, double *pfhpsn, void *stream);

/*
 * CLOUD_SATADJ, the saturation adjustment CALLPAR runs before CLOUDSC
 * (callpar.F90:1253-1279), FP64, bit-identical to a C restatement of the
 * reference built with the kernels' libm.
 *
 * Per-block drop-in with HOST pointers: the argument list of
 * ifs-source/arpifs/phys_ec/cloud_satadj.F90:13-26 in the same order (derived
 * types -> cloudsc_params).  Replaces CALL CLOUD_SATADJ at
 * callpar.F90:1253-1279.  PL/PI and their tendencies are the liquid and ice
 * (KLON,KLEV) slices of the cloud arrays.  Not read at the default
 * configuration, may be NULL: ktype, pmfu, pmfd, pgp2dspp, pextra (the
 * budget switches and SPP are rejected with CLOUDSC_E_UNSUPPORTED).  Only
 * components 3 and 4 of PLUDELI are read.  Columns KIDIA..KFDIA of the five
 * tendencies are written, zero above NCLDTOP.  Returns the number of
 * negative-condensate warnings (cloud_satadj.F90:828,836) or a CLOUDSC_E_*.
 */
int cloudsc_b200_satadj_block(
    const cloudsc_params *p, int32_t kidia, int32_t kfdia, int32_t klon, int32_t klev,
    const int32_t *ktype, int32_t lddiag, double ptsphy, const double *pap, const double *paph,
    const double *pt, const double *pq, const double *pa, const double *pl, const double *pi,
    const double *ptendency_cml_t, const double *ptendency_cml_q, const double *ptendency_cml_a,
    const double *ptendency_cml_l, const double *ptendency_cml_i, const double *phrsw,
    const double *phrlw, const double *ptendency_vdf_t, const double *ptendency_vdf_q,
    const double *pmfu, const double *pmfd, const double *pludeli, const double *pvervel,
    const double *pgp2dspp, double *ptendency_loc_t, double *ptendency_loc_q,
    double *ptendency_loc_a, double *ptendency_loc_l, double *ptendency_loc_i,
    double *pextra, int32_t kfldx);

/*
 * Batched CLOUD_SATADJ with DEVICE pointers over NGPBLKS blocks stored
 * (NPROMA, ..., NGPBLKS) like cloudsc_b200_batched; one kernel launch, one
 * GPU thread per (column, level) point.  Argument order: that of
 * cloud_satadj.F90:13-26 without the arguments the default configuration does
 * not read, NPROMA/NGPBLKS/NGPTOT for KIDIA/KFDIA/KLON.  `ncounters` (may be
 * NULL) receives the warning count (uint32, added to).  Returns without
 * synchronising.
 */
int cloudsc_b200_satadj_batched(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot,
    double ptsphy, const double *pap, const double *paph, const double *pt, const double *pq,
    const double *pa, const double *pl, const double *pi, const double *ptendency_cml_t,
    const double *ptendency_cml_q, const double *ptendency_cml_a, const double *ptendency_cml_l,
    const double *ptendency_cml_i, const double *phrsw, const double *phrlw,
    const double *ptendency_vdf_t, const double *ptendency_vdf_q, const double *pludeli,
    const double *pvervel, double *ptendency_loc_t, double *ptendency_loc_q,
    double *ptendency_loc_a, double *ptendency_loc_l, double *ptendency_loc_i,
    uint32_t *ncounters, void *stream);

/*
 * The supersaturation adjustment of SLTEND (sltend.F90:380-410), the second
 * caller of CLOUD_SUPERSATCHECK (cloud_supersatcheck.F90:9-231, KFTLIQICE =
 * 1), batched with DEVICE pointers over (NPROMA, ..., NGPBLKS) blocks, one GPU
 * thread per point; FP64, bit-identical to the oracle's restatement.  On
 * levels NCLDTOP..KLEV the state PT + TSPHY*(PCENT+PTENT) (and the same for
 * q and cloud fraction) is checked and the adjustments are added to PTENT,
 * PTENQ, PTENA and the liquid and ice species of PTENCLD (KLON,KLEV,NCLV)
 * (INOUT); padja/padjl/padji (may be NULL) receive the cloud-fraction, liquid
 * and ice adjustment rates (SLTEND's ZADJA/ZADJL/ZADJI).  prs1 (half-level
 * pressure) is accepted for the reference's argument list; its surface value
 * feeds only a quantity CLOUD_SUPERSATCHECK never uses.  Returns without
 * synchronising.
 */
int cloudsc_b200_sltend_supersat_batched(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot,
    double tsphy, const double *pt, const double *pq, const double *pa, const double *prsf1,
    const double *prs1, const double *pcent, const double *pcenq, const double *pcena,
    double *ptent, double *ptenq, double *ptena, double *ptencld, double *padja, double *padjl,
    double *padji, void *stream);

/*
 * STATE_INCREMENT (ifs-source/arpifs/phys_ec/state_increment.F90:9-105):
 * POSTATE%X(KIDIA:KFDIA,:) = POSTATE%X(KIDIA:KFDIA,:) + PA_X(KIDIA:KFDIA,:)
 * for every increment PA_X that is present.  CALLPAR calls it on the cloud
 * path after CLOUD_SATADJ (callpar.F90:1278-1280: T, Q, A, QL, QI) and after
 * CLOUDSC (:1308-1311: T, Q, A, QL, QI, QR, QS) to add the tendencies into
 * the cumulative ones (TENDENCY_CML) that the next scheme reads.
 *
 * POSTATE: the state's fields (KLON, KLEV) and CLD (KLON, KLEV, NCLV), NULL
 * where the state does not carry the field; KEYMASK: its switches as
 * CLOUDSC_KEY_* bits -- Q, O3, A, TKE and the four condensate species are
 * incremented only when their bit is set, U, V and T whenever their increment
 * is present (state_increment.F90:42-103).  An increment given for a field
 * the state lacks is an error (CLOUDSC_E_NULL).
 */
#define CLOUDSC_KEY_Q 0x01u
#define CLOUDSC_KEY_O3 0x02u
#define CLOUDSC_KEY_A 0x04u
#define CLOUDSC_KEY_TKE 0x08u
#define CLOUDSC_KEY_QL 0x10u
#define CLOUDSC_KEY_QI 0x20u
#define CLOUDSC_KEY_QR 0x40u
#define CLOUDSC_KEY_QS 0x80u
typedef struct cloudsc_state {
  double *u, *v, *t, *o3, *q, *a, *cld, *tke;
  uint32_t keymask;
  int32_t nclv; /* species of CLD (CLOUDSC_NCLV in the default configuration) */
} cloudsc_state;
typedef struct cloudsc_increments {
  const double *pa_u, *pa_v, *pa_t, *pa_o3, *pa_q, *pa_a, *pa_ql, *pa_qi, *pa_qr, *pa_qs, *pa_tke;
  /* 0: PA_QL..PA_QS are (KLON, KLEV) arrays of their own; n > 0: each points
   * to its species slice of one (KLON, KLEV, n) array, e.g. the four
   * condensate slices of CLOUDSC's PTENDENCY_LOC_CLD (n = NCLV) */
  int32_t nclv_pa;
} cloudsc_increments;

/*
 * STATE_INCREMENT over NGPBLKS blocks with DEVICE pointers, every field
 * stored (NPROMA, KLEV[, NCLV], NGPBLKS) like cloudsc_b200_batched: columns
 * KIDIA..MIN(NPROMA, NGPTOT - (block-1)*NPROMA) of every block (one block of
 * the reference's call: ngpblks = 1, ngptot = KFDIA).  One GPU thread per
 * (column, level) point adds every present increment (one addition each,
 * bit-identical to the reference).  Returns without synchronising.
 */
int cloudsc_b200_state_increment_batched(int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot,
                                         int32_t kidia, const cloudsc_state *postate,
                                         const cloudsc_increments *inc, void *stream);

/*
 * CLOUD_SATADJ followed by the STATE_INCREMENT of its tendencies
 * (callpar.F90:1253-1280) in one kernel: the arguments of
 * cloudsc_b200_satadj_batched, with the five cumulative tendencies
 * TENDENCY_CML%T, %Q, %A, %CLD(:,:,NCLDQL), %CLD(:,:,NCLDQI) updated in place
 * (each point reads them once for the adjustment and writes them once,
 * incremented, as STATE_INCREMENT does; Q, A, QL and QI only when `keymask`
 * has their CLOUDSC_KEY_* bit).  The five TENDENCY_LOC outputs are written as
 * by cloudsc_b200_satadj_batched.  Results bit-identical to the two calls.
 * No reference counterpart as one routine: it fuses two consecutive calls of
 * CALLPAR.
 */
int cloudsc_b200_satadj_increment_batched(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks, int32_t ngptot,
    double ptsphy, const double *pap, const double *paph, const double *pt, const double *pq,
    const double *pa, const double *pl, const double *pi, double *ptendency_cml_t,
    double *ptendency_cml_q, double *ptendency_cml_a, double *ptendency_cml_l,
    double *ptendency_cml_i, const double *phrsw, const double *phrlw,
    const double *ptendency_vdf_t, const double *ptendency_vdf_q, const double *pludeli,
    const double *pvervel, double *ptendency_loc_t, double *ptendency_loc_q,
    double *ptendency_loc_a, double *ptendency_loc_l, double *ptendency_loc_i,
    uint32_t keymask, uint32_t *ncounters, void *stream);

/*
 * cloudsc_b200_batched (FP64) with the optional configurations: the cloud
 * budget diagnostics (cloudsc.F90:3832-4110) that LCLDBUDC, LCLDBUDL,
 * LCLDBUDI, LCLDBUDT and LCLDBUD_VERTINT switch on, with LCLDBUD_TIMEINT and
 * LBUD23 as in the reference; the SPP perturbations (LSPP and the spp_*
 * fields of cloudsc_params, cloudsc.F90:850-939); the cloud-inhomogeneity
 * paths (LCLOUD_INHOMOG: autoconversion/accretion enhancement from the
 * liquid FSD, :1937-2098; LRAD_CLOUD_INHOMOG: PFSD, :3819-3823, 4112-4125,
 * 4307-4359); the aerosol-aware ice fall speed (LAERICESED, :1798-1803) and
 * ice-to-snow autoconversion (LAERICEAUTO, :2776-2779).  The same arrays as
 * cloudsc_b200_batched, then the inputs only these read: PVFA, PDYNA, PDYNL,
 * PDYNI, PDYNS, PHRSW, PHRLW (budgets), PGAW (NPROMA, NGPBLKS;
 * inhomogeneity), KCTOP, KPBLTYPE (vertical-integral budget), PGP2DSPP
 * (NPROMA, NRFTOTAL, NGPBLKS; SPP), PRE_ICE (NPROMA, KLEV, NGPBLKS;
 * LAERICESED), PICRIT_AER and PNICE (NPROMA, KLEV, NGPBLKS; LAERICEAUTO), PFSD (NPROMA, KLEV,
 * NGPBLKS; written with LRAD_CLOUD_INHOMOG), PEXTRA (NPROMA, KLEV, KFLDX,
 * NGPBLKS, INOUT: the budgets are added to it); arrays of options that are
 * off may be NULL.  CLOUDSC_E_SHAPE when KFLDX is below the
 * fields the sections need (the reference ABORTs, cloudsc.F90:3945-4106) or,
 * with the vertical integral, KLEV < 84, or an SPP field pointer is outside
 * 1..NRFTOTAL.  With no option on it is cloudsc_b200_batched at FP64.  The
 * options also work through cloudsc_b200_block (its own arguments);
 * cloudsc_b200_batched, cloudsc_b200_batched_host and
 * cloudsc_b200_block_noalloc return
 * CLOUDSC_E_UNSUPPORTED when one of these options is on.  No reference
 * counterpart beyond the CLOUDSC call itself: this is its batched form.
 */
int cloudsc_b200_batched_diag(
    const cloudsc_params *p, int32_t nproma, int32_t klev, int32_t ngpblks,
    int32_t ngptot, double ptsphy, const double *pt, const double *pq,
    const double *ptendency_cml_t, const double *ptendency_cml_q,
    const double *ptendency_cml_a, const double *ptendency_cml_cld,
    double *ptendency_loc_t, double *ptendency_loc_q, double *ptendency_loc_a,
    double *ptendency_loc_cld, const double *pvfl, const double *pvfi,
    const double *pap, const double *paph, const double *plsm,
    const int32_t *ldcum, const int32_t *ktype, const double *peis,
    const double *plu, double *plude, const double *pludeli, const double *psnde,
    const double *pmfu, const double *pmfd, const double *pa, const double *pclv,
    double *pcovptot, double *prainfrac_toprfz, double *pfsqlf, double *pfsqif,
    double *pfcqnng, double *pfcqlng, double *pfsqrf, double *pfsqsf,
    double *pfcqrng, double *pfcqsng, double *pfsqltur, double *pfsqitur,
    double *pfplsl, double *pfplsn, double *pfhpsl, double *pfhpsn,
    const double *pvfa, const double *pdyna, const double *pdynl, const double *pdyni,
    const double *pdyns, const double *phrsw, const double *phrlw, const double *pgaw,
    const int32_t *kctop, const int32_t *kpbltype, const double *pgp2dspp, const double *pre_ice,
    const double *picrit_aer, const double *pnice, double *pfsd,
    double *pextra, int32_t kfldx, uint32_t *ncounters, void *stream);

/* Bytes of the fixed device array cloudsc_b200_block_noalloc works in. */
size_t cloudsc_b200_block_noalloc_capacity(void);

/* sizeof(cloudsc_params) as compiled into the library (binding check). */
size_t cloudsc_b200_params_size(void);

/*
 * Launch schedule of the kernels (the autotuner's knobs; no reference
 * counterpart: the reference runs CLOUDSC on CPU threads, one NPROMA block
 * per call, ec_phys_drv.F90:438).  Every entry point that launches a kernel
 * uses the schedule set for its precision (0 FP64, 1 FP32-mixed, 2 FP32
 * physics).
 *
 * The kernels are compiled in several variants, each a
 * __launch_bounds__(max_threads, min_ctas) pair that fixes the register
 * budget per thread.  cloudsc_b200_num_variants() gives their number;
 * cloudsc_b200_variant_info() the bounds of variant v and, when a device is
 * present, its registers and local (spill) bytes per thread (-1 without one).
 *
 * cloudsc_b200_set_schedule(): variant, columns per CTA (a multiple of 32 up
 * to the variant's max_threads) and ctas_per_sm, the persistent CTAs resident
 * per SM (0 = one CTA per tile of columns, a grid over all tiles).  Default:
 * the (448, 1) variant, 448 columns per CTA, ctas_per_sm 0.
 * cloudsc_b200_set_launch(): the same with the variant chosen as the one-CTA-
 * per-SM variant with the most registers that holds threads_per_cta.
 * Return CLOUDSC_E_SHAPE for values outside these limits.
 */
int cloudsc_b200_num_variants(void);
int cloudsc_b200_variant_info(int32_t precision, int32_t variant, int32_t *max_threads,
                              int32_t *min_ctas, int32_t *regs, int32_t *local_bytes);
int cloudsc_b200_set_schedule(int32_t precision, int32_t variant, int32_t threads_per_cta,
                              int32_t ctas_per_sm);
int cloudsc_b200_get_schedule(int32_t precision, int32_t *variant, int32_t *threads_per_cta,
                              int32_t *ctas_per_sm);
int cloudsc_b200_set_launch(int32_t precision, int32_t threads_per_cta, int32_t ctas_per_sm);

/*
 * Self-check of the division the column kernels use (no reference
 * counterpart).  The column kernels divide in double precision with a
 * branch-free reciprocal-and-residual sequence that returns IEEE a/b exactly
 * for 2^-256 <= |b| < 2^256 and a = 0 or 2^-256 <= |a| < 2^256, and records
 * every operand outside that window; a column with such an operand is run
 * again with IEEE division, so the kernels' results are those of IEEE
 * division throughout.  This entry runs that division alone on n device
 * operand pairs: q[i] = its quotient, bad[i] = 1 where an operand lies outside
 * the window (0 otherwise).  Device pointers; stream may be NULL.
 * CLOUDSC_E_SHAPE for n < 0, CLOUDSC_E_NULL for a NULL array with n > 0.
 */
int cloudsc_b200_division_check(const double *a, const double *b, int64_t n, double *q, int32_t *bad,
                                void *stream);

/*
 * The reciprocal half of that division on its own (no reference
 * counterpart): the kernels take 1/b this way, and the reciprocal of a
 * divisor shared by several quotients once.  y[i] = the reciprocal of b[i],
 * IEEE 1/b bit for bit for 2^-256 <= |b| < 2^256; bad[i] = 1 where b lies
 * outside that window (0 otherwise).  Device pointers; stream may be NULL.
 * CLOUDSC_E_SHAPE for n < 0, CLOUDSC_E_NULL for a NULL array with n > 0.
 */
int cloudsc_b200_reciprocal_check(const double *b, int64_t n, double *y, int32_t *bad, void *stream);

/* Last CUDA error string recorded by this library on the calling thread. */
const char *cloudsc_b200_last_error(void);

/* Library version string. */
const char *cloudsc_b200_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CLOUDSC_B200_H */
