/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.  Never linked into the product library;
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * A line-by-line CPU restatement of the reference's double-precision CLOUDSC
 * (ifs-source/arpifs/phys_ec/cloudsc.F90), of CLOUD_SATADJ
 * (ifs-source/arpifs/phys_ec/cloud_satadj.F90) and of their helpers, used as
 * the checker for the B200 kernels.  Parity unpinned: the reference ships no CLOUDSC golden
 * vectors and cannot be compiled here (no Fortran compiler in the image).
 */
#ifndef CLOUDSC_ORACLE_H
#define CLOUDSC_ORACLE_H

#include <stdint.h>
#include "../include/cloudsc_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

double oracle_fcgeneralized_gamma(double px);
int oracle_params_default(double tsphy, int ncldtop, cloudsc_params *p);

/* One NPROMA block, the argument list of cloudsc.F90:14-44 (derived types -> p). */
int oracle_cloudsc(
    const cloudsc_params *p, int kidia, int kfdia, int klon, int klev, int lddiag,
    double ptsphy, const double *pt, const double *pq, const double *ptendency_cml_t,
    const double *ptendency_cml_q, const double *ptendency_cml_a,
    const double *ptendency_cml_cld, double *ptendency_loc_t, double *ptendency_loc_q,
    double *ptendency_loc_a, double *ptendency_loc_cld, const double *pvfa,
    const double *pvfl, const double *pvfi, const double *pdyna, const double *pdynl,
    const double *pdyni, const double *pdynr, const double *pdyns, const double *phrsw,
    const double *phrlw, const double *pvervel, const double *pap, const double *paph,
    const double *pgeom, const double *plsm, const double *pgaw, const int32_t *ldcum,
    const int32_t *kctop, const int32_t *ktype, const int32_t *kpbltype, double *peis,
    const double *plu, double *plude, const double *pludeli, const double *psnde,
    const double *pmfu, const double *pmfd, const double *pgp2dspp, int ldslphy,
    const double *pa, const double *pclv, const double *plcrit_aer,
    const double *picrit_aer, const double *pre_ice, const double *pccn,
    const double *pnice, double *pcovptot, double *pfsd, double *prainfrac_toprfz,
    double *pfsqlf, double *pfsqif, double *pfcqnng, double *pfcqlng, double *pfsqrf,
    double *pfsqsf, double *pfcqrng, double *pfcqsng, double *pfsqltur,
    double *pfsqitur, double *pfplsl, double *pfplsn, double *pfhpsl, double *pfhpsn,
    double *pextra, int kfldx);

/*
 * The EC_PHYS_DRV block loop (ec_phys_drv.F90:430-442): OpenMP
 * SCHEDULE(DYNAMIC,1) over NPROMA blocks of arrays stored (NPROMA,...,NGPBLKS),
 * the same storage and argument order as cloudsc_b200_batched.  nthreads <= 0
 * uses the OpenMP default.  Returns the summed warning count.
 */
int oracle_cloudsc_batched(
    const cloudsc_params *p, int nproma, int klev, int ngpblks, int ngptot,
    double ptsphy, const double *pt, const double *pq, const double *ptendency_cml_t,
    const double *ptendency_cml_q, const double *ptendency_cml_a,
    const double *ptendency_cml_cld, double *ptendency_loc_t, double *ptendency_loc_q,
    double *ptendency_loc_a, double *ptendency_loc_cld, const double *pvfl,
    const double *pvfi, const double *pap, const double *paph, const double *plsm,
    const int32_t *ldcum, const int32_t *ktype, const double *peis, const double *plu,
    double *plude, const double *pludeli, const double *psnde, const double *pmfu,
    const double *pmfd, const double *pa, const double *pclv, double *pcovptot,
    double *prainfrac_toprfz, double *pfsqlf, double *pfsqif, double *pfcqnng,
    double *pfcqlng, double *pfsqrf, double *pfsqsf, double *pfcqrng, double *pfcqsng,
    double *pfsqltur, double *pfsqitur, double *pfplsl, double *pfplsn, double *pfhpsl,
    double *pfhpsn, int nthreads);

/*
 * CLOUD_SATADJ, one NPROMA block, the argument list of cloud_satadj.F90:13-26
 * (derived types -> p; PGP2DSPP and the PEXTRA budgets are not used at the
 * default configuration).  Returns the negative-condensate warning count.
 */
int oracle_cloud_satadj(
    const cloudsc_params *p, int kidia, int kfdia, int klon, int klev, const int32_t *ktype,
    int lddiag, double ptsphy, const double *pap, const double *paph, const double *pt,
    const double *pq, const double *pa, const double *pl, const double *pi,
    const double *ptendency_cml_t, const double *ptendency_cml_q, const double *ptendency_cml_a,
    const double *ptendency_cml_l, const double *ptendency_cml_i, const double *phrsw,
    const double *phrlw, const double *ptendency_vdf_t, const double *ptendency_vdf_q,
    const double *pmfu, const double *pmfd, const double *pludeli, const double *pvervel,
    double *ptendency_loc_t, double *ptendency_loc_q, double *ptendency_loc_a,
    double *ptendency_loc_l, double *ptendency_loc_i);

/* CLOUD_SATADJ over NPROMA blocks stored (NPROMA,...,NGPBLKS), OpenMP over blocks. */
int oracle_cloud_satadj_batched(
    const cloudsc_params *p, int nproma, int klev, int ngpblks, int ngptot, double ptsphy,
    const double *pap, const double *paph, const double *pt, const double *pq, const double *pa,
    const double *pl, const double *pi, const double *ptendency_cml_t, const double *ptendency_cml_q,
    const double *ptendency_cml_a, const double *ptendency_cml_l, const double *ptendency_cml_i,
    const double *phrsw, const double *phrlw, const double *ptendency_vdf_t,
    const double *ptendency_vdf_q, const double *pludeli, const double *pvervel,
    double *ptendency_loc_t, double *ptendency_loc_q, double *ptendency_loc_a,
    double *ptendency_loc_l, double *ptendency_loc_i, int nthreads);

/* oracle_cloudsc_batched with the cloud budget diagnostics' inputs and
 * PEXTRA (NPROMA, KLEV, KFLDX, NGPBLKS), INOUT. */
int oracle_cloudsc_batched_diag(
    const cloudsc_params *p, int nproma, int klev, int ngpblks, int ngptot,
    double ptsphy, const double *pt, const double *pq, const double *ptendency_cml_t,
    const double *ptendency_cml_q, const double *ptendency_cml_a,
    const double *ptendency_cml_cld, double *ptendency_loc_t, double *ptendency_loc_q,
    double *ptendency_loc_a, double *ptendency_loc_cld, const double *pvfl,
    const double *pvfi, const double *pap, const double *paph, const double *plsm,
    const int32_t *ldcum, const int32_t *ktype, const double *peis, const double *plu,
    double *plude, const double *pludeli, const double *psnde, const double *pmfu,
    const double *pmfd, const double *pa, const double *pclv, double *pcovptot,
    double *prainfrac_toprfz, double *pfsqlf, double *pfsqif, double *pfcqnng,
    double *pfcqlng, double *pfsqrf, double *pfsqsf, double *pfcqrng, double *pfcqsng,
    double *pfsqltur, double *pfsqitur, double *pfplsl, double *pfplsn, double *pfhpsl,
    double *pfhpsn, const double *pvfa, const double *pdyna, const double *pdynl,
    const double *pdyni, const double *pdyns, const double *phrsw, const double *phrlw,
    const double *pgaw, const int32_t *kctop, const int32_t *kpbltype, const double *pgp2dspp,
    const double *pre_ice, const double *picrit_aer, const double *pnice,
    double *pfsd, double *pextra, int kfldx, int nthreads);

/* The supersaturation adjustment of SLTEND (sltend.F90:380-410), one block
 * and batched over (NPROMA,...,NGPBLKS) blocks. */
int oracle_sltend_supersat(
    const cloudsc_params *p, int kidia, int kfdia, int klon, int klev, double tsphy, const double *pt,
    const double *pq, const double *pa, const double *prsf1, const double *prs1, const double *pcent,
    const double *pcenq, const double *pcena, double *ptent, double *ptenq, double *ptena, double *ptencld,
    double *padja, double *padjl, double *padji);
int oracle_sltend_supersat_batched(
    const cloudsc_params *p, int nproma, int klev, int ngpblks, int ngptot, double tsphy, const double *pt,
    const double *pq, const double *pa, const double *prsf1, const double *prs1, const double *pcent,
    const double *pcenq, const double *pcena, double *ptent, double *ptenq, double *ptena, double *ptencld,
    double *padja, double *padjl, double *padji, int nthreads);

/* STATE_INCREMENT (state_increment.F90:9-105), one block (columns
 * KIDIA..KFDIA of (KLON, KLEV) fields) and batched over (NPROMA, ...,
 * NGPBLKS) blocks; the cloudsc_state / cloudsc_increments conventions of
 * cloudsc_b200_state_increment_batched. */
int oracle_state_increment(int kidia, int kfdia, int klon, int klev, const cloudsc_state *st,
                           const cloudsc_increments *inc);
int oracle_state_increment_batched(int nproma, int klev, int ngpblks, int ngptot, int kidia,
                                   const cloudsc_state *st, const cloudsc_increments *inc);

#ifdef __cplusplus
}
#endif
#endif
