// Shared device-side definitions for the CLOUDSC kernels (FP64 and FP32-mixed).
//
// Species indices follow yoecldp.F90:102-107 shifted to 0-based:
//   L=0 (NCLDQL) cloud liquid, I=1 (NCLDQI) cloud ice, R=2 (NCLDQR) rain,
//   S=3 (NCLDQS) snow, V=4 (NCLDQV) vapour.
#pragma once
#include <cstdint>
#include "../../include/cloudsc_b200.h"

namespace cloudsc {

constexpr int L = 0, I = 1, R = 2, S = 3, V = 4;

// Loop-invariant values hoisted out of the level loop and computed once on the
// host with the same libm expression the reference evaluates per point.
struct Derived {
  double zconst_pow_land;  // RCL_KK_CLOUD_NUM_LAND**RCL_KKBAUN (cloudsc.F90:2179-2181)
  double zconst_pow_sea;   // RCL_KK_CLOUD_NUM_SEA**RCL_KKBAUN
  double flt_0p4;          // REAL(0.4,4) widened: the default-REAL exponent at :2320,:2980
  double flt_0p8;          // REAL(0.8,4) widened: the threshold at :2889
};

// Pointers of the batched (NPROMA, <dims>, NGPBLKS) arrays; block ib of an
// array with per-block size S starts at ib*S.
struct Fields {
  const double *pt, *pq, *cml_t, *cml_q, *cml_a, *cml_cld;
  double *loc_t, *loc_q, *loc_a, *loc_cld;
  const double *pvfl, *pvfi, *pap, *paph, *plsm;
  const int32_t *ldcum, *ktype;
  const double *peis, *plu;
  double *plude;
  const double *pludeli, *psnde, *pmfu, *pmfd, *pa, *pclv;
  double *pcovptot, *prainfrac_toprfz;
  double *pfsqlf, *pfsqif, *pfcqnng, *pfcqlng, *pfsqrf, *pfsqsf, *pfcqrng, *pfcqsng;
  double *pfsqltur, *pfsqitur, *pfplsl, *pfplsn, *pfhpsl, *pfhpsn;
  uint32_t *ncounters;
  // read only by the cloud budget diagnostics (the kernel form with budgets)
  const double *pvfa, *pdyna, *pdynl, *pdyni, *pdyns, *phrsw, *phrlw;
  const int32_t *kctop, *kpbltype;
  double *pextra;  // PEXTRA (NPROMA, KLEV, KFLDX) per block, INOUT
  int kfldx;
  // read only by the SPP / cloud-inhomogeneity form
  const double *pgaw;      // (NPROMA) per block
  const double *pgp2dspp;  // (NPROMA, NRFTOTAL) per block
  double *pfsd;            // (NPROMA, KLEV) per block, written with LRAD_CLOUD_INHOMOG
  int nrftotal;
  // read only with the aerosol switches (same form): (NPROMA, KLEV) per block
  const double *pre_ice;     // LAERICESED: ice effective radius
  const double *picrit_aer;  // LAERICEAUTO: critical ice amount
  const double *pnice;       // LAERICEAUTO: ice number concentration
};

// Pointers of the batched arrays of the single-precision interface
// (JPRB = REAL(4), the OpenIFS single-precision build: parkind1.F90:41-44):
// the arrays the default configuration reads and writes, in float, with the
// member names of Fields so that the column body reads them unchanged (each
// load widened to double, each store rounded to float).
struct FieldsSP {
  const float *pt, *pq, *cml_t, *cml_q, *cml_a, *cml_cld;
  float *loc_t, *loc_q, *loc_a, *loc_cld;
  const float *pvfl, *pvfi, *pap, *paph, *plsm;
  const int32_t *ldcum, *ktype;
  const float *peis, *plu;
  float *plude;
  const float *pludeli, *psnde, *pmfu, *pmfd, *pa, *pclv;
  float *pcovptot, *prainfrac_toprfz;
  float *pfsqlf, *pfsqif, *pfcqnng, *pfcqlng, *pfsqrf, *pfsqsf, *pfcqrng, *pfcqsng;
  float *pfsqltur, *pfsqitur, *pfplsl, *pfplsn, *pfhpsl, *pfhpsn;
  uint32_t *ncounters;
};

// Pointers of the batched CLOUD_SATADJ arrays (same block layout).
struct SatadjFields {
  const double *pap, *paph, *pt, *pq, *pa, *pl, *pi;
  const double *cml_t, *cml_q, *cml_a, *cml_l, *cml_i;
  const double *phrsw, *phrlw, *vdf_t, *vdf_q, *pludeli, *pvervel;
  double *loc_t, *loc_q, *loc_a, *loc_l, *loc_i;
  uint32_t *ncounters;
  // the fused STATE_INCREMENT (callpar.F90:1278-1280): where not NULL, the
  // cumulative tendency written back incremented by SATADJ's (these alias
  // cml_t .. cml_i; NULL for a field the state's KEYMASK leaves out)
  double *inc_t, *inc_q, *inc_a, *inc_l, *inc_i;
};

// STATE_INCREMENT's fields (state_increment.F90): n pairs dst += src, each an
// (NPROMA, KLEV) slab per block with its own block stride in elements (a
// species slice of a (NPROMA, KLEV, NCLV) array has stride NCLV*KLEV*NPROMA).
struct IncFields {
  double *dst[11];
  const double *src[11];
  unsigned long long dst_bs[11], src_bs[11];
  int n;
};

// Pointers of the batched arrays of SLTEND's supersaturation adjustment
// (same block layout; ptencld has NCLV species per block).
struct SltendFields {
  const double *pt, *pq, *pa, *prsf1, *prs1, *pcent, *pcenq, *pcena;
  double *ptent, *ptenq, *ptena, *ptencld, *padja, *padjl, *padji;
};

struct Shape {
  int nproma, klev, ngpblks, ngptot;
  int kidia0;  // first column of every block computed (0-based KIDIA-1)
  double ptsphy;
};

// Levels whose PLUDE input the kernels' fast pass keeps for a rerun of the
// column (a per-thread array); with more levels (KLEV above this) every form
// runs its plain kernel, IEEE division throughout.
constexpr int kMaxLevFast = 256;

}  // namespace cloudsc
