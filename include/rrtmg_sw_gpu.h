/*
 * rrtmg_sw_gpu.h -- C ABI of the B200 RRTMG shortwave column path.
 *
 * The library (ccpp_physics_b200/librrtmg_lw_gpu.so, the same library as the
 * longwave path) replaces the two public entry points of the Fortran module
 * rrtmg_sw in ccpp-physics:
 *
 *   rswinit       physics/Radiation/RRTMG/radsw_main.F90:1388-1390
 *   rrtmg_sw_run  physics/Radiation/RRTMG/radsw_main.F90:493-510
 *                 (argument declarations radsw_main.F90:688-782)
 *
 * and the CCPP schemes either side of the run:
 *
 *   rad_sw_pre_run     physics/Radiation/RRTMG/rad_sw_pre.F90:14-51
 *   rrtmg_sw_post_run  physics/Radiation/RRTMG/rrtmg_sw_post.F90:13-129
 *
 * Array conventions are those of rrtmg_lw_gpu.h: the caller's Fortran arrays,
 * column-major, real(8); element (i, k) of an (npts, nlay) array is at
 * ptr[(i-1) + (k-1)*ldim], element (i, k, b) of an (npts, nlay, nbands)
 * array at ptr[(i-1) + ldim*((k-1) + nlay*(b-1))].  Logicals are int32 0/1,
 * absent optional arguments are NULL.  The derived-type outputs are arrays
 * of records of doubles in the field order of radsw_param.f:
 *   topfsw_type {upfxc, dnfxc, upfx0}
 *   sfcfsw_type {upfxc, dnfxc, upfx0, dnfx0}
 *   profsw_type {upfxc, dnfxc, upfx0, dnfx0}
 *   cmpfsw_type {uvbfc, uvbf0, nirbm, nirdf, visbm, visdf}
 * The functions return errflg (0 = success, 1 = error) and copy errmsg into
 * the caller's buffer (NUL-terminated, truncated to errmsg_len).
 *
 * Every cloud treatment of rrtmg_sw_run is built, in FP64: McICA
 * sub-columns (isubcsw = 1, 2; transfer spcvrtm) with every overlap of
 * mcica_subcol (iovr 0..5), and grid-mean clouds (isubcsw = 0; transfer
 * spcvrtc).  Also built: every cloud-optics option (iswcliq 0, 1, 2;
 * iswcice 1, 2, 3), every two-stream option (iswmode 1, 2, 3) and every
 * output.
 */
#ifndef RRTMG_SW_GPU_H
#define RRTMG_SW_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RRTMG_SW_NBANDS 14   /* radsw_param.f: NBANDS = NBHGH - NBLOW + 1 */
#define RRTMG_SW_NGPT 112    /* radsw_param.f: NGPTSW */

/* Arguments of rswinit (radsw_main.F90:1388-1390), plus the CUDA device. */
typedef struct rrtmg_sw_init_args {
  int32_t me;            /* print control: banner when me == 0 */
  int32_t rad_hr_units;  /* 1: heating rates in K/day, otherwise K/s */
  int32_t inc_minor_gas; /* logical; banner only (as in rswinit) */
  int32_t iswcliq;
  int32_t isubcsw;
  int32_t iovr, iovr_rand, iovr_maxrand, iovr_max, iovr_dcorr, iovr_exp,
      iovr_exprand;
  int32_t iswmode;
  int32_t device;        /* CUDA device ordinal (extension; 0 by default) */
} rrtmg_sw_init_args;

/* Arguments of rrtmg_sw_run (radsw_main.F90:493-510), same names. */
typedef struct rrtmg_sw_run_args {
  int32_t npts, nlay, nlp1;
  int32_t ldim;          /* leading dimension of (npts,...) arrays; 0 = npts */
  int32_t nday;          /* number of daytime points listed in idxday */
  int32_t lprnt, lsswr, top_at_1, inc_minor_gas;
  int32_t iovr, iovr_rand, iovr_maxrand, iovr_max, iovr_dcorr, iovr_exp,
      iovr_exprand;
  int32_t iswcliq, iswcice, isubcsw, iswmode;
  double solcon;         /* solar constant [W/m2] */
  /* inputs */
  const double *plyr, *plvl, *tlyr, *tlvl, *qlyr, *olyr;
  const double *gasvmr_co2, *gasvmr_n2o, *gasvmr_ch4, *gasvmr_o2, *gasvmr_co,
      *gasvmr_cfc11, *gasvmr_cfc12, *gasvmr_cfc22, *gasvmr_ccl4;
  const int32_t *icseed;                 /* (npts) */
  const int32_t *idxday;                 /* (nday) 1-based daytime columns */
  const double *aeraod, *aerssa, *aerasy;  /* (npts, nlay, nbands) */
  const double *sfcalb_nir_dir, *sfcalb_nir_dif, *sfcalb_uvis_dir,
      *sfcalb_uvis_dif;                  /* (npts) */
  const double *dzlyr, *delpin;          /* (npts, nlay) */
  const double *de_lgth;                 /* (npts) */
  const double *alpha;                   /* (npts, nlay) */
  const double *cosz;                    /* (npts) */
  const double *cld_cf;                  /* (npts, nlay) */
  /* optional cloud inputs (iswcliq > 0 needs the first eight, else the last three) */
  const double *cld_lwp, *cld_ref_liq, *cld_iwp, *cld_ref_ice, *cld_rwp,
      *cld_ref_rain, *cld_swp, *cld_ref_snow, *cld_od, *cld_ssa, *cld_asy;
  /* outputs */
  double *hswc;    /* (npts, nlay) total-sky heating rate */
  double *topflx;  /* (npts) topfsw_type records */
  double *sfcflx;  /* (npts) sfcfsw_type records */
  double *cldtau;  /* (npts, nlay) layer cloud optical depth of band 25 (0.55 um) */
  /* optional outputs (NULL = not present) */
  double *hsw0;    /* (npts, nlay) clear-sky heating rate */
  double *hswb;    /* (npts, nlay, nbands) spectral-band heating rates */
  double *flxprf;  /* (npts, nlp1) profsw_type records */
  double *fdncmp;  /* (npts) cmpfsw_type records */
} rrtmg_sw_run_args;

/* Execution options (extension): the same record as rrtmg_lw_exec;
 * precision must be 0 (FP64).  memory 0 = host pointers, 1 = device. */
typedef struct rrtmg_sw_exec {
  int32_t precision;
  int32_t memory;
  void *stream;            /* cudaStream_t; NULL = the calling thread's stream */
  int32_t sync;
  int32_t reserved;
  float *kernel_ms;        /* optional float[3]: device ms of the McICA, gas
                              optics and transfer kernels (forces a sync) */
} rrtmg_sw_exec;

/* rswinit (radsw_main.F90:1388): validates iovr, sets heatfac, builds the
 * exp_tbl transmittance table (radsw_main.F90:1521-1531) and uploads every
 * coefficient table to the device.  Returns errflg. */
int rrtmg_sw_gpu_init(const rrtmg_sw_init_args *args, char *errmsg,
                      int32_t errmsg_len);

/* rrtmg_sw_run (radsw_main.F90:493) on the GPU, FP64, host pointers,
 * synchronous.  Returns errflg. */
int rrtmg_sw_gpu_run(const rrtmg_sw_run_args *args, char *errmsg,
                     int32_t errmsg_len);

/* rrtmg_sw_run with an explicit memory space / stream. */
int rrtmg_sw_gpu_run_ex(const rrtmg_sw_run_args *args,
                        const rrtmg_sw_exec *exec, char *errmsg,
                        int32_t errmsg_len);

/* Gas optics alone (setcoef + taumol, radsw_main.F90:2242-2389, 4094-5573)
 * for the daytime columns of `args`, device pointers: writes, for daytime
 * point p (0-based, in idxday order) and internal (surface-first) layer k,
 * taug[(p*nlay + k)*112 + ig], taur[(p*nlay + k)*112 + ig] and
 * sfluxzen[p*112 + ig].  Stage entry point for parity tests. */
int rrtmg_sw_gpu_gas_optics(const rrtmg_sw_run_args *args, double *taug,
                            double *taur, double *sfluxzen, void *stream,
                            char *errmsg, int32_t errmsg_len);

/* UFS-style physics blocks in one call.  The reference host calls
 * rrtmg_sw_run once per block of columns; here blocks[b] is the
 * rrtmg_sw_run argument set of block b, every pointer device memory, all
 * blocks with the same nlay and flags and all or none with hswb.  The daytime
 * points of all blocks form one index space and run in one launch of each
 * kernel (repeated only when the scratch budget splits them), with no
 * per-block launches; the results equal per-block rrtmg_sw_gpu_run_ex calls
 * (isubcsw = 1 seeds stay block-relative, as the reference's are).  Blocks
 * with lsswr = 0 or nday <= 0 are left untouched.  exec: memory must be 1;
 * stream, sync and kernel_ms as in rrtmg_sw_gpu_run_ex.  Returns errflg. */
int rrtmg_sw_gpu_run_blocks(const rrtmg_sw_run_args *blocks, int32_t nblocks,
                            const rrtmg_sw_exec *exec, char *errmsg,
                            int32_t errmsg_len);

/* Sub-column generator alone (mcica_subcol, radsw_main.F90:1952-2212, with
 * the GFS Mersenne twister), on the GPU, for every overlap iovr 0..5.  For
 * each column i: seed[i]; cldf (ldim, nlay) the layer cloud fraction already
 * floored at 1e-12 as cldprop does (radsw_main.F90:1904-1908), internal
 * (surface-first) layer order; dz (ldim, nlay) [km] and de_lgth (npts) [km]
 * for iovr 3, alpha (ldim, nlay) for iovr 4, 5 (NULL otherwise).  Writes
 * lcloudy as bits: bits[(i*RRTMG_SW_NGPT + ig) * nwords + (k >> 5)] bit
 * (k & 31), nwords = (nlay + 31) / 32.  Device pointers only.  Stage entry
 * point for bit-exact tests.  Returns errflg. */
int rrtmg_sw_gpu_mcica(int32_t npts, int32_t nlay, int32_t ldim, int32_t iovr,
                       const int32_t *seed, const double *cldf,
                       const double *dz, const double *de_lgth,
                       const double *alpha, uint32_t *bits, void *stream,
                       char *errmsg, int32_t errmsg_len);

/* rad_sw_pre_run (physics/Radiation/RRTMG/rad_sw_pre.F90:14-51), same
 * argument names: the daytime points of the call.  When lsswr, idxday(1:nday)
 * lists, in increasing order, the 1-based columns i with coszen(i) >= 0.0001,
 * and idxday(nday+1:im) = 0; otherwise nday = 0 and idxday = 0.  coszen and
 * idxday are (im) arrays in the exec's memory space; nday is always a host
 * int32, so the call waits for its stream to read it back (exec.sync is not
 * read).  With memory = 1 the idxday it writes feeds rrtmg_sw_gpu_run_ex
 * directly.  Returns errflg. */
typedef struct rrtmg_sw_pre_args {
  int32_t im, lsswr;
  const double *coszen;  /* (im) */
  int32_t *nday;         /* host */
  int32_t *idxday;       /* (im) */
} rrtmg_sw_pre_args;
int rrtmg_sw_gpu_pre(const rrtmg_sw_pre_args *args, const rrtmg_sw_exec *exec,
                     char *errmsg, int32_t errmsg_len);

/* rrtmg_sw_post_run (physics/Radiation/RRTMG/rrtmg_sw_post.F90:13-129), same
 * argument names; every array (im[, levels]) with leading dimension im.
 * When lsswr:
 *   nday > 0:  htrsw(:,k) = htswc(:,k+kd) for k = 1..lm and htrsw(:,lm) for
 *              k = lm+1..levs; the same from htsw0 into swhc when swhtr;
 *              nirbmdi, nirdfdi, visbmdi, visdfdi = scmpsw%nirbm, %nirdf,
 *              %visbm, %visdf and the ...ui fields those times sfcalb1..4;
 *   nday <= 0: htrsw (im, levs), swhc (when swhtr), the eight component
 *              fields and the sfcfsw, topfsw and scmpsw records set to 0;
 * then sfcnsw = sfcfsw%dnfxc - sfcfsw%upfxc and sfcdsw = sfcfsw%dnfxc.
 * levr is accepted and unused, as in the reference.  With nday > 0 it
 * requires kd <= ltp, lm <= levs and lm >= 1 when levs > lm.  exec: memory,
 * stream and sync as in rrtmg_sw_gpu_run_ex; precision is not read.  On the
 * device-resident outputs of a run this keeps them on the device. */
typedef struct rrtmg_sw_post_args {
  int32_t im, levr, levs, ltp, nday, lm, kd;
  int32_t lsswr, swhtr;
  const double *sfcalb1, *sfcalb2, *sfcalb3, *sfcalb4;   /* (im) */
  const double *htswc, *htsw0;                          /* (im, lm+ltp) */
  double *nirbmdi, *nirdfdi, *visbmdi, *visdfdi;         /* (im) */
  double *nirbmui, *nirdfui, *visbmui, *visdfui;         /* (im) */
  double *sfcdsw, *sfcnsw;                              /* (im) */
  double *htrsw, *swhc;          /* (im, levs); swhc only when swhtr */
  double *scmpsw;                /* (im) cmpfsw_type records, inout */
  double *sfcfsw;                /* (im) sfcfsw_type records, inout */
  double *topfsw;                /* (im) topfsw_type records, inout */
} rrtmg_sw_post_args;
int rrtmg_sw_gpu_post(const rrtmg_sw_post_args *args,
                      const rrtmg_sw_exec *exec, char *errmsg,
                      int32_t errmsg_len);

/* Releases the device tables of rrtmg_sw_gpu_init. */
void rrtmg_sw_gpu_finalize(void);

#ifdef __cplusplus
}
#endif
#endif /* RRTMG_SW_GPU_H */
