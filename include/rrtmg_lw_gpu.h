/*
 * rrtmg_lw_gpu.h -- C ABI of the B200 RRTMG longwave column path.
 *
 * The library (ccpp_physics_b200/librrtmg_lw_gpu.so) replaces the two public
 * entry points of the Fortran module rrtmg_lw in ccpp-physics:
 *
 *   rlwinit       physics/Radiation/RRTMG/radlw_main.F90:1322-1324
 *   rrtmg_lw_run  physics/Radiation/RRTMG/radlw_main.F90:419-434
 *                 (argument declarations radlw_main.F90:609-656,
 *                  CCPP metadata radlw_main.meta:1-444)
 *
 * A Fortran host reaches these through an ISO_C_BINDING shim that keeps the
 * original rlwinit / rrtmg_lw_run interfaces (ccpp_physics_b200/fortran/).  Every
 * array is the caller's Fortran array, column-major, kind_phys = real(8):
 * element (i, k) of an (npts, nlay) array is at ptr[(i-1) + (k-1)*ldim],
 * element (i, k, b) of an (npts, nlay, nbands) array at
 * ptr[(i-1) + ldim*((k-1) + nlay*(b-1))].  Fortran logicals are passed as
 * int32 0/1.  Optional Fortran arguments are NULL when absent.
 *
 * Error convention (radlw_main.F90:713-760, 1415-1420): the functions return
 * errflg (0 = success, 1 = error) and copy errmsg into the caller's buffer
 * (NUL-terminated, truncated to errmsg_len).  Calls never abort the process.
 *
 * Threading: rrtmg_lw_gpu_run* may be called concurrently from several host
 * threads (the CCPP host calls rrtmg_lw_run once per physics block from
 * OpenMP threads).  Each host thread gets its own CUDA stream and device
 * workspace; the only shared state is the immutable device tables written
 * by rrtmg_lw_gpu_init.
 */
#ifndef RRTMG_LW_GPU_H
#define RRTMG_LW_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RRTMG_LW_NBANDS 16   /* radlw_param.f:103 */
#define RRTMG_LW_NGPT 140    /* radlw_param.f:104 */

/* Arguments of rlwinit (radlw_main.F90:1322-1324), plus the CUDA device. */
typedef struct rrtmg_lw_init_args {
  int32_t me;            /* print control: banner when me == 0 */
  int32_t rad_hr_units;  /* 1: heating rates in K/day, otherwise K/s */
  int32_t inc_minor_gas; /* logical; only affects the banner (as in rlwinit) */
  int32_t ilwcliq;
  int32_t isubclw;
  int32_t iovr, iovr_rand, iovr_maxrand, iovr_max, iovr_dcorr, iovr_exp,
      iovr_exprand;
  int32_t device;        /* CUDA device ordinal (extension; 0 by default) */
} rrtmg_lw_init_args;

/* Arguments of rrtmg_lw_run (radlw_main.F90:419-434), same names. */
typedef struct rrtmg_lw_run_args {
  int32_t npts, nlay, nlp1;
  int32_t ldim;          /* leading dimension of (npts,...) arrays; 0 = npts */
  int32_t lprnt, lslwr, top_at_1, inc_minor_gas;
  int32_t iovr, iovr_rand, iovr_maxrand, iovr_max, iovr_dcorr, iovr_exp,
      iovr_exprand;
  int32_t ilwcliq, ilwcice, isubclw;
  /* inputs */
  const double *plyr, *plvl, *tlyr, *tlvl, *qlyr, *olyr;
  const double *gasvmr_co2, *gasvmr_n2o, *gasvmr_ch4, *gasvmr_o2, *gasvmr_co,
      *gasvmr_cfc11, *gasvmr_cfc12, *gasvmr_cfc22, *gasvmr_ccl4;
  const int32_t *icseed;                 /* (npts) */
  const double *aeraod, *aerssa;         /* (npts, nlay, nbands) */
  const double *sfemis, *sfgtmp;         /* (npts) */
  const double *dzlyr, *delpin;          /* (npts, nlay) */
  const double *de_lgth;                 /* (npts) */
  const double *alpha;                   /* (npts, nlay) */
  const double *cld_cf;                  /* (npts, nlay) */
  /* optional cloud inputs (ilwcliq > 0 needs the first eight, else cld_od) */
  const double *cld_lwp, *cld_ref_liq, *cld_iwp, *cld_ref_ice, *cld_rwp,
      *cld_ref_rain, *cld_swp, *cld_ref_snow, *cld_od;
  /* outputs */
  double *hlwc;    /* (npts, nlay) total-sky heating rate */
  double *topflx;  /* (npts) records {upfxc, upfx0} = topflw_type */
  double *sfcflx;  /* (npts) records {upfxc, upfx0, dnfxc, dnfx0} = sfcflw_type */
  double *cldtau;  /* (npts, nlay) band-7 layer cloud optical depth */
  /* optional outputs (NULL = not present) */
  double *hlw0;    /* (npts, nlay) clear-sky heating rate */
  double *hlwb;    /* (npts, nlay, nbands) spectral-band heating rates */
  double *flxprf;  /* (npts, nlp1) records {upfxc, dnfxc, upfx0, dnfx0} = proflw_type */
} rrtmg_lw_run_args;

/* Execution options (extension, no counterpart in the reference). */
enum rrtmg_lw_precision {
  RRTMG_LW_FP64 = 0,       /* plain FP64 path, matches the Fortran within 1e-10 */
  RRTMG_LW_FP32 = 1,       /* FP32 gas optics + transfer, FP64 interpolation weights
                              and flux divergence */
  RRTMG_LW_SURROGATE = 2   /* learned gas optics (BF16 MLP) + FP32 transfer */
};
enum rrtmg_lw_memory {
  RRTMG_LW_HOST = 0,       /* every pointer is host memory (pageable or pinned) */
  RRTMG_LW_DEVICE = 1      /* every pointer is device memory on the init device */
};
typedef struct rrtmg_lw_exec {
  int32_t precision;       /* enum rrtmg_lw_precision */
  int32_t memory;          /* enum rrtmg_lw_memory */
  void *stream;            /* cudaStream_t; NULL = the calling thread's stream */
  int32_t sync;            /* 1 = return after the results are in place (host
                              memory always syncs); 0 = leave work queued */
  int32_t reserved;
  float *kernel_ms;        /* optional float[3]: device time in ms of the McICA,
                              gas-optics and transfer kernels of this call
                              (first chunk for the last two; forces a sync) */
} rrtmg_lw_exec;

/* rlwinit (radlw_main.F90:1322): validates iovr, sets fluxfac/heatfac, builds
 * the transmittance/tau-transition tables (radlw_main.F90:1474-1501) and
 * uploads every coefficient table to the device.  Returns errflg. */
int rrtmg_lw_gpu_init(const rrtmg_lw_init_args *args, char *errmsg,
                      int32_t errmsg_len);

/* rrtmg_lw_run (radlw_main.F90:419) on the GPU, FP64, host pointers.  Every
 * cloud treatment of the reference: isubclw = 1, 2 (McICA with overlap iovr
 * 0..5, transfer rtrnmc) and isubclw = 0 (grid-mean clouds, transfer rtrn for
 * iovr <= 0 and rtrnmr otherwise, radlw_main.F90:1190-1224).
 * Returns errflg. */
int rrtmg_lw_gpu_run(const rrtmg_lw_run_args *args, char *errmsg,
                     int32_t errmsg_len);

/* rrtmg_lw_run with explicit precision / memory space / stream. */
int rrtmg_lw_gpu_run_ex(const rrtmg_lw_run_args *args,
                        const rrtmg_lw_exec *exec, char *errmsg,
                        int32_t errmsg_len);

/* McICA sub-column generator alone (mcica_subcol, radlw_main.F90:1847-2107,
 * with the GFS Mersenne Twister, mersenne_twister.f:285-372), on the GPU.
 * For each column i: seed[i], cldf (ldim, nlay) layer cloud fraction already
 * floored as in cldprop (radlw_main.F90:1805-1811), dz (ldim, nlay) [km]
 * and de_lgth (npts) [km] for iovr 3, alpha (ldim, nlay) for iovr 4/5
 * (NULL otherwise); every overlap 0..5 of mcica_subcol.  Writes lcloudy as bits:
 * bits[(i*RRTMG_LW_NGPT + ig) * nwords + (k >> 5)] bit (k & 31) for g-point
 * ig (0-based) and layer k (0-based, surface first), nwords = (nlay+31)/32.
 * Device pointers only.  Returns errflg. */
int rrtmg_lw_gpu_mcica(int32_t npts, int32_t nlay, int32_t ldim, int32_t iovr,
                       const int32_t *seed, const double *cldf,
                       const double *dz, const double *de_lgth,
                       const double *alpha, uint32_t *bits, void *stream,
                       char *errmsg, int32_t errmsg_len);

/* Gas optics alone (setcoef + taumol, radlw_main.F90:2151-2406, 3836-6840)
 * for the same inputs as rrtmg_lw_run, device pointers, internal (surface
 * first) layer order: writes taug[(i*nlay + k)*140 + ig] (gas optical depth
 * before aerosol is added) and fracs[(i*nlay + k)*140 + ig] (Planck
 * fraction), precision RRTMG_LW_FP64 or RRTMG_LW_FP32 (outputs are always
 * double).  Used to generate training data for the learned gas optics and
 * for stage-level parity tests.  Returns errflg. */
int rrtmg_lw_gpu_gas_optics(const rrtmg_lw_run_args *args, int32_t precision,
                            double *taug, double *fracs, void *stream,
                            char *errmsg, int32_t errmsg_len);

/* rrtmg_lw_run for callers that cannot allocate device memory during a run:
 * hosts that give (nearly) all GPU memory to their own pool at start-up and
 * time-step loops that must not call cudaMalloc/cudaFree, which synchronize
 * the device.  No counterpart in the reference.  Same arguments and results
 * as rrtmg_lw_gpu_run_ex with RRTMG_LW_DEVICE memory (every pointer is device
 * memory owned by the caller), precision RRTMG_LW_FP64 or RRTMG_LW_FP32, work
 * queued on `stream` (NULL = default stream) and synchronized before return.
 * The kernels' scratch is a fixed 64 MiB array inside the library (held by
 * every GPU that loads it until exit); calls whose columns do not fit are
 * rejected with an error giving the maximum (about 190 columns of 127 layers
 * in FP64).  All calls share that array: calls that overlap on the GPU race.
 * The first call on a device looks up the array's device address; make it
 * before any stream capture.  Returns errflg. */
int rrtmg_lw_gpu_run_noalloc(const rrtmg_lw_run_args *args, int32_t precision,
                             void *stream, char *errmsg, int32_t errmsg_len);

/* Launch shape of the column kernels.  Chosen by rrtmg_lw_gpu_autotune or
 * given by the caller; zero fields take the defaults. */
typedef struct rrtmg_lw_tuning {
  int32_t rt_warps;        /* columns (one warp each) per CTA of the transfer
                              kernel: 1, 2 or 4 (default 4) */
  int32_t gas_per_sm;      /* resident gas-optics CTAs per SM to launch
                              (0 = the occupancy limit) */
  int32_t chunk_cols;      /* columns per gas-optics -> transfer hand-off
                              (0 = as many as the scratch budget holds) */
  int32_t use_graph;       /* run_blocks only: 1 = capture the call's launches
                              in a CUDA graph on first use and replay it when
                              the same block set (same pointers, sizes, flags
                              and shape) is called again */
} rrtmg_lw_tuning;

/* UFS-style physics blocks in one call.  The reference host calls
 * rrtmg_lw_run once per block of columns (radlw_main.F90:419, from OpenMP
 * threads); here blocks[b] is the rrtmg_lw_run argument set of block b, all
 * blocks with the same nlay and flags, every pointer device memory.  The
 * columns of all blocks form one index space and run in one persistent
 * launch of each kernel (McICA, gas optics, transfer; the last two repeat
 * only when the scratch budget splits the columns into chunks), with no
 * per-block launches.  exec: precision FP64 or FP32, memory must be
 * RRTMG_LW_DEVICE, stream, sync; kernel_ms is filled only without a graph.
 * tune: launch shape and graph use (NULL = the autotuned shape if
 * rrtmg_lw_gpu_autotune ran for this layer count and precision, else the
 * defaults, no graph).  A replayed graph reads the blocks' arrays through the
 * same pointers, so inputs updated in place are picked up.  No counterpart
 * in the reference.  Returns errflg. */
int rrtmg_lw_gpu_run_blocks(const rrtmg_lw_run_args *blocks, int32_t nblocks,
                            const rrtmg_lw_exec *exec,
                            const rrtmg_lw_tuning *tune, char *errmsg,
                            int32_t errmsg_len);

/* Autotuner of the launch shape: runs the first blocks totalling at least
 * sample_cols columns (0 = all blocks) with each candidate shape (transfer
 * CTA of 1, 2 or 4 columns x chunk sizes), timing two runs of each with CUDA
 * events, and keeps the fastest as the default shape of later calls with the
 * same layer count and precision.  Writes the blocks' outputs.  best and
 * best_ms (optional) receive the chosen shape and its time per call.  No
 * counterpart in the reference.  Returns errflg. */
int rrtmg_lw_gpu_autotune(const rrtmg_lw_run_args *blocks, int32_t nblocks,
                          int32_t precision, void *stream,
                          int64_t sample_cols, rrtmg_lw_tuning *best,
                          float *best_ms, char *errmsg, int32_t errmsg_len);
/* Sets the default launch shape of later calls with this layer count and
 * precision, as the autotuner does after timing (NULL clears it): a host
 * that saved the autotuner's choice per layer count, precision and GPU
 * restores it without re-timing (ccpp_physics_b200.rrtmg_lw.autotune keeps
 * such a JSON cache).  No counterpart in the reference.  Returns errflg. */
int rrtmg_lw_gpu_set_tuning(int32_t nlay, int32_t precision,
                            const rrtmg_lw_tuning *tune, char *errmsg,
                            int32_t errmsg_len);

/* ---- Learned gas optics (no counterpart in the reference) -------------
 * A BF16 MLP 8 -> 128 -> 128 -> 288 (SiLU) on the tensor cores replaces
 * setcoef + taumol (radlw_main.F90:2151-2406, 3836-6840) for every layer
 * whose features lie inside the training envelope; the gas-optics kernel
 * recomputes the other layers with plain taumol.  Run it through
 * rrtmg_lw_gpu_run_ex / _run_blocks with precision RRTMG_LW_SURROGATE (cloud
 * optics, McICA and the transfer then run in FP32).
 * Features per layer (float[8], internal order: row = column * nlay + layer,
 * surface first): ln p[hPa], T[K], ln h2o vmr, ln o3 vmr, co2, ch4, n2o
 * [ppmv], 1.  Outputs (float[288], normalised): [0,140) log(taug/coldry)
 * for the 140 g-points, [144,284) Planck fractions, the rest padding.
 * Normalisation, float[RRTMG_LW_SURROGATE_NORM]: input mean[8], std[8],
 * envelope low[8], high[8], output mean[288], std[288].
 * Weights, float[RRTMG_LW_SURROGATE_NPARAM]: W1[128][8] (column 7 = bias of
 * layer 1), W2[128][128], b2[128], W3[280][128], b3[280]. */
#define RRTMG_LW_SURROGATE_NORM 608
#define RRTMG_LW_SURROGATE_NPARAM 53656
#define RRTMG_LW_SURROGATE_NGRAD 54688   /* gradient export, padded output rows */

/* Features and dry-air column amount (coldry of radlw_main.F90:835, in
 * 1e20 molecules/cm^2) of every layer of one block, device pointers:
 * feats[npts*nlay][8], coldry[npts*nlay] (may be NULL). */
int rrtmg_lw_gpu_surrogate_features(const rrtmg_lw_run_args *args, float *feats,
                                    float *coldry, void *stream, char *errmsg,
                                    int32_t errmsg_len);
/* Random initial weights (seeded) and the normalisation (host float[608]). */
int rrtmg_lw_gpu_surrogate_init(const float *norm, uint64_t seed, char *errmsg,
                                int32_t errmsg_len);
/* Load / read trained weights and normalisation (host arrays). */
int rrtmg_lw_gpu_surrogate_set(const float *weights, const float *norm,
                               char *errmsg, int32_t errmsg_len);
int rrtmg_lw_gpu_surrogate_get(float *weights, float *norm, char *errmsg,
                               int32_t errmsg_len);
/* Adam training on device data feats[n][8], targets[n][288] (normalised,
 * padded), batch a multiple of 128, learning rate decaying from lr to
 * lr_final (cosine); loss_per_epoch optional host float[epochs] (MSE).
 * flags bit 0: weight every optical-depth error by 1 / (1 + 1.66 tau) of its
 * target (opaque layers barely change the fluxes), with the layer's coldry
 * stored in feats[., 7]. */
int rrtmg_lw_gpu_surrogate_train(const float *feats, const float *targets,
                                 int64_t n, int32_t epochs, int32_t batch,
                                 float lr, float lr_final, uint64_t seed,
                                 int32_t flags, float *loss_per_epoch,
                                 void *stream,
                                 char *errmsg, int32_t errmsg_len);
/* Training checkpoint: the FP32 master parameters and Adam's first and
 * second moment estimates, each host float[RRTMG_LW_SURROGATE_NSTATE] in the
 * padded layout of the gradient export, the optimizer step count and the
 * normalisation (float[608]).  get_state fills any non-NULL argument;
 * set_state restores all of them, so training resumes where it stopped. */
#define RRTMG_LW_SURROGATE_NSTATE 54688
int rrtmg_lw_gpu_surrogate_get_state(float *params, float *m, float *v,
                                     int64_t *step, float *norm, char *errmsg,
                                     int32_t errmsg_len);
int rrtmg_lw_gpu_surrogate_set_state(const float *params, const float *m,
                                     const float *v, int64_t step,
                                     const float *norm, char *errmsg,
                                     int32_t errmsg_len);
/* Network outputs (normalised) for device features: y[n][288]. */
int rrtmg_lw_gpu_surrogate_forward(const float *feats, int64_t n, float *y,
                                   void *stream, char *errmsg,
                                   int32_t errmsg_len);
/* One forward + backward pass over the first `batch` samples without an
 * update: host grads[RRTMG_LW_SURROGATE_NGRAD] in the padded parameter order
 * (W1[128][8], W2[128][128], b2[128], W3[288][128], b3[288]) and the MSE. */
int rrtmg_lw_gpu_surrogate_grads(const float *feats, const float *targets,
                                 int32_t batch, float *grads, float *loss,
                                 void *stream, char *errmsg, int32_t errmsg_len);
/* Layers recomputed with taumol since the last reset, and the tensor-core
 * wait-timeout flag of the surrogate kernels.  Returns 0 on success. */
int rrtmg_lw_gpu_surrogate_stats(uint64_t *fallback_layers, int32_t *mma_error,
                                 int32_t reset);
/* Failure-detection hook: the number of polls a tensor-core wait of the
 * network's forward kernel makes before it gives up (polls < 0 restores the
 * default of 2^22; 0 gives up at the first wait).  A kernel that gives up
 * still waits, bounded, for the MMA it issued, frees its tensor memory, and
 * the call reports "tensor-core wait timed out" (mma_error of _stats).  For
 * tests; returns 0 on success. */
int rrtmg_lw_gpu_surrogate_wait_limit(int64_t polls);

/* ---- Steps either side of rrtmg_lw_run ------------------------------------
 * They need no tables: they run on the device rrtmg_lw_gpu_init selected (the
 * current device before init).  The exec struct gives memory, stream (NULL =
 * the per-thread default stream) and sync; precision is ignored.  Host memory
 * is staged through the device and always syncs.  Each returns 0, or 1 with
 * a message. */

/* Seed part of GFS_rad_time_vary_timestep_init
 * (physics/Interstitials/UFS_SCM_NEPTUNE/GFS_rad_time_vary.fv3.F90:59-84).
 * Only when (lsswr or lslwr) and (isubc_lw == 2 or isubc_sw == 2):
 *   lrseeds: icsdsw(ix) = rseeds(ix,1), icsdlw(ix) = rseeds(ix,2);
 *   else:    ipseed = mod(nint(100 sqrt(sec)), ipsdlim) + 1 + ipsd0 seeds one
 *            twister stream, numrdm(1:2 cnx cny) = random_index(ipsdlim)
 *            (mersenne_twister.f:489-503: max(ceiling(h ipsdlim), 1)), and
 *            with (i, j) = (imap(ix), jmap(ix)), p = i+isc-1 + (j+jsc-2) cnx:
 *            icsdsw(ix) = numrdm(p), icsdlw(ix) = numrdm(p + cnx cny).
 * Otherwise the outputs are left as they are.  A p outside 1..cnx cny is an
 * error (the Fortran would read out of bounds); the call syncs to report it. */
typedef struct rrtmg_lw_seed_args {
  double sec;                      /* seconds since the forecast start */
  int32_t lslwr, lsswr, isubc_lw, isubc_sw;
  int32_t lrseeds;                 /* logical: seeds supplied in rseeds */
  int32_t ipsd0, ipsdlim;
  int32_t cnx, cny, isc, jsc;
  int32_t n;                       /* columns: size(jmap) */
  int32_t ld_rseeds;               /* leading dimension of rseeds; 0 = n */
  const int32_t *imap, *jmap;      /* (n), 1-based grid indices */
  const int32_t *rseeds;           /* (ld_rseeds, 2) when lrseeds */
  int32_t *icsdsw, *icsdlw;        /* (n) */
} rrtmg_lw_seed_args;
int rrtmg_lw_gpu_seeds(const rrtmg_lw_seed_args *args, const rrtmg_lw_exec *exec,
                       char *errmsg, int32_t errmsg_len);

/* Cloud-overlap parameters: the block of radiation_clouds.f:837-856 with the
 * routines of physics/Radiation/radiation_cloud_overlap.F90.
 *   de_lgth by idcor: idcor_hogan       max(0.6, 2.78 - 4.6 |xlat / con_pi|)
 *                                       (cmp_dcorr_lgth_hogan, :28-50);
 *                     idcor_oreopoulos  am1 + am2 exp(-(latdeg - am3)^2 / am4^2),
 *                                       am3 by julian and yearlen (:58-93);
 *                     idcor_con         dcorr_con;
 *                     other             de_lgth left as it is.
 *   alpha (get_alpha_exper, :99-145) when iovr is iovr_dcorr, iovr_exp or
 *   iovr_exprand: alpha(:,1) = 0, alpha(:,k) = exp(-dzlay(:,k) / de_lgth), and
 *   for iovr_exprand 0 where a clear layer follows a cloudy one (cld_frac);
 *   for any other iovr de_lgth = 0 and alpha = 0.
 * mode selects the block (both steps) or one routine alone. */
enum rrtmg_lw_overlap_mode {
  RRTMG_LW_OVERLAP_CLOUDS = 0,     /* the radiation_clouds.f block */
  RRTMG_LW_OVERLAP_DCORR = 1,      /* cmp_dcorr_lgth by idcor only */
  RRTMG_LW_OVERLAP_ALPHA = 2       /* get_alpha_exper only; de_lgth is an input */
};
typedef struct rrtmg_lw_overlap_args {
  int32_t mode;                    /* enum rrtmg_lw_overlap_mode */
  int32_t npts, nlay, ldim;        /* ldim: leading dimension of (npts, nlay); 0 = npts */
  int32_t idcor, idcor_con, idcor_hogan, idcor_oreopoulos;
  int32_t iovr, iovr_dcorr, iovr_exp, iovr_exprand;
  int32_t yearlen;                 /* days in the year (Oreopoulos) */
  double julian;                   /* julian day (Oreopoulos) */
  double dcorr_con;                /* km (idcor_con) */
  double con_pi;
  const double *xlat;              /* (npts) radians (Hogan) */
  const double *latdeg;            /* (npts) degrees (Oreopoulos) */
  const double *dzlay;             /* (npts, nlay) km between layer centres */
  const double *cld_frac;          /* (npts, nlay), read for iovr_exprand */
  double *de_lgth;                 /* (npts) km */
  double *alpha;                   /* (npts, nlay) */
} rrtmg_lw_overlap_args;
int rrtmg_lw_gpu_overlap_params(const rrtmg_lw_overlap_args *args, const rrtmg_lw_exec *exec,
                                char *errmsg, int32_t errmsg_len);

/* rrtmg_lw_post_run (physics/Radiation/RRTMG/rrtmg_lw_post.F90:13-77): when
 * lslwr, tsflw = tsfa; htrlw(:,k) = htlwc(:,k+kd) for k = 1..lm and htrlw(:,lm)
 * for k = lm+1..levs; the same from htlw0 into lwhc when lwhtr; sfcdlw =
 * sfcflw%dnfxc.  On the device-resident outputs of a run this keeps the
 * heating-rate arrays on the device (no host read-back).  Requires kd <= ltp,
 * lm <= levs and lm >= 1 when levs > lm. */
typedef struct rrtmg_lw_post_args {
  int32_t im, levs, ltp, lm, kd;
  int32_t lslwr, lwhtr;
  const double *tsfa;              /* (im) */
  const double *htlwc, *htlw0;     /* (im, lm+ltp) */
  const double *sfcflw;            /* (im) records {upfxc, upfx0, dnfxc, dnfx0} */
  double *tsflw, *sfcdlw;          /* (im) */
  double *htrlw, *lwhc;            /* (im, levs); lwhc only when lwhtr */
} rrtmg_lw_post_args;
int rrtmg_lw_gpu_post(const rrtmg_lw_post_args *args, const rrtmg_lw_exec *exec,
                      char *errmsg, int32_t errmsg_len);

/* Kernels enqueued by the calling thread's most recent rrtmg_lw_gpu_run,
 * _run_ex or _run_blocks call (a replayed CUDA graph counts the kernels it
 * holds; a host-memory call counts its last chunk).  Diagnostics for
 * benchmarks; no counterpart in the reference. */
int32_t rrtmg_lw_gpu_last_launch_count(void);

/* Release device tables and per-thread workspaces (call once at exit). */
void rrtmg_lw_gpu_finalize(void);

#ifdef __cplusplus
}
#endif
#endif /* RRTMG_LW_GPU_H */
