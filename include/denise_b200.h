/*
 * denise_b200.h - C ABI of the B200 P-SV propagator and FWI adjoint gradient.
 *
 * This library replaces the reference's single-shot time loop
 *   psv()                     src/PSV/psv.c:17            (modes 0/1/2)
 * and everything it calls per time step:
 *   update_v_PML_PSV          include/fd.h:324            (velocity + CPML + force/adjoint sources)
 *   update_s_elastic_PML_PSV  include/fd.h:309            (elastic stress + CPML)
 *   update_s_visc_PML_PSV     include/fd.h:316            (viscoelastic stress + memory variables)
 *   surface_elastic_PML_PSV   include/fd.h:297, surface_visc_PML_PSV include/fd.h:300
 *   psource / msource         include/fd.h:858 / :827
 *   seismo_ssg                include/fd.h:904
 *   eprecond                  include/fd.h:779
 *   zero_denise_*_PSV         include/fd.h:331 / :335
 *   the forward-snapshot store and adjoint cross-correlation inlined at src/PSV/psv.c:240-387,
 *   the per-shot gradient assembly ass_gradPSV (src/PSV/ass_gradPSV.c:10),
 * together with the MPI halo exchange (exchange_v/s_PSV), which disappears because
 * the whole grid of a shot lives on one GPU.
 *
 * Set-up numerics that the reference computes on the host (PML_pro, holbergcoeff,
 * av_mue/av_rho/av_tau with the single-rank periodic material wrap of matcopy_*,
 * prepare_update_s_visc_PSV) are exported too; they are computed in host C with
 * the reference's float/double promotion rules and are bit-identical to it.
 *
 * Conventions
 *  - Grid indices are the reference's: i = 1..nx (x, contiguous in its files),
 *    j = 1..ny (depth).  A source/receiver at (i, j) is the reference's
 *    srcpos_loc[1..2] / recpos_loc[1..2].
 *  - Model, gradient and snapshot arrays cross the ABI in the reference's FILE
 *    order (readmod_elastic_PSV.c:72-85, extract_LBFGS_PSV.c:84-200): x-major,
 *    z contiguous, a[(i-1)*ny + (j-1)].
 *  - Seismic sections are [ntr][nt] row-major, sample k = time step k+1
 *    (the reference's section[itr][nt], seismo_ssg.c:24).
 *  - Every entry point returns an int status (DN_OK or a negative DN_E* code).
 *    Nothing in the library exits or aborts; the host driver maps errors to the
 *    reference's err() behaviour.
 *  - Objects are not thread-safe; use one model/shot set per host thread.
 */
#ifndef DENISE_B200_H
#define DENISE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DN_VERSION_MAJOR 0
#define DN_VERSION_MINOR 1

/* ---- status codes ------------------------------------------------------ */
#define DN_OK 0
#define DN_EINVAL (-1)     /* bad parameter: FDORDER, MAXRELERROR, sizes, CFL ... */
#define DN_ENOMEM (-2)     /* device or host allocation failed */
#define DN_EUNSTABLE (-3)  /* NaN in the wavefield (psv.c:99-103 "Simulation is unstable") */
#define DN_ETIMEDOUT (-4)  /* a bounded device/host wait ran out */
#define DN_EDEVICE (-5)    /* CUDA error; see dn_last_error() */
#define DN_ENOTSUP (-6)    /* option the propagator does not implement */
#define DN_EIO (-7)        /* file could not be read / written */
#define DN_ESTATE (-8)     /* call out of order (e.g. adjoint before a stored forward) */

/* ---- enums ------------------------------------------------------------- */
#define DN_MAX_L 5           /* max relaxation mechanisms */

#define DN_MODE_FORWARD 0    /* psv() mode 0: forward, stores snapshots if params.store_snapshots */
#define DN_MODE_ADJOINT 1    /* psv() mode 1: back-propagation + cross-correlation */
#define DN_MODE_OBJECTIVE 2  /* psv() mode 2: forward for the objective only */

#define DN_SNAP_F32 0        /* snapshot storage precision */
#define DN_SNAP_F16 1        /* IEEE half with a per-snapshot, per-field power-of-two scale */
#define DN_SNAP_BF16 2       /* bfloat16 with the same scaling */

#define DN_ACC_F32 0         /* gradient accumulation in float, in the reference's order */
#define DN_ACC_F64 1         /* gradient accumulation in double */

#define DN_ARITH_EXACT 0     /* FP32 with the reference's operation order and double promotions */
#define DN_ARITH_FMA 1       /* FP32 with fused multiply-add contraction (faster, not bit-exact) */

/* section components (seismo_ssg.c SEISMO cases) */
#define DN_SEC_VX 0
#define DN_SEC_VY 1
#define DN_SEC_P 2
#define DN_SEC_CURL 3
#define DN_SEC_DIV 4

/* gradient components */
#define DN_GRAD_VP 0
#define DN_GRAD_VS 1
#define DN_GRAD_RHO 2

/* ---- parameters (the subset of read_par.c globals the path reads) ---------- */
typedef struct dn_params {
    int nx, ny;              /* NX, NY                               read_par.c case 7, 8 */
    float dh;                /* DH                                   case 9 */
    float dt;                /* DT                                   case 11 */
    int nt;                  /* NT = iround(TIME/DT)                 FD_PSV.c:68 */
    int fdorder;             /* FDORDER 2,4,...,12                   case 5 */
    int maxrelerror;         /* MAXRELERROR 0..4                     case 6 */
    int free_surf;           /* FREE_SURF                            case 28 */
    int fw;                  /* FW (CPML width in points)            case 29 */
    float damping;           /* DAMPING                              case 30 */
    float fpml;              /* FPML                                 case 31 */
    float npower;            /* npower                               case 32 */
    float k_max_pml;         /* k_max_PML                            case 33 */
    int boundary;            /* BOUNDARY (only 0 supported)          case 34 */
    int L;                   /* relaxation mechanisms, 0 = elastic   case 25 */
    float fl[DN_MAX_L];      /* FL[1..L]                             case 26 */
    float ts;                /* TS = 1/max source fc (sources.c:90); used by the visco free surface */
    int invmat1;             /* INVMAT1 (1 = vp,vs,rho)              case 66 */
    int grad_form;           /* GRAD_FORM (1)                        case 67 */
    int quelltypb;           /* QUELLTYPB adjoint source type        case 68 */
    int seismo;              /* SEISMO 0..4                          case 44 */
    int dtinv;               /* DTINV snapshot interval              case 95 */
    int eprecond;            /* EPRECOND (0,1,3)                     workflow file */
    int store_snapshots;     /* store forward snapshots in mode 0 (MODE>0 in the reference) */
    int snap_precision;      /* DN_SNAP_* */
    int grad_accum;          /* DN_ACC_* */
    int arith;               /* DN_ARITH_* */
    int honor_q;             /* 0: Q forced to 30 as readmod_visc_PSV.c:106-107; 1: use the qp/qs arrays */
    int ckpt_steps;          /* 0: store every snapshot of the forward run; > 0 (a multiple of dtinv):
                                checkpointed adjoint - the forward run keeps the full state every
                                ckpt_steps steps and the adjoint recomputes one segment of snapshots
                                at a time (no counterpart in the reference, which stores all) */
} dn_params;

/* One shot's acquisition: sources (psource/update_v injection points) and
 * receivers (seismo_ssg).  All pointers are host memory; copied at create. */
typedef struct dn_acq {
    int nsrc;
    const int *src_i, *src_j;      /* grid indices of the sources, 1-based (splitsrc.c:27-28) */
    const int *src_type;           /* QUELLTYP per source (srcpos[8]) 1 explosive, 2/3 force, 4 rotated, 5 moment */
    const float *src_azi;          /* azimuth in degrees (srcpos[7]), may be NULL */
    const float *signals;          /* [nsrc][nt] source time functions (wavelet.c) */
    int ntr;
    const int *rec_i, *rec_j;      /* receiver grid indices, 1-based (receiver.c:55-57) */
} dn_acq;

/* CPML profile vectors, each [2*fw], index h-1 for the reference's h = 1..2*FW
 * (left/top frame in 1..FW, right/bottom in FW+1..2*FW; PML_pro.c:65-407). */
typedef struct dn_pml {
    float *d_x, *K_x, *alpha_prime_x, *a_x, *b_x;
    float *d_x_half, *K_x_half, *alpha_prime_x_half, *a_x_half, *b_x_half;
    float *d_y, *K_y, *alpha_prime_y, *a_y, *b_y;
    float *d_y_half, *K_y_half, *alpha_prime_y_half, *a_y_half, *b_y_half;
} dn_pml;

typedef struct dn_model dn_model;   /* device-resident material coefficients for one grid */
typedef struct dn_shot dn_shot;     /* device-resident wavefield state of one shot */

/* ---- library ------------------------------------------------------------ */
const char *dn_last_error(void);      /* thread-local text of the last failure */
int dn_version(int *major, int *minor);
int dn_device_count(int *count);
/* Free and total memory of a device (cudaMemGetInfo with that device current);
 * free includes the blocks the library keeps cached for reuse. */
int dn_device_memory(int device, size_t *free_bytes, size_t *total_bytes);
/* Device memory of models and shots is cached per device when freed and
 * handed to the next request of nearly the same size (DN_POOL=0: plain
 * cudaMalloc / cudaFree).  Frees the cached blocks, e.g. before another
 * allocator needs the memory. */
int dn_device_trim(int device);

/* ---- host set-up numerics (bit-identical to the reference) ----------------- */
/* holbergcoeff(): src/holbergcoeff.c:19-90; hc[0..6] */
int dn_holbergcoeff(int fdorder, int maxrelerror, float hc[7]);
/* PML_pro(): src/PML_pro.c:65-407; every dn_pml vector must hold 2*fw floats */
int dn_pml_profiles(const dn_params *p, dn_pml *out);
/* CFL limit of checkfd_ssg_elastic(): src/checkfd_ssg_elastic.c:89,126 */
int dn_cfl_check(const dn_params *p, float vp_max, double *dtstab);
/* matcopy_elastic_PSV (single-rank periodic wrap) + av_mue + av_rho:
 * src/PSV/matcopy_elastic_PSV.c, src/av_mue.c:4-51, src/av_rho.c:5-28.
 * Inputs and outputs in file order [nx*ny]. */
int dn_average_materials(const dn_params *p, const float *vp, const float *vs, const float *rho,
                         float *uipjp, float *rip, float *rjp);
/* readmod_visc_PSV tau/eta (src/PSV/readmod_visc_PSV.c:31-120), matcopy_PSV wrap, av_tau
 * (src/av_tau.c:5-15) and prepare_update_s_visc_PSV (src/PSV/prepare_update_s_visc_PSV.c:9-94).
 * Outputs: fipjp, f, g [nx*ny] and dip, d, e [L][nx*ny] (file order per l), bip, bjm, cip, cjm,
 * eta [L]. */
int dn_prepare_visc(const dn_params *p, const float *vp, const float *vs, const float *rho,
                    const float *qp, const float *qs, float *fipjp, float *f, float *g,
                    float *dip, float *d, float *e, float *bip, float *bjm, float *cip, float *cjm,
                    float *eta);
/* Ricker / fumue / sin^3 / Gaussian-derivative / spike wavelets of wavelet.c:12-120
 * (QUELLART 1,2,4,5,6) for one source, with N_ORDER time integrations.  out[nt]. */
int dn_wavelet(int quellart, int nt, float dt, float tshift, float fc, float amp, int n_order, float *out);
/* wavelet(): src/wavelet.c:33-106 for one source, every QUELLART: 3 takes its
 * samples from `file_signal` (file_ns >= nt values, as dn_read_signal_file
 * reads "<SIGNAL_FILE>_shot_<n>.dat"), 6 is the unfiltered spike (the callers
 * of wavelet() band-limit it with apply_tdfilt(ORDER_SPIKE, FC_SPIKE_2,
 * FC_SPIKE_1): dn_tdfilt), 7 the Klauder chirp from FC_SPIKE_1 to FC_SPIKE_2
 * over TS (ts_chirp).  dn_wavelet covers QUELLART 1, 2, 4, 5 and 6. */
int dn_wavelet_ex(int quellart, int nt, float dt, float tshift, float fc, float amp, int n_order, float fc_spike_1,
                  float fc_spike_2, float ts_chirp, const float *file_signal, int file_ns, float *out);

/* ---- models and shots (device) -------------------------------------------- */
/* Uploads the model files to `device` and builds every derived coefficient
 * there, with the float / double operations of the host functions above (the
 * same bits; DN_HOST_MATERIALS=1 in the environment builds them on the host
 * instead).  vp, vs, rho (and qp, qs when p->L > 0) are in file order. */
int dn_model_create(const dn_params *p, const float *vp, const float *vs, const float *rho,
                    const float *qp, const float *qs, int device, dn_model **out);
int dn_model_destroy(dn_model *m);
int dn_model_params(const dn_model *m, dn_params *out);
/* One of a model's material planes, nx*ny floats in file order:
 * 0 rip, 1 rjp, 2 uipjp (av_rho / av_mue), 3 mu, 4 lambda, 5 rho, 6 vp, 7 vs,
 * 8 muss, 9 lamss (the gradient's), and for L > 0: 10 mu at (i+1/2, j+1/2),
 * 11 its tau_s, 12 mu, 13 tau_s, 14 pi, 15 tau_p (the relaxed moduli and
 * relaxation times the viscoelastic stress update is formed from). */
#define DN_MAT_COUNT 16
int dn_model_get_material(const dn_model *m, int which, float *out);
/* Bytes of device memory a model / a shot of this acquisition will hold. */
int dn_model_footprint(const dn_params *p, size_t *bytes);
int dn_shot_footprint(const dn_params *p, int ntr, int store_snapshots, size_t *bytes);

int dn_shot_create(dn_model *m, const dn_acq *acq, dn_shot **out);
int dn_shot_destroy(dn_shot *s);

/* Runs the whole time loop (nt = 1..NT) of psv() for n shots at once in one
 * batched launch per half-step (shots may belong to different models and grid
 * sizes; they must share FDORDER and elastic/visco).  mode: DN_MODE_*.
 * Mode 0 stores snapshots iff the model's params.store_snapshots.  Mode 1
 * needs dn_shot_set_residuals() and a previous stored mode-0 run of the shot.
 * Returns DN_EUNSTABLE if a NaN appeared (checked at the psv.c:99 cell). */
int dn_run(dn_shot *const *shots, int n, int mode);
/* Plain path: one shot, one kernel launch per operation, no batching/graphs. */
int dn_run_plain(dn_shot *s, int mode);

/* Sections recorded in the last forward run; comp = DN_SEC_*; out [ntr][nt]. */
int dn_shot_get_sections(const dn_shot *s, int comp, float *out);
/* Adjoint sources for mode 1: residuals [ntr][nt] as calc_res() leaves them
 * (time-reversed, src/calc_res.c:432-445).  NULL = component not used. */
int dn_shot_set_residuals(dn_shot *s, const float *vxdiff, const float *vydiff, const float *pdiff);
/* ass_gradPSV (src/PSV/ass_gradPSV.c:10-152) of this shot's correlation, then
 * added to the model's stacked gradient (grad_obj_psv.c:253-261). */
int dn_shot_accumulate_gradient(dn_shot *s);
/* The same with the per-shot energy preconditioning of grad_obj_psv.c:218-240
 * (eprecond1.c): the shot must have run with params.eprecond 1 (We = sqrt(Ws Wr),
 * forward and adjoint energies) or 3 (We = sqrt(Ws) times the asinh receiver
 * term); We += 0.005 max(We); the shot's vp, vs, rho gradients are divided by
 * We c^2 with c = c_vp, c_vs, c_rho (the reference's model averages; c_vs = 0
 * zeroes the vs gradient) before they are stacked. */
int dn_shot_accumulate_gradient_precond(dn_shot *s, float c_vp, float c_vs, float c_rho);
/* The model's stacked gradients (waveconv, waveconv_u, waveconv_rho) in file order. */
int dn_model_get_gradient(const dn_model *m, float *g_vp, float *g_vs, float *g_rho);
int dn_model_zero_gradient(dn_model *m);
/* Replaces the model's stacked gradients (file order; NULL leaves a class as it
 * is), e.g. with the sum over ranks before the conditioning below. */
int dn_model_set_gradient(dn_model *m, const float *g_vp, const float *g_vs, const float *g_rho);

/* The model's stacked gradients as one vector of 3 nx ny doubles in device
 * memory of the model's device (classes vp, vs, rho, each row-major [j][i]),
 * e.g. for an all-reduce sum over ranks in place of grad_obj_psv.c:371-390's
 * element-wise MPI_Allreduce, and back (rounded to the model's accumulator
 * type).  Both wait for the device's pending work first. */
int dn_model_gradient_to_device(const dn_model *m, double *d_out);
int dn_model_gradient_from_device(dn_model *m, const double *d_in);

/* ---- gradient conditioning ------------------------------------------------
 * smooth_grad (src/smooth_grad.c) of the three stacked gradients followed by
 * precond_PSV (src/PSV/precond_PSV.c), FWI_PSV.c:628-634, and the per-shot
 * circular taper taper_grad_shot (src/taper_grad_shot.c) that
 * grad_obj_psv.c:242-250 applies before stacking.  Field names are the .inp
 * keywords of the reference. */
typedef struct dn_precond {
    /* smooth_grad: 0 none, 2 smooth2 (tridiagonal smoothing, WD_DAMP along z,
     * WD_DAMP1 along x), 3 gauss_filt (Gaussian of WD_DAMP * C_vs / FC_END),
     * 4 gauss_filt_var (Gaussian of WD_DAMP, WD_DAMP1 times the local S
     * wavelength vs / FC_END).  1 (wavenumber filter) needs FFTW: DN_ENOTSUP. */
    int spatfilter;
    float wd_damp, wd_damp1, fc_end, c_vs;
    /* precond_PSV tapers, applied in this order to each class */
    int taper_vert;                     /* SWS_TAPER_GRAD_VERT (taper_grad sws 1) */
    int taper_hor;                      /* SWS_TAPER_GRAD_HOR (sws 2) */
    int taper_sources;                  /* SWS_TAPER_GRAD_SOURCES (sws 3) */
    int taper_file;                     /* SWS_TAPER_FILE (sws 4-6) */
    int gradt[4];                       /* GRADT1..GRADT4 */
    float exp_taper_grad_hor;           /* EXP_TAPER_GRAD_HOR */
    int srtshape;                       /* SRTSHAPE: 1 erf, 2 log */
    float srtradius;                    /* SRTRADIUS (m) */
    int filtsize;                       /* FILTSIZE: half-width of the zeroed box at each source */
    /* taper_file: coefficients of TFILE.bin, TFILE_u.bin, TFILE_rho.bin (file order) */
    const float *taper_vp, *taper_vs, *taper_rho;
    /* acquisition: all sources of the survey (metres, srcpos[1..2]) and receivers (grid indices) */
    int nsrc;
    const float *src_x, *src_z;
    int ntr;
    const int *rec_i, *rec_j;
} dn_precond;

typedef struct dn_precond_plan dn_precond_plan;
/* Validates `c` and computes, on the host, everything that depends on the
 * geometry only (taper coefficients, zeroed cells, smoothing factorisations,
 * Gaussian weights), stored on `device` for dn_precond_apply. */
int dn_precond_create(int nx, int ny, float dh, const dn_precond *c, int device, dn_precond_plan **out);
int dn_precond_destroy(dn_precond_plan *p);
/* Conditions the model's stacked gradients in place on the device (smoothing,
 * then the tapers).  SPATFILTER 4 reads the model's vs. */
int dn_precond_apply(const dn_precond_plan *p, dn_model *m);
/* The taper coefficients of one taper_grad switch (sws 1 vertical, 2
 * horizontal, 3 sources; before the zeroed source boxes) in file order: the
 * TFILE_coeff_*.bin the reference writes. */
int dn_taper_coefficients(int nx, int ny, float dh, const dn_precond *c, int sws, float *coeff);

/* Per-shot options of the gradient assembly (grad_obj_psv.c:214-250). */
typedef struct dn_accum_opts {
    int energy;                         /* 1: EPRECOND 1/3 scaling (as dn_shot_accumulate_gradient_precond) */
    float c_vp, c_vs, c_rho;
    int circular_taper;                 /* SWS_TAPER_CIRCULAR_PER_SHOT: taper_grad_shot around this shot's source */
    int srtshape;
    float srtradius;
    int filtsize;
    float src_x, src_z;                 /* this shot's source position (m) */
} dn_accum_opts;
int dn_shot_accumulate_gradient_ex(dn_shot *s, const dn_accum_opts *o);

/* Unit-level access for parity tests: full-grid interior copies in file order.
 * field ids: 0 vx, 1 vy, 2 sxx, 3 syy, 4 sxy, 5 vxp1, 6 vyp1,
 *            7 waveconv_shot, 8 waveconv_u_shot, 9 waveconv_rho_shot, 10 Ws, 11 Wr */
int dn_shot_get_field(const dn_shot *s, int field, float *out);
/* Runs only time steps [nt0, nt1] of `mode` on one shot (nt0 == 1 zeroes the state). */
int dn_run_steps(dn_shot *s, int mode, int nt0, int nt1);
/* Decoded forward snapshot k (0-based) of one stored field (0 rho_x, 1 rho_y, 2 x, 3 y, 4 u). */
int dn_shot_get_snapshot(const dn_shot *s, int k, int field, float *out);

/* Device time of the last dn_run / dn_run_plain in milliseconds (CUDA events
 * around the time loop only) and the number of kernel launches it issued. */
int dn_last_run_stats(double *device_ms, long long *launches);

/* calc_res() for LNORM = 2 (src/calc_res.c:306-445 residual, :514-568 misfit) on
 * the device.  syn_tm: synthetic section, time-major [nt][ntr] (the layout the
 * propagator records); obs: observed section [ntr][nt]; res (out): adjoint
 * source [ntr][nt], time-reversed, first observed sample replaced by the
 * synthetic one, time-integrated when grad_form == 1; l2 (out, host): the misfit
 * 0.5*sum(res^2) accumulated in double.  All arrays are device pointers; the
 * call allocates ntr+1 doubles of device scratch for the per-trace sums.  The
 * kernels run on the legacy default stream, which does not wait for work on
 * non-blocking streams: the producers of syn_tm and obs must have finished
 * (e.g. their stream synchronised) before the call; it returns after the misfit
 * has been read back. */
int dn_residual_l2(const float *syn_tm, const float *obs, float *res, int ntr, int nt, float dt, int grad_form,
                   double *l2);
/* dn_residual_l2 for callers that cannot allocate device memory during the
 * call (an inversion loop that has reserved all device memory for its shots
 * and snapshots, or that must not let cudaMalloc/cudaFree synchronise the
 * device between shots).  No counterpart in the reference: calc_res() works
 * on host arrays.  Same arguments and results as dn_residual_l2, but the
 * per-trace sums use a static device array, so ntr <= 16384 (DN_EINVAL
 * beyond).  The first call on each device (with that device current) looks up
 * the array and should come before any stream capture; the address it keeps
 * does not survive a cudaDeviceReset of the device (not supported between
 * calls).  Calls that overlap on one device share that array and race;
 * serialise them.  Inputs must be complete as for dn_residual_l2. */
int dn_residual_l2_noalloc(const float *syn_tm, const float *obs, float *res, int ntr, int nt, float dt,
                           int grad_form, double *l2);
/* The same for a shot after its forward run: obs [ntr][nt] in host memory,
 * comp = DN_SEC_VX / DN_SEC_VY / DN_SEC_P; the residual becomes the shot's
 * adjoint source of that component (calc_res_PSV.c), l2 the component's misfit. */
int dn_shot_residual(dn_shot *s, int comp, const float *obs, double *l2);
/* Reverse-time migration (MODE 2): the shot's adjoint source of `comp` becomes the
 * observed data itself, time-reversed and (GRAD_FORM 1) time-integrated, as
 * calc_res.c:436/441 forms it for MODE 2; the adjoint run then images instead
 * of computing a gradient (RTM_PSV.c: P image = the vp gradient, S image = the
 * vs gradient of dn_model_get_gradient). */
int dn_shot_rtm_source(dn_shot *s, int comp, const float *obs);

/* calc_res (src/calc_res.c) with the objective functions that need no Fourier
 * transform and its trace selections.  LNORM 6 (envelope, Hilbert transform)
 * and TIMEWIN 1-4 (picked or STA/LTA windows) are DN_ENOTSUP; LNORM 8 needs
 * GRAD_FORM 2 (the reference has no AGC array otherwise). */
typedef struct dn_residual_opts {
    int lnorm;                /* LNORM: 1 L1 sign, 2 L2, 3 Cauchy, 4 sech, 5 global correlation,
                                 7 normalised integration, 8 AGC-weighted L2 */
    int grad_form;            /* GRAD_FORM 1 (time-integrated) or 2 */
    int mode;                 /* MODE 1 or 3: residual; 2: the RTM source (LNORM 2) */
    int n_order;              /* N_ORDER time integrations of both sections */
    int comp_weight;          /* COMP_WEIGHT > 0: both sections times c_vp * c_rho */
    float c_vp, c_rho;
    float fc_start, fc_end;   /* LNORM 8: AGC half window iround(2 / ((FC_START + FC_END) DT)) samples */
    const int *kill;          /* TRKILL: per-trace flags (host array of ntr), 1 = killed; NULL: none */
    int offset_mute;          /* OFFSET_MUTE 1: mute offsets >= offsetc; 2: offsets <= offsetc */
    float offsetc;
    int timewin;              /* TIMEWIN 0, or 5: surface-wave damping of the L2 residual */
    float gamma, twlength_minus;
    float src_x, src_z;       /* source position (m), for the offsets */
} dn_residual_opts;
/* The residual of one shot's recorded component against obs [ntr][nt] (host),
 * stored as the shot's adjoint source; *misfit = the objective's value. */
int dn_shot_residual_ex(dn_shot *s, int comp, const float *obs, const dn_residual_opts *o, double *misfit);
/* The same on device buffers: syn_tm [nt][ntr], obs and res [ntr][nt];
 * rec_i/rec_j (host) are the receivers' grid indices for the offsets. */
int dn_residual_ex(const float *syn_tm, const float *obs, float *res, int ntr, int nt, float dt, float dh,
                   const int *rec_i, const int *rec_j, const dn_residual_opts *o, double *misfit);

/* apply_tdfilt (src/apply_tdfilt.c, TIME_FILT and the QUELLART 6 spike band):
 * Butterworth low-pass of `order` (1..16) at corner fc_low, then, if
 * fc_high > 0, high-pass at fc_high - the recursive filters of libcseife's
 * seife_lpb/seife_hpb that timedomain_filt.c calls, in double, with the
 * reference's float conversions around each and its last sample of every
 * trace left unfiltered.  traces [ntr][ns], in place: device memory
 * (dn_tdfilt) or host memory (dn_tdfilt_host, filtered on `device`). */
int dn_tdfilt(float *traces, int ntr, int ns, float dt, int order, float fc_low, float fc_high);
int dn_tdfilt_host(float *traces, int ntr, int ns, float dt, int order, float fc_low, float fc_high, int device);

/* Per-kernel device time of `nsteps` time steps of a batch (direct launches with
 * CUDA events between kernels, for measurement only; leaves the shots' results
 * undefined).  ms_out[8] = average ms per launch of: velocity update, velocity
 * source injection, stress update, stress source injection, free surface,
 * receivers, snapshot store, cross-correlation (0 where not launched). */
int dn_profile_steps(dn_shot *const *shots, int n, int mode, int nsteps, double *ms_out);

/* ---- run queues: continuous batching ---------------------------------------
 * A queue runs shots of one FDORDER, L and arithmetic together, each at its own
 * time step, on its own CUDA stream (queues overlap on the device).  Shots join
 * and leave between chunks of `chunk` time steps.  A shot must not be destroyed
 * or run elsewhere while it is in a queue (until dn_queue_step returns it).
 * The batched launch this builds on replaces the reference's one-shot psv()
 * loop; the queue itself has no counterpart in the reference. */
typedef struct dn_queue dn_queue;
int dn_queue_create(int device, int chunk, dn_queue **out);
int dn_queue_destroy(dn_queue *q);
/* the shot runs `mode` (DN_MODE_*) from its step 1, joining at the next dn_queue_step */
int dn_queue_add(dn_queue *q, dn_shot *s, int mode);
/* Waits for the chunk in flight; returns the shots it finished (at most cap) in
 * done[0..*ndone) with their status (DN_OK, DN_EUNSTABLE); admits the added
 * shots; enqueues the next chunk and returns without waiting for it. */
int dn_queue_step(dn_queue *q, dn_shot **done, int *status, int cap, int *ndone);
int dn_queue_count(const dn_queue *q, int *running, int *waiting);

/* ---- tile shapes ------------------------------------------------------------
 * Shots created after this call whose FDORDER and L match and whose nx*ny lies in
 * [cells_min, cells_max] use tiles of bx columns (a multiple of 32, <= 256) by zch
 * rows; the last matching rule wins; the environment variable DN_TILE="WxZ"
 * overrides all rules.  Results do not depend on the tile shape. */
int dn_set_tile_shape(int fdorder, int L, long long cells_min, long long cells_max, int bx, int zch);
int dn_clear_tile_shapes(void);
/* the tile shape a new shot with these parameters gets */
int dn_get_tile_shape(const dn_params *p, int *bx, int *zch);
/* Stencil kernel variants (the register blocking of the stencil kernels; no
 * counterpart in the reference, whose loops have one form): */
#define DN_KERN_PAIRED 0   /* two adjacent columns per thread, packed FP32x2 arithmetic (default) */
#define DN_KERN_COLUMN 1   /* one column per thread, z stencils in register windows */
#define DN_KERN_VPIPE 2    /* paired, with the velocity update fed by a warp-specialised copy pipeline */
#define DN_KERN_FUSED 3    /* elastic shots without snapshots: velocity, force sources, stress,
                              explosive source and free surface of a time step in one kernel
                              (fields in two alternating buffers; other shots fall back to PAIRED) */
/* A rule as dn_set_tile_shape's, for shots that store snapshots (store 1), that
 * do not (0) or both (-1), which also picks the kernel variant (-1: default).
 * A batch runs the variant of its first shot. */
int dn_set_kernel_rule(int fdorder, int L, int store, long long cells_min, long long cells_max, int bx, int zch,
                       int variant);
/* the tile shape and kernel variant a new shot with these parameters gets */
int dn_get_kernel_choice(const dn_params *p, int *bx, int *zch, int *variant);
/* a shot's kernel variant, and 1 in *fused when its forward runs take the fused
 * elastic step (DN_KERN_FUSED and eligible: elastic, no snapshots, at most 32
 * source cells, no moment-tensor source; environment DN_FUSED=1 / 0 forces it) */
int dn_shot_kernel(const dn_shot *s, int *variant, int *fused);

/* ---- FWI outer loop (FP64) ------------------------------------------------- */
/* Deterministic FP64 dot product of two device vectors (fixed reduction order). */
int dn_dot(const double *a, const double *b, long long n, double *out);

/* L-BFGS of src/LBFGS.c (two-loop recursion, H0 = gamma I from the newest pair)
 * on device-resident FP64 vectors of length n, keeping the m newest pairs. */
typedef struct dn_lbfgs dn_lbfgs;
int dn_lbfgs_create(long long n, int m, int device, dn_lbfgs **out);
int dn_lbfgs_destroy(dn_lbfgs *L);
/* s = x_{k+1} - x_k, y = g_{k+1} - g_k (device); rho = 1/(y.s), 0 when y.s = 0 */
int dn_lbfgs_push(dn_lbfgs *L, const double *d_s, const double *d_y);
int dn_lbfgs_count(const dn_lbfgs *L, int *count);
/* r = H g (device vectors); the model update is x - eps r */
int dn_lbfgs_direction(dn_lbfgs *L, const double *d_g, double *d_r);

/* The reference's optimisers, FWI_PSV.c:637-676, on a model's stacked and
 * conditioned gradient, which the call replaces by the search direction that
 * calc_mat_change_test_PSV then applies (dn_mat_update):
 *  - grad_method 2, L-BFGS with nlbfgs pairs: the LBFGS_pointer rule of
 *    FWI_PSV.c:452-466, store_LBFGS_PSV (src/PSV/store_LBFGS_PSV.c: gradients
 *    normalised by c = {C_vp, C_vs, C_rho}, the model averages of the starting
 *    model; y and s against the previous call's normalised gradient and model),
 *    LBFGS (src/LBFGS.c) and extract_LBFGS_PSV (src/PSV/extract_LBFGS_PSV.c:
 *    the direction times c; in iteration 1 the normalised gradient);
 *  - grad_method 1, PCG with PCG_BETA pcg_beta (1 Fletcher-Reeves, 2
 *    Polak-Ribiere, 3 Hestenes-Stiefel, 4 Dai-Yuan): descent, store_PCG_PSV,
 *    PCG (src/PCG.c), extract_PCG_PSV, descent.
 * iter is FWI_PSV.c's per-stage iteration counter (1 at a stage's start).  The
 * vectors are float as in the reference; the dot products are summed in FP64.
 * The history lives on `device` (2 nlbfgs + 5 vectors of 3 nx ny floats for
 * L-BFGS, 3 for PCG).  The model (vp, vs, rho) of the step is the model `m`
 * was created from. */
typedef struct dn_optim dn_optim;
int dn_optim_create(int grad_method, int nx, int ny, int nlbfgs, int pcg_beta, int device, dn_optim **out);
int dn_optim_destroy(dn_optim *o);
/* zero_LBFGS / zero_PCG and LBFGS_pointer = 1 at a stage change (FWI_PSV.c:800-811) */
int dn_optim_reset(dn_optim *o);
int dn_optim_step(dn_optim *o, dn_model *m, int iter, const float c[3]);
/* After an L-BFGS step, the vectors extract_LBFGS_PSV writes as the JACOBIAN
 * files, in file order: which 0, 1, 2 = the normalised gradients
 * (<JACOBIAN>_p.old, _p_u.old, _p_rho.old), 3, 4, 5 = the model
 * (_p_vp.old, _p_vs.old, _p_mrho.old), 6, 7, 8 = the direction (_c.old,
 * _c_u.old, _c_rho.old).  out holds nx*ny floats. */
int dn_optim_get(const dn_optim *o, int which, float *out);

/* calc_opt_step (src/calc_opt_step.c): the step length at the extremum of the
 * parabola through (epst[k], L2t[k]), k = 0..2, with the reference's clamping
 * (beyond epst[2] or a maximum: epst[2]; negative: epst[0]); solved in FP64. */
int dn_calc_opt_step(const double L2t[3], const float epst[3], float *opteps);

/* calc_mat_change_test_PSV (INVMAT1 = 1): vp/vs/rho (file order, host) moved
 * against the direction d* by eps_scale times max(model)/max|d| per parameter
 * (rho additionally times scalerho; a parameter whose INV_*_ITER is above iter
 * stays), then values outside lim = {vp_lo, vp_hi, vs_lo, vs_hi, rho_lo,
 * rho_hi} or below 0 keep their old value (vs below vs_lo only when above
 * 1e-6).  eps_out = {EPSILON, EPSILON_u, EPSILON_rho}. */
int dn_mat_update(int nx, int ny, const float *vp, const float *vs, const float *rho, const float *dvp,
                  const float *dvs, const float *drho, float eps_scale, const float lim[6], int iter,
                  const int inv_iter[3], float scalerho, float *vp_out, float *vs_out, float *rho_out,
                  float eps_out[3]);

#ifdef __cplusplus
}
#endif

#endif
