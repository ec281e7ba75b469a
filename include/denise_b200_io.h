/*
 * denise_b200_io.h - host-side file I/O of the P-SV path: the reference's
 * parameter file, model files, source and receiver tables and SU seismograms,
 * and a forward-modelling driver that runs a parameter file end to end on the
 * GPU library (include/denise_b200.h).
 *
 * Replaces, for the P-SV forward path:
 *   read_par            src/read_par.c:15      (positional .inp reader)
 *   readmod_elastic_PSV src/PSV/readmod_elastic_PSV.c:72-85, readmod_visc_PSV (model files)
 *   sources             src/sources.c:11       (SOURCE_FILE table)
 *   receiver            src/receiver.c:11      (REC_FILE table, READREC = 1)
 *   rd_sour             src/rd_sour.c:9        (QUELLART 3 wavelet file)
 *   splitsrc            src/splitsrc.c         (source grid indices, one rank)
 *   outseis_glob        src/outseis_glob.c:12  (SU output, SEIS_FORMAT = 1)
 *   saveseis_glob       src/saveseis_glob.c    (file names per SEISMO)
 *   the MODE = 0 shot loop of FD_PSV            src/PSV/FD_PSV.c:252-360
 *
 * All functions return DN_OK or a negative DN_E* status (dn_last_error() has
 * the text); nothing exits.
 */
#ifndef DENISE_B200_IO_H
#define DENISE_B200_IO_H

#include "denise_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define DN_STR 256

/* The parameters of a DENISE .inp file.  Field names follow the reference's
 * globals; values not present keep their zero defaults (as the reference's
 * zero-initialised globals do). */
typedef struct dn_inp {
    int mode, physics, nprocx, nprocy, fdorder, maxrelerror, nx, ny;
    float dh, time, dt;
    int quellart;
    char signal_file[DN_STR];
    float ts;
    int srcrec;
    char source_file[DN_STR];
    int run_multiple_shots;
    float fc_spike_1, fc_spike_2;
    int order_spike, write_stf, readmod;
    char mfile[DN_STR];
    int writemod, L;
    float fl[DN_MAX_L + 1];    /* FL[1..L], as read (index 0 unused) */
    float tau;
    int free_surf, fw;
    float damping, fpml, npower, k_max_pml;
    int boundary, snap, snap_shot;
    float tsnap1, tsnap2, tsnapinc;
    int idx, idy, snap_format;
    char snap_file[DN_STR];
    int seismo, readrec;
    char rec_file[DN_STR];
    float refrec[4];           /* REFREC[1..2] read, [3] = 0 */
    int n_streamer;
    float rec_incr_x, rec_incr_y;
    int ndt, seis_format;
    char seis_file_vx[DN_STR], seis_file_vy[DN_STR], seis_file_curl[DN_STR], seis_file_div[DN_STR],
        seis_file_p[DN_STR], log_file[DN_STR];
    int log, itermax;
    char jacobian[DN_STR], data_dir[DN_STR];
    int taper, taperlength, gradt[5], invmat1, grad_form, quelltypb, testshot[4];
    int dtinv, lnorm;
    int lines;                 /* parameter lines counted (the reference's lineno) */
    /* lines 70-115 (inversion; read_par.c cases 70-115) */
    int sws_taper_grad_vert, sws_taper_grad_hor;
    float exp_taper_grad_hor;
    int sws_taper_grad_sources, sws_taper_circular_per_shot, srtshape;
    float srtradius;
    int filtsize, sws_taper_file;
    char tfile[DN_STR];
    int inv_mod_out;
    char inv_modelfile[DN_STR];
    float vpupperlim, vplowerlim, vsupperlim, vslowerlim, rhoupperlim, rholowerlim, qsupperlim, qslowerlim;
    int grad_method, pcg_beta, nlbfgs, model_filter, filt_size;
    float eps_scale;
    int stepmax;
    float scalefac;
    int trkill;
    char trkill_file[DN_STR], picks_file[DN_STR], misfit_log_file[DN_STR];
    int min_iter, grad_filter, filt_size_grad, timelapse;
    char data_dir_t0[DN_STR];
    int rtmod, gravity, ngravb, nzgrav, grav_type, back_density;
    char dfile[DN_STR];
    int rtm_shot;
} dn_inp;

/* read_par: the reference's positional reader.  After a newline, the next
 * character is consumed; unless it is '#', the line counter advances and the
 * line's value is scanned with the format of that line number.  So the first
 * line of the file is never a parameter line, an empty line is absorbed by the
 * scan of the line it precedes, and any other line that does not start with
 * '#' counts.  FW < 0 becomes 0. */
int dn_inp_read(const char *path, dn_inp *out);

/* NT = iround(TIME / DT) (FD_PSV.c:68) */
int dn_inp_nt(const dn_inp *in);

/* dn_params of the propagator from a parameter file (NT, FDORDER ... DTINV);
 * TS is taken from the source table when SRCREC = 1 (sources.c:90). */
int dn_inp_params(const dn_inp *in, float ts, dn_params *out);

/* One model file MFILE.<ext>: NX * NY native-endian float32, x-major
 * (readmod_elastic_PSV.c:72-85), out[(i-1)*ny + (j-1)].  A short file is an
 * error (DN_EIO) where the reference would keep reading stale values. */
int dn_read_model_file(const char *path, int nx, int ny, float *out);

/* SOURCE_FILE: first line the count, then one line per source
 * "x z y tshift fc amp [azimuth [type]]" (sources.c:49); the vertical
 * coordinate is the third column.  srcpos receives 8 floats per source in the
 * reference's srcpos[1..8] order: x, y(depth), 0, tshift, fc, amp, azimuth,
 * type.  *ts = 1 / max fc.  The caller frees *srcpos with free(). */
int dn_read_sources(const char *path, int *nsrc, float **srcpos, float *ts);

/* rd_sour (src/rd_sour.c): the wavelet file of QUELLART 3,
 * "<SIGNAL_FILE>_shot_<n>.dat", one sample per line; *ns = the number of
 * newlines.  The caller frees *samples with free(). */
int dn_read_signal_file(const char *path, int *ns, float **samples);

/* Source grid indices of one rank (splitsrc.c): iround(x / DH), iround(y / DH). */
int dn_source_cell(float x, float y, float dh, int *i, int *j);

/* REC_FILE.dat: "x y" per line, counted by newlines (receiver.c:36-48);
 * grid index iround((x + REFREC[1]) / DH); receivers sharing a grid point,
 * and those at x index <= 0, are dropped as receiver.c:63-83 does.  The caller
 * frees *rec_i / *rec_j. */
int dn_read_receivers(const char *path, const float refrec[4], float dh, int *ntr, int **rec_i, int **rec_j);

/* outseis_glob, SEIS_FORMAT 1 (SU): one 240-byte header + ns float samples per
 * trace, samples NDT, 2 NDT, ... of section[ntr][nt] (sws = 1).  xs, ys: the
 * shot's source position in metres.  Header bytes the reference leaves
 * unassigned (210-239) are written as zero. */
int dn_write_su(const char *path, const float *section, int ntr, int nt, int ndt, float dt, float time, float dh,
                const int *rec_i, const int *rec_j, const float refrec[4], float xs, float ys);
/* The seismogram file of one component in SEIS_FORMAT `format` (outseis_glob.c):
 * 1 SU (dn_write_su), 2 ASCII one value per line ("%e"), 3 raw native float32,
 * trace after trace; the same NDT-decimated samples in every format. */
int dn_write_seis(const char *path, int format, const float *section, int ntr, int nt, int ndt, float dt, float time,
                  float dh, const int *rec_i, const int *rec_j, const float refrec[4], float xs, float ys);

/* SU reader for observed data (inseis.c): ntr traces of ns samples each. */
int dn_read_su(const char *path, int ntr, int ns, float *section);

/* MODE 0 of FD_PSV for a parameter file: models, sources, receivers, wavelets
 * (QUELLART 1-7; 3 from "<SIGNAL_FILE>_shot_<n>.dat", the spike of 6
 * band-limited by ORDER_SPIKE, FC_SPIKE_2, FC_SPIKE_1); one shot per line of the source table, firing that
 * source (RUN_MULTIPLE_SHOTS = 1) or all sources (0), as count_src.c and
 * FD_PSV.c:252-300 do; the shots run as batches on `device` and the
 * seismograms are written as saveseis_glob names them (SEIS_FILE_*.shot<n>).
 * Paths in the file are relative to the current directory, as in the
 * reference. */
int dn_forward_inp(const char *inp_path, int device);

#ifdef __cplusplus
}
#endif

#endif
