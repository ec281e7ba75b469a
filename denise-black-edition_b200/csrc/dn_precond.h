/* Host set-up of the gradient conditioning (dn_precond_host.c), used by the
 * device side in dn_precond.cu and dn_engine.cu.  Arrays are row-major [j][i],
 * element (j, i) of the 1-based grid at (j-1)*nx + (i-1). */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

/* taper_grad sws 1: the vertical taper's coefficient of column i (the same on every row) */
void dnp_taper_vertical_row(int nx, const int gradt[4], float *row);
/* taper_grad sws 2: the horizontal taper's coefficient of row j */
void dnp_taper_horizontal_col(int ny, float dh, const int gradt[4], float exp_hor, float *col);
/* the G x G radial taper around a source ([iy-1][ix-1], malloc'ed) and its centre ijc */
int dnp_source_matrix(int srtshape, float srtradius, float dh, float **m, int *G, int *ijc);
/* iround(srcpos / DH) */
void dnp_source_cell(float x, float z, float dh, int *i, int *j);
/* taper_grad sws 3 coefficients over the grid (minimum over sources, normalised) */
int dnp_taper_sources(int nx, int ny, float dh, int srtshape, float srtradius, int nsrc, const float *src_x,
                      const float *src_z, float *coeff);

/* taper_grad_shot of one source: coefficient (msum - minm) / maxm with msum = m
 * inside the G x G box whose column 1 / row 1 sit at grid column x0 / row z0,
 * 1 elsewhere */
typedef struct {
    int G, x0, z0;
    float *m;       /* malloc'ed, [iy-1][ix-1] */
    float minm, maxm;
} dnp_shot_taper_t;
int dnp_shot_taper(int nx, int ny, float dh, int srtshape, float srtradius, float src_x, float src_z,
                   dnp_shot_taper_t *t);

/* Interior cells (0-based row-major indices) that the reference's
 * `waveconvtmp[jj][ii] = 0` loops over (2 size + 1)^2 boxes around the points
 * reach (need_row: the loop also requires jj > 0).  malloc'ed. */
int dnp_zero_cells(int nx, int ny, int npts, const int *pi, const int *pj, int size, int need_row, int **cells,
                   int *ncells);

/* smooth2: the factored constant-coefficient systems along x (NX unknowns per
 * row) and along z (NY - 1 unknowns per column) */
typedef struct {
    int nx_line, nz_line;
    float *dx, *ex, *dz, *ez;
    float r1w;      /* r1 * w of the z boundary term */
} dnp_smooth2_t;
int dnp_smooth2_factor(int nx, int ny, float wd_damp, float wd_damp1, dnp_smooth2_t *s);
void dnp_smooth2_free(dnp_smooth2_t *s);

/* round((wd * (vel / fc_end)) / dh) in float, as gauss_filt(_var) size their filters */
int dnp_gauss_size(float wd, float vel, float fc_end, float dh);
/* Gaussian weights k[(ii+hx)*(2hz+1) + (jj+hz)] and their float sum in the
 * reference's loop order (ii outer, jj inner) */
float dnp_gauss_kernel(int hx, int hz, float *k);

#ifdef __cplusplus
}
#endif
