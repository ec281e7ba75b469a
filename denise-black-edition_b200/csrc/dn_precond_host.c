/* Host set-up of the gradient conditioning: the taper coefficients of
 * taper_grad.c / taper_grad_shot.c, the zeroed source boxes, the smooth2
 * factorisation and the Gaussian weights of gauss_filt.c / gauss_filt_var.c.
 *
 * These depend only on the geometry and the .inp switches, so they are
 * computed once on the host (compiled with -ffp-contract=off, calling the C
 * library's exp, erf, log and pow as the reference does, in the same float and
 * double steps), and the device applies them to the gradients.  Arrays are
 * row-major [j][i] (row j = depth), 0-based: element (j, i) at (j-1)*nx + i-1.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "dn_precond.h"

/* util.c minimum_m/maximum_m: the scan starts at the first element and keeps
 * strict improvements, so a NaN is only ever chosen as the first element. */
static float scan_min(const float *a, size_t n)
{
    float m = a[0];
    for (size_t k = 1; k < n; k++)
        if (a[k] < m) m = a[k];
    return m;
}
static float scan_max(const float *a, size_t n)
{
    float m = a[0];
    for (size_t k = 1; k < n; k++)
        if (a[k] > m) m = a[k];
    return m;
}

/* exp(-(1.0/2.0) * (a*k/(tl/2.0)) * (a*k/(tl/2.0))) with float a = 3 and int k
 * (taper_grad.c:74, :79): a*k in float, the rest in double, stored as float. */
static float gauss_ramp(int k, int tl)
{
    const float a = 3.0f;
    const float ak = a * (float)k;
    const double x = (double)ak / ((double)tl / 2.0);
    return (float)exp(-(1.0 / 2.0) * x * x);
}

void dnp_taper_vertical_row(int nx, const int gradt[4], float *row)
{
    const int g1 = gradt[0], g2 = gradt[1], g3 = gradt[2], g4 = gradt[3];
    const int tl = g2 - g1, tl2 = g4 - g3, ifw = g4 - g1;
    float *win = (float *)calloc((size_t)(ifw > 0 ? ifw : 0) + 1, sizeof(float));
    for (int i = 1; i <= ifw; i++) {
        win[i] = 1.0f;
        if (i <= tl) win[i] = gauss_ramp(i - tl, tl);
        if (i >= ifw - tl2) win[i] = gauss_ramp(i - (ifw - tl2), tl2);
    }
    int h = 1;
    for (int i = 1; i <= nx; i++) {
        float t = 0.0f;
        if (i > g1 && i < g4) t = win[h++];
        row[i - 1] = t;
    }
    free(win);
}

void dnp_taper_horizontal_col(int ny, float dh, const int gradt[4], float exp_hor, float *col)
{
    const int g1 = gradt[0], g2 = gradt[1];
    const int tl = g2 - g1, ifw = g2 - g1 + 1;
    float *win = (float *)calloc((size_t)(ifw > 0 ? ifw : 0) + 1, sizeof(float));
    for (int i = 1; i <= ifw; i++) {
        win[i] = 1.0f;
        if (i <= tl) win[i] = gauss_ramp(i - tl, tl);
    }
    int h = 1;
    for (int j = 1; j <= ny; j++) {
        float t = 0.0f;
        if (j >= g1 && j <= g2) t = win[h];
        if (j > g2) t = (float)pow((float)(j * dh), exp_hor);
        col[j - 1] = t;
        if (j >= g1) h++;
    }
    free(win);
}

int dnp_source_matrix(int srtshape, float srtradius, float dh, float **m_out, int *G_out, int *ijc_out)
{
    int G = (int)(ceil(2.0 * srtradius / dh));
    if (G < 5) G = 5;
    float *m = (float *)calloc((size_t)G * G, sizeof(float));
    if (!m) return -1;
    const float a = 1.0f;
    const float maxrad = (float)sqrt(2.0 * srtradius * srtradius);
    for (int j = 1; j <= G; j++)
        for (int i = 1; i <= G; i++) {
            const float x = (float)(((float)i - ((float)G) / 2.0 - 0.5) * dh);
            const float y = (float)(((float)j - ((float)G) / 2.0 - 0.5) * dh);
            const float rad = (float)sqrt(x * x + y * y);
            float v = 0.0f;
            if (srtshape == 1) v = (float)erf(a * rad / maxrad);
            if (srtshape == 2) v = rad > 0 ? (float)log(rad) : 0.0f;
            m[(size_t)(j - 1) * G + (i - 1)] = v;
        }
    /* minimum over the matrix: minimum_m scans x outer, z inner; the first
     * element is m[1][1] either way and min does not depend on the order */
    const float minm = scan_min(m, (size_t)G * G);
    for (size_t k = 0; k < (size_t)G * G; k++) m[k] -= minm;
    const int h = G / 2;
    const float edge[4] = {m[(size_t)0 * G + (h - 1)], m[(size_t)(h - 1) * G + 0], m[(size_t)(h - 1) * G + (G - 1)],
                           m[(size_t)(G - 1) * G + (h - 1)]};
    const float maxm = scan_max(edge, 4);
    for (size_t k = 0; k < (size_t)G * G; k++) {
        m[k] /= maxm;
        if (m[k] > 1.0) m[k] = 1.0f;
    }
    *m_out = m;
    *G_out = G;
    *ijc_out = (int)(ceil((float)G / 2));
    return 0;
}

void dnp_source_cell(float x, float z, float dh, int *i, int *j)
{
    *i = (int)floor(x / dh + 0.5);
    *j = (int)floor(z / dh + 0.5);
}

/* (msum - min) / max over the grid (taper_grad.c:458-479), in place */
static void normalise(float *msum, size_t n)
{
    const float minm = scan_min(msum, n);
    for (size_t k = 0; k < n; k++) msum[k] -= minm;
    const float maxm = scan_max(msum, n);
    for (size_t k = 0; k < n; k++) msum[k] = msum[k] / maxm;
}

int dnp_taper_sources(int nx, int ny, float dh, int srtshape, float srtradius, int nsrc, const float *src_x,
                      const float *src_z, float *coeff)
{
    float *m;
    int G, ijc;
    if (dnp_source_matrix(srtshape, srtradius, dh, &m, &G, &ijc)) return -1;
    const size_t n = (size_t)nx * ny;
    for (size_t k = 0; k < n; k++) coeff[k] = 1.0f;
    for (int s = 0; s < nsrc; s++) {
        int i, j;
        dnp_source_cell(src_x[s], src_z[s], dh, &i, &j);
        /* msum = min(msum, mm) with mm = 1 outside the box: only box cells can lower it */
        for (int iy = 1; iy <= G; iy++)
            for (int ix = 1; ix <= G; ix++) {
                const int xx = i + ix - ijc, yy = j + iy - ijc;
                if (xx < 1 || xx > nx || yy < 1 || yy > ny) continue;
                float *c = &coeff[(size_t)(yy - 1) * nx + (xx - 1)];
                const float v = m[(size_t)(iy - 1) * G + (ix - 1)];
                if (*c > v) *c = v;
            }
    }
    free(m);
    normalise(coeff, n);
    return 0;
}

int dnp_shot_taper(int nx, int ny, float dh, int srtshape, float srtradius, float src_x, float src_z,
                   dnp_shot_taper_t *t)
{
    float *m;
    int G, ijc;
    if (dnp_source_matrix(srtshape, srtradius, dh, &m, &G, &ijc)) return -1;
    int i, j;
    dnp_source_cell(src_x, src_z, dh, &i, &j);
    /* msum (taper_grad_shot.c) is 1 where the box does not reach and min(1, m)
     * inside it, never NaN, so its minimum and maximum over the grid do not
     * depend on the scan order and follow from the box alone; the device
     * evaluates (msum - minm) / maxm per cell */
    long long covered = 0;
    for (int iy = 1; iy <= G; iy++)
        for (int ix = 1; ix <= G; ix++) {
            const int xx = i + ix - ijc, yy = j + iy - ijc;
            float *v = &m[(size_t)(iy - 1) * G + (ix - 1)];
            if (xx < 1 || xx > nx || yy < 1 || yy > ny) {
                *v = 1.0f;   /* not used: outside the grid */
                continue;
            }
            covered++;
            const float one = 1.0f;
            *v = one > *v ? *v : one;
        }
    const int uncovered = covered < (long long)nx * ny;
    float minm = 1.0f, maxv = 1.0f;
    int first = 1;
    for (int iy = 1; iy <= G; iy++)
        for (int ix = 1; ix <= G; ix++) {
            const int xx = i + ix - ijc, yy = j + iy - ijc;
            if (xx < 1 || xx > nx || yy < 1 || yy > ny) continue;
            const float v = m[(size_t)(iy - 1) * G + (ix - 1)];
            if (first || v < minm) minm = v;
            if (first || v > maxv) maxv = v;
            first = 0;
        }
    if (uncovered) {
        if (first || 1.0f < minm) minm = 1.0f;
        if (first || 1.0f > maxv) maxv = 1.0f;
    }
    /* max(msum - minm) = the largest msum minus minm: float subtraction of a
     * constant is monotone */
    t->G = G;
    t->x0 = i + 1 - ijc;   /* grid column of box column 1 */
    t->z0 = j + 1 - ijc;
    t->m = m;
    t->minm = minm;
    t->maxm = maxv - minm;
    return 0;
}

/* C division truncates towards zero: (i - 1) / n == 0 <=> 2 - n <= i <= n */
static int same_block(int i, int n) { return (i - 1) / n == 0; }

int dnp_zero_cells(int nx, int ny, int npts, const int *pi, const int *pj, int size, int need_row, int **cells,
                   int *ncells)
{
    const int ncol = nx + 2;   /* waveconvtmp = matrix(0, NY+1, 0, NX+1): rows of NX + 2 floats */
    const int box = (2 * size + 1) * (2 * size + 1);
    int *c = (int *)malloc(sizeof(int) * ((size_t)npts * box + 1));
    if (!c) return -1;
    int k = 0;
    for (int p = 0; p < npts; p++)
        for (int i = pi[p] - size; i <= pi[p] + size; i++)
            for (int j = pj[p] - size; j <= pj[p] + size; j++) {
                if (!same_block(i, nx) || !same_block(j, ny)) continue;
                if (need_row && j <= 0) continue;
                /* an index left of column 0 lands in the previous row of the block */
                const long long off = (long long)j * ncol + i;
                long long r = off / ncol, col = off % ncol;
                if (col < 0) {
                    col += ncol;
                    r -= 1;
                }
                if (r < 1 || r > ny || col < 1 || col > nx) continue;
                c[k++] = (int)((r - 1) * nx + (col - 1));
            }
    *cells = c;
    *ncells = k;
    return 0;
}

/* `1.0 + x` with float x, stored as float (the sum in double, rounded once) */
static float one_plus(float x) { return (float)(1.0 + x); }

/* util.c tripd, decomposition part, on constant-coefficient systems */
static void tripd_factor(float *d, float *e, int n)
{
    for (int k = 1; k < n; k++) {
        const float t = e[k - 1];
        e[k - 1] = t / d[k - 1];
        d[k] -= t * e[k - 1];
    }
}

int dnp_smooth2_factor(int nx, int ny, float wd_damp, float wd_damp1, dnp_smooth2_t *s)
{
    const float w = 1.0f;
    float r1 = wd_damp, r2 = wd_damp1;
    r1 = r1 * r1 * 0.25;
    r2 = r2 * r2 * 0.25;
    const int n2 = nx, n1 = ny - 1;
    s->nx_line = n2;
    s->nz_line = n1;
    s->dx = (float *)calloc((size_t)n2, sizeof(float));
    s->ex = (float *)calloc((size_t)n2, sizeof(float));
    s->dz = (float *)malloc(sizeof(float) * (n1 > 0 ? n1 : 1));
    s->ez = (float *)malloc(sizeof(float) * (n1 > 0 ? n1 : 1));
    if (!s->dx || !s->ex || !s->dz || !s->ez) return -1;
    /* along x (smooth2.c:138-150): d = 1 + 2 r2 (first: minus r2, last: 1 + r2), e = -r2 */
    for (int k = 0; k < n2 - 1; k++) {
        s->dx[k] = one_plus(r2 * (w + w));
        s->ex[k] = -r2 * w;
    }
    s->dx[0] -= r2 * w;
    s->dx[n2 - 1] = one_plus(r2 * w);
    s->ex[n2 - 1] = 0.0f;
    tripd_factor(s->dx, s->ex, n2);
    /* along z (smooth2.c:151-163): n1 = NY - 1 unknowns, rows 1..NY-1 */
    for (int k = 0; k < n1 - 1; k++) {
        s->dz[k] = one_plus(r1 * (w + w));
        s->ez[k] = -r1 * w;
    }
    if (n1 > 0) {
        s->dz[n1 - 1] = one_plus(r1 * w);
        s->ez[n1 - 1] = 0.0f;
        tripd_factor(s->dz, s->ez, n1);
    }
    s->r1w = r1 * w;
    return 0;
}

void dnp_smooth2_free(dnp_smooth2_t *s)
{
    free(s->dx);
    free(s->ex);
    free(s->dz);
    free(s->ez);
    memset(s, 0, sizeof *s);
}

int dnp_gauss_size(float wd, float vel, float fc_end, float dh)
{
    const float lam = vel / fc_end;
    return (int)round((wd * lam) / dh);
}

float dnp_gauss_kernel(int hx, int hz, float *k)
{
    const float sigx = (float)(hx / 2), sigz = (float)(hz / 2);
    const float sx = 2.0 * sigx * sigx, sz = 2.0 * sigz * sigz;
    float sum = 0.0f;
    const int nz = 2 * hz + 1;
    for (int ii = -hx; ii <= hx; ii++)
        for (int jj = -hz; jj <= hz; jj++) {
            const float v = (float)exp(-((ii * ii) / sx) - ((jj * jj) / sz));
            k[(size_t)(ii + hx) * nz + (jj + hz)] = v;
            sum += v;
        }
    return sum;
}
