// Gradient conditioning on the device: smooth_grad (src/smooth_grad.c) and
// precond_PSV (src/PSV/precond_PSV.c) applied to a model's stacked gradients,
// FWI_PSV.c:628-634.
//
// The plan holds what depends on the geometry only, computed once on the host
// by dn_precond_host.c: the taper coefficients (a row vector for the vertical
// taper, a column vector for the horizontal one, a grid for the source taper
// and for each class of the file taper), a byte per cell marking the cells the
// reference zeroes after the vertical taper (bit 0) and after the source taper
// (bit 1), the factored smooth2 systems and the gauss_filt weights.  Applying it
// is one pass per class for the tapers (the per-cell operations in the
// reference's order) plus the smoothing kernels.  The float path repeats the
// reference's float operations with explicit round-to-nearest intrinsics, so a
// float gradient comes out bit-identical to the reference's; a double gradient
// (DN_ACC_F64 models) is conditioned with the same steps in double.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "denise_b200.h"
#include "dn_internal.h"
#include "dn_precond.h"

namespace {

template <typename T> __device__ __forceinline__ T mulr(T a, T b) { return a * b; }
template <> __device__ __forceinline__ float mulr(float a, float b) { return __fmul_rn(a, b); }
template <typename T> __device__ __forceinline__ T addr(T a, T b) { return a + b; }
template <> __device__ __forceinline__ float addr(float a, float b) { return __fadd_rn(a, b); }
template <typename T> __device__ __forceinline__ T subr(T a, T b) { return a - b; }
template <> __device__ __forceinline__ float subr(float a, float b) { return __fsub_rn(a, b); }
template <typename T> __device__ __forceinline__ T divr(T a, T b) { return a / b; }
template <> __device__ __forceinline__ float divr(float a, float b) { return __fdiv_rn(a, b); }

// precond_PSV for one class: vertical taper (times row coefficient, zero bit 0),
// horizontal (times column coefficient), sources (times grid coefficient, zero
// bit 1), file (times the class's grid coefficient)
template <typename T>
__global__ void k_tapers(T *g, int nx, int ny, const float *vrow, const float *hcol, const float *src,
                         const float *file, const unsigned char *mask)
{
    const long long n = (long long)nx * ny;
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n; w += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(w / nx), i = (int)(w % nx);
        const unsigned char z = mask ? mask[w] : 0;
        T v = g[w];
        if (vrow) {
            v = mulr<T>(v, (T)vrow[i]);
            if (z & 1) v = (T)0;
        }
        if (hcol) v = mulr<T>(v, (T)hcol[j]);
        if (src) {
            v = mulr<T>(v, (T)src[w]);
            if (z & 2) v = (T)0;
        }
        if (file) v = mulr<T>(v, (T)file[w]);
        g[w] = v;
    }
}

// smooth2 along x (smooth2.c:138-150): row j (1 .. NY-1) is the line
// [0, g(j,1), ..., g(j,NX-1)] of NX unknowns; forward and back substitution
// with the factored (d, e) of util.c tripd, in place.  Position 0 (a zero
// column of the reference's work array) stays in a register and the last
// column is not part of the line.
template <typename T>
__global__ void k_smooth2_x(T *g, int nx, int ny, const float *d, const float *e)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (j > ny - 1) return;
    T *r = g + (long long)(j - 1) * nx - 1;   // r[k] = line position k, k >= 1
    const int n = nx;
    T b0 = (T)0, prev = b0;
    for (int k = 1; k < n; k++) {
        const T v = subr<T>(r[k], mulr<T>((T)e[k - 1], prev));
        r[k] = v;
        prev = v;
    }
    T next = divr<T>(r[n - 1], (T)d[n - 1]);
    r[n - 1] = next;
    for (int k = n - 1; k > 1; k--) {
        const T v = subr<T>(divr<T>(r[k - 1], (T)d[k - 1]), mulr<T>((T)e[k - 1], next));
        r[k - 1] = v;
        next = v;
    }
}

// smooth2 along z (smooth2.c:151-163): column i (1 .. NX-1), unknowns rows
// 1 .. NY-1, the zero row above as boundary (f[0] += r1 w v[0])
template <typename T>
__global__ void k_smooth2_z(T *g, int nx, int ny, const float *d, const float *e, float r1w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (i > nx - 1) return;
    const int n = ny - 1;
    T *c = g + (i - 1);
    const long long P = nx;
    T prev = addr<T>(c[0], mulr<T>((T)r1w, (T)0));
    c[0] = prev;
    for (int k = 1; k < n; k++) {
        const T v = subr<T>(c[k * P], mulr<T>((T)e[k - 1], prev));
        c[k * P] = v;
        prev = v;
    }
    T next = divr<T>(c[(n - 1) * P], (T)d[n - 1]);
    c[(n - 1) * P] = next;
    for (int k = n - 1; k > 0; k--) {
        const T v = subr<T>(divr<T>(c[(k - 1) * P], (T)d[k - 1]), mulr<T>((T)e[k - 1], next));
        c[(k - 1) * P] = v;
        next = v;
    }
}

// gauss_filt (gauss_filt.c:128-145): normalised (2h+1)^2 kernel k[(ii+h)(2h+1) + jj+h],
// sum in the reference's order (x offset outer, z offset inner), edge-replicated input
template <typename T>
__global__ void k_gauss(const T *in, T *out, int nx, int ny, int h, const float *k)
{
    const long long n = (long long)nx * ny;
    const int nk = 2 * h + 1;
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n; w += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(w / nx), i = (int)(w % nx);
        T conv = (T)0;
        for (int ii = -h; ii <= h; ii++) {
            const int x = min(max(i + ii, 0), nx - 1);
            for (int jj = -h; jj <= h; jj++) {
                const int z = min(max(j + jj, 0), ny - 1);
                conv = addr<T>(conv, mulr<T>(in[(long long)z * nx + x], (T)k[(ii + h) * nk + (jj + h)]));
            }
        }
        out[w] = conv;
    }
}

// gauss_filt_var (gauss_filt_var.c:140-183): per cell sizes from the local S
// wavelength; weights of the size pair (hx, hz) at tab + off[(hx-3)*(HZ-2) + hz-3],
// their sum at sums[...]; sizes outside the table (a NaN or negative velocity)
// leave the cell as it is and raise *flag
template <typename T>
__global__ void k_gauss_var(const T *in, T *out, int nx, int ny, const float *vs, int pitch, float wd, float wd1,
                            float fc_end, float dh, int HX, int HZ, const float *tab, const long long *off,
                            const float *sums, int *flag)
{
    const long long n = (long long)nx * ny;
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n; w += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(w / nx), i = (int)(w % nx);
        const float vel = vs[(long long)(j + 1) * pitch + (i + 1)];
        const float lam = __fdiv_rn(vel, fc_end);
        const float qx = __fdiv_rn(__fmul_rn(wd, lam), dh), qz = __fdiv_rn(__fmul_rn(wd1, lam), dh);
        if (!(fabsf(qx) < 1e8f) || !(fabsf(qz) < 1e8f)) {
            out[w] = in[w];
            atomicOr(flag, 1);
            continue;
        }
        int fx = (int)roundf(qx), fz = (int)roundf(qz);
        if (fz <= 0) {
            out[w] = in[w];
            continue;
        }
        if (!(fx % 2)) fx += 1;
        if (!(fz % 2)) fz += 1;
        fx = max(fx, 6);
        fz = max(fz, 6);
        const int hx = abs(fx) / 2, hz = abs(fz) / 2;
        if (hx > HX || hz > HZ) {
            out[w] = in[w];
            atomicOr(flag, 1);
            continue;
        }
        const int p = (hx - 3) * (HZ - 2) + (hz - 3);
        const float *k = tab + off[p];
        const int nk = 2 * hz + 1;
        T conv = (T)0;
        for (int ii = -hx; ii <= hx; ii++) {
            const int x = min(max(i + ii, 0), nx - 1);
            for (int jj = -hz; jj <= hz; jj++) {
                const int z = min(max(j + jj, 0), ny - 1);
                conv = addr<T>(conv, mulr<T>(in[(long long)z * nx + x], (T)k[(ii + hx) * nk + (jj + hz)]));
            }
        }
        out[w] = divr<T>(conv, (T)sums[p]);
    }
}

__global__ void k_max_bits(const float *vs, int pitch, int nx, int ny, unsigned *out)
{
    const long long n = (long long)nx * ny;
    unsigned m = 0;
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n; w += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(w / nx), i = (int)(w % nx);
        const float v = vs[(long long)(j + 1) * pitch + (i + 1)];
        if (v > 0.0f) m = max(m, __float_as_uint(v));   // positive floats order like their bits
    }
    atomicMax(out, m);
}

int grid_blocks(long long n) { return (int)std::min<long long>((n + 255) / 256, 148 * 16); }

}   // namespace

struct dn_precond_plan {
    int nx = 0, ny = 0, device = 0;
    float dh = 0.0f;
    dn_precond c;                      // scalars; the array pointers are not kept
    float *vrow = nullptr, *hcol = nullptr, *src = nullptr, *file[3] = {nullptr, nullptr, nullptr};
    unsigned char *mask = nullptr;
    float *dx = nullptr, *ex = nullptr, *dz = nullptr, *ez = nullptr;
    float r1w = 0.0f;
    int gauss_h = -1;                  // SPATFILTER 3: half size, -1 = no smoothing (filter size 0)
    float *gk = nullptr;
    // SPATFILTER 4 weight table for sizes up to (HX, HZ), rebuilt when they change
    mutable int HX = 0, HZ = 0;
    mutable float *tab = nullptr, *sums = nullptr;
    mutable long long *off = nullptr;
    mutable int *flag = nullptr;
    mutable unsigned *maxbits = nullptr;
    mutable void *scratch = nullptr;   // one class, float or double
    cudaStream_t stream = nullptr;
};

static int upload(void **dst, const void *src, size_t bytes)
{
    if (dn_malloc(dst, bytes) != cudaSuccess) return dn_fail(DN_ENOMEM, "gradient conditioning: %zu bytes", bytes);
    if (cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
        return dn_fail(DN_EDEVICE, "gradient conditioning: copy to the device failed");
    return DN_OK;
}

static int validate(int nx, int ny, float dh, const dn_precond *c)
{
    if (!c) return dn_fail(DN_EINVAL, "null conditioning parameters");
    if (nx < 2 || ny < 3 || !(dh > 0.0f)) return dn_fail(DN_EINVAL, "gradient conditioning: grid %d x %d, DH %g", nx, ny, dh);
    if (c->spatfilter == 1)
        return dn_fail(DN_ENOTSUP, "SPATFILTER 1 (wavenumber damping) needs FFTW, which this library does not use");
    if (c->spatfilter < 0 || c->spatfilter > 4) return dn_fail(DN_EINVAL, "SPATFILTER %d", c->spatfilter);
    if ((c->spatfilter == 3 || c->spatfilter == 4) && !(c->fc_end > 0.0f))
        return dn_fail(DN_EINVAL, "gauss_filt needs FC_END > 0 (got %g)", c->fc_end);
    if (c->spatfilter == 4 && (c->wd_damp < 0.0f || c->wd_damp1 < 0.0f))
        return dn_fail(DN_EINVAL, "gauss_filt_var needs WD_DAMP, WD_DAMP1 >= 0");
    // GRADT1..4 need no check: the taper windows are only read at indices the
    // loops of taper_grad.c reach for any values (an empty ramp reads nothing)
    if (c->taper_sources && c->srtshape != 1 && c->srtshape != 2)
        return dn_fail(DN_EINVAL, "SRTSHAPE must be 1 or 2 (got %d)", c->srtshape);
    if (c->taper_sources && (!(c->srtradius >= 0.0f) || c->srtradius > 1e6f || c->filtsize < 0 || c->filtsize > 1000))
        return dn_fail(DN_EINVAL, "SRTRADIUS %g / FILTSIZE %d out of range", c->srtradius, c->filtsize);
    if ((c->taper_vert || c->taper_sources) && c->nsrc > 0 && (!c->src_x || !c->src_z))
        return dn_fail(DN_EINVAL, "source positions missing");
    if (c->taper_vert && c->ntr > 0 && (!c->rec_i || !c->rec_j)) return dn_fail(DN_EINVAL, "receiver positions missing");
    if (c->taper_file && (!c->taper_vp || !c->taper_vs || !c->taper_rho))
        return dn_fail(DN_EINVAL, "SWS_TAPER_FILE needs the three taper arrays");
    return DN_OK;
}

extern "C" int dn_taper_coefficients(int nx, int ny, float dh, const dn_precond *c, int sws, float *coeff)
{
    int st = validate(nx, ny, dh, c);
    if (st) return st;
    if (!coeff || sws < 1 || sws > 3) return dn_fail(DN_EINVAL, "dn_taper_coefficients: sws must be 1, 2 or 3");
    std::vector<float> rm((size_t)nx * ny);
    if (sws == 1) {
        std::vector<float> row(nx);
        dnp_taper_vertical_row(nx, c->gradt, row.data());
        for (int j = 0; j < ny; j++) std::copy(row.begin(), row.end(), rm.begin() + (size_t)j * nx);
    } else if (sws == 2) {
        std::vector<float> col(ny);
        dnp_taper_horizontal_col(ny, dh, c->gradt, c->exp_taper_grad_hor, col.data());
        for (int j = 0; j < ny; j++) std::fill(rm.begin() + (size_t)j * nx, rm.begin() + (size_t)(j + 1) * nx, col[j]);
    } else {
        if (c->srtshape != 1 && c->srtshape != 2) return dn_fail(DN_EINVAL, "SRTSHAPE must be 1 or 2");
        if (dnp_taper_sources(nx, ny, dh, c->srtshape, c->srtradius, c->nsrc, c->src_x, c->src_z, rm.data()))
            return dn_fail(DN_ENOMEM, "dn_taper_coefficients");
    }
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) coeff[(size_t)i * ny + j] = rm[(size_t)j * nx + i];
    return DN_OK;
}

extern "C" int dn_precond_destroy(dn_precond_plan *p)
{
    if (!p) return DN_OK;
    cudaSetDevice(p->device);
    if (p->stream) cudaStreamSynchronize(p->stream);
    void *bufs[] = {p->vrow, p->hcol, p->src, p->file[0], p->file[1], p->file[2], p->mask, p->dx, p->ex, p->dz,
                    p->ez, p->gk, p->tab, p->sums, p->off, p->flag, p->maxbits, p->scratch};
    for (void *b : bufs) dn_free(b);
    if (p->stream) cudaStreamDestroy(p->stream);
    delete p;
    return DN_OK;
}

extern "C" int dn_precond_create(int nx, int ny, float dh, const dn_precond *c, int device, dn_precond_plan **out)
{
    if (!out) return dn_fail(DN_EINVAL, "dn_precond_create: null output");
    *out = nullptr;
    int st = validate(nx, ny, dh, c);
    if (st) return st;
    CU(cudaSetDevice(device));
    dn_precond_plan *p = new dn_precond_plan();
    p->nx = nx;
    p->ny = ny;
    p->dh = dh;
    p->device = device;
    p->c = *c;
    p->c.taper_vp = p->c.taper_vs = p->c.taper_rho = nullptr;
    p->c.src_x = p->c.src_z = nullptr;
    p->c.rec_i = p->c.rec_j = nullptr;
    const size_t n = (size_t)nx * ny;
    auto fail = [&](int code) {
        dn_precond_destroy(p);
        return code;
    };
    if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(dn_fail(DN_EDEVICE, "dn_precond_create: stream"));
    std::vector<unsigned char> mask(n, 0);
    bool any_zero = false;
    std::vector<int> si(c->nsrc), sj(c->nsrc);
    for (int s = 0; s < c->nsrc; s++) dnp_source_cell(c->src_x[s], c->src_z[s], dh, &si[s], &sj[s]);
    auto mark = [&](int npts, const int *pi, const int *pj, int size, int need_row, unsigned char bit) {
        int *cells = nullptr, nc = 0;
        if (dnp_zero_cells(nx, ny, npts, pi, pj, size, need_row, &cells, &nc)) return false;
        for (int k = 0; k < nc; k++) mask[cells[k]] |= bit;
        any_zero = any_zero || nc > 0;
        free(cells);
        return true;
    };
    if (c->taper_vert) {
        std::vector<float> row(nx);
        dnp_taper_vertical_row(nx, c->gradt, row.data());
        if ((st = upload((void **)&p->vrow, row.data(), sizeof(float) * nx))) return fail(st);
        // taper_grad.c:113-160: the source cells, then the receiver cells
        if (!mark(c->nsrc, si.data(), sj.data(), 0, 0, 1) || !mark(c->ntr, c->rec_i, c->rec_j, 0, 0, 1))
            return fail(dn_fail(DN_ENOMEM, "dn_precond_create"));
    }
    if (c->taper_hor) {
        std::vector<float> col(ny);
        dnp_taper_horizontal_col(ny, dh, c->gradt, c->exp_taper_grad_hor, col.data());
        if ((st = upload((void **)&p->hcol, col.data(), sizeof(float) * ny))) return fail(st);
    }
    if (c->taper_sources) {
        std::vector<float> co(n);
        if (dnp_taper_sources(nx, ny, dh, c->srtshape, c->srtradius, c->nsrc, c->src_x, c->src_z, co.data()))
            return fail(dn_fail(DN_ENOMEM, "dn_precond_create"));
        if ((st = upload((void **)&p->src, co.data(), sizeof(float) * n))) return fail(st);
        if (!mark(c->nsrc, si.data(), sj.data(), c->filtsize, 1, 2)) return fail(dn_fail(DN_ENOMEM, "dn_precond_create"));
    }
    if (c->taper_file) {
        const float *tf[3] = {c->taper_vp, c->taper_vs, c->taper_rho};
        std::vector<float> rm(n);
        for (int k = 0; k < 3; k++) {
            for (int i = 0; i < nx; i++)
                for (int j = 0; j < ny; j++) rm[(size_t)j * nx + i] = tf[k][(size_t)i * ny + j];
            if ((st = upload((void **)&p->file[k], rm.data(), sizeof(float) * n))) return fail(st);
        }
    }
    if (any_zero && (st = upload((void **)&p->mask, mask.data(), n))) return fail(st);
    if (c->spatfilter == 2) {
        dnp_smooth2_t s2;
        if (dnp_smooth2_factor(nx, ny, c->wd_damp, c->wd_damp1, &s2)) {
            dnp_smooth2_free(&s2);
            return fail(dn_fail(DN_ENOMEM, "dn_precond_create"));
        }
        p->r1w = s2.r1w;
        st = upload((void **)&p->dx, s2.dx, sizeof(float) * s2.nx_line);
        if (!st) st = upload((void **)&p->ex, s2.ex, sizeof(float) * s2.nx_line);
        if (!st) st = upload((void **)&p->dz, s2.dz, sizeof(float) * s2.nz_line);
        if (!st) st = upload((void **)&p->ez, s2.ez, sizeof(float) * s2.nz_line);
        dnp_smooth2_free(&s2);
        if (st) return fail(st);
    }
    if (c->spatfilter == 3) {
        // gauss_filt.c:54-118: size WD_DAMP * C_vs / FC_END in grid points, made odd
        int F = dnp_gauss_size(c->wd_damp, c->c_vs, c->fc_end, dh);
        if (F != 0) {
            if (!(F % 2)) F += F > 0 ? 1 : -1;
            const int h = std::abs(F) / 2;
            if (h > 2000) return fail(dn_fail(DN_EINVAL, "gauss_filt: filter of %d grid points", F));
            std::vector<float> k((size_t)(2 * h + 1) * (2 * h + 1));
            const float sum = dnp_gauss_kernel(h, h, k.data());
            if (F > 0)
                for (float &v : k) v /= sum;
            p->gauss_h = h;
            if ((st = upload((void **)&p->gk, k.data(), sizeof(float) * k.size()))) return fail(st);
        }
    }
    if (c->spatfilter >= 2 && dn_malloc(&p->scratch, n * sizeof(double)) != cudaSuccess)
        return fail(dn_fail(DN_ENOMEM, "dn_precond_create: scratch"));
    if (c->spatfilter == 4 && (dn_malloc(&p->flag, sizeof(int)) != cudaSuccess ||
                               dn_malloc(&p->maxbits, sizeof(unsigned)) != cudaSuccess))
        return fail(dn_fail(DN_ENOMEM, "dn_precond_create"));
    *out = p;
    return DN_OK;
}

// SPATFILTER 4 weights for every size pair up to the model's largest (HX, HZ)
static int gauss_var_table(const dn_precond_plan *p, const dn_model_view &v, cudaStream_t st)
{
    CU(cudaMemsetAsync(p->maxbits, 0, sizeof(unsigned), st));
    k_max_bits<<<grid_blocks((long long)v.nx * v.ny), 256, 0, st>>>(v.vs, v.pitch, v.nx, v.ny, p->maxbits);
    unsigned bits = 0;
    CU(cudaMemcpyAsync(&bits, p->maxbits, sizeof bits, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    float vmax;
    memcpy(&vmax, &bits, sizeof vmax);
    auto half = [&](float wd) {
        int f = dnp_gauss_size(wd, vmax, p->c.fc_end, p->dh);
        if (!(f % 2)) f += 1;
        f = std::max(f, 6);
        return std::abs(f) / 2;
    };
    const int HX = half(p->c.wd_damp), HZ = half(p->c.wd_damp1);
    if (HX == p->HX && HZ == p->HZ && p->tab) return DN_OK;
    long long total = 0;
    std::vector<long long> off;
    for (int hx = 3; hx <= HX; hx++)
        for (int hz = 3; hz <= HZ; hz++) {
            off.push_back(total);
            total += (long long)(2 * hx + 1) * (2 * hz + 1);
        }
    if (total > (1LL << 27))
        return dn_fail(DN_ENOTSUP, "gauss_filt_var: filters up to %d x %d grid points", 2 * HX + 1, 2 * HZ + 1);
    std::vector<float> tab((size_t)total), sums(off.size());
    size_t q = 0;
    for (int hx = 3; hx <= HX; hx++)
        for (int hz = 3; hz <= HZ; hz++, q++) sums[q] = dnp_gauss_kernel(hx, hz, tab.data() + off[q]);
    dn_free(p->tab);
    dn_free(p->sums);
    dn_free(p->off);
    p->tab = p->sums = nullptr;
    p->off = nullptr;
    int s = upload((void **)&p->tab, tab.data(), sizeof(float) * tab.size());
    if (!s) s = upload((void **)&p->sums, sums.data(), sizeof(float) * sums.size());
    if (!s) s = upload((void **)&p->off, off.data(), sizeof(long long) * off.size());
    if (s) return s;
    p->HX = HX;
    p->HZ = HZ;
    return DN_OK;
}

template <typename T>
static int apply_t(const dn_precond_plan *p, const dn_model_view &v)
{
    cudaStream_t st = p->stream;
    const int nx = v.nx, ny = v.ny;
    const long long n = (long long)nx * ny;
    const int B = grid_blocks(n);
    T *g = (T *)v.dgrad;
    T *tmp = (T *)p->scratch;
    if (p->c.spatfilter == 4) {
        int s = gauss_var_table(p, v, st);
        if (s) return s;
        CU(cudaMemsetAsync(p->flag, 0, sizeof(int), st));
    }
    for (int cls = 0; cls < 3; cls++) {
        T *gc = g + cls * n;
        switch (p->c.spatfilter) {
        case 2:
            k_smooth2_x<T><<<(ny + 127) / 128, 128, 0, st>>>(gc, nx, ny, p->dx, p->ex);
            k_smooth2_z<T><<<(nx + 127) / 128, 128, 0, st>>>(gc, nx, ny, p->dz, p->ez, p->r1w);
            break;
        case 3:
            if (p->gauss_h >= 0) {
                k_gauss<T><<<B, 256, 0, st>>>(gc, tmp, nx, ny, p->gauss_h, p->gk);
                CU(cudaMemcpyAsync(gc, tmp, sizeof(T) * n, cudaMemcpyDeviceToDevice, st));
            }
            break;
        case 4:
            k_gauss_var<T><<<B, 256, 0, st>>>(gc, tmp, nx, ny, v.vs, v.pitch, p->c.wd_damp, p->c.wd_damp1, p->c.fc_end,
                                              p->dh, p->HX, p->HZ, p->tab, p->off, p->sums, p->flag);
            CU(cudaMemcpyAsync(gc, tmp, sizeof(T) * n, cudaMemcpyDeviceToDevice, st));
            break;
        default:
            break;
        }
        if (p->vrow || p->hcol || p->src || p->file[cls])
            k_tapers<T><<<B, 256, 0, st>>>(gc, nx, ny, p->vrow, p->hcol, p->src, p->file[cls], p->mask);
    }
    CU(cudaGetLastError());
    int flag = 0;
    if (p->c.spatfilter == 4) CU(cudaMemcpyAsync(&flag, p->flag, sizeof flag, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    if (flag) return dn_fail(DN_EINVAL, "gauss_filt_var: the S-velocity model holds values outside the filter table");
    return DN_OK;
}

extern "C" int dn_precond_apply(const dn_precond_plan *p, dn_model *m)
{
    DnRange range("gradient conditioning");
    if (!p || !m) return dn_fail(DN_EINVAL, "dn_precond_apply: null argument");
    dn_model_view v;
    int st = dn_model_view_get(m, &v);
    if (st) return st;
    if (v.nx != p->nx || v.ny != p->ny || v.device != p->device)
        return dn_fail(DN_EINVAL, "dn_precond_apply: plan for %d x %d on device %d, model %d x %d on device %d", p->nx,
                       p->ny, p->device, v.nx, v.ny, v.device);
    CU(cudaSetDevice(p->device));
    CU(cudaDeviceSynchronize());   // gradient accumulation runs on the engine's stream
    return v.grad64 ? apply_t<double>(p, v) : apply_t<float>(p, v);
}
