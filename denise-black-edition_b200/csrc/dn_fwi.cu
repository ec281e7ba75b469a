// FWI outer-loop linear algebra on the device, in FP64: the deterministic dot
// product and the L-BFGS direction of src/LBFGS.c (Nocedal and Wright 2006,
// two-loop recursion) over a device-resident history of model and gradient
// differences.  The reference keeps these vectors in float with float dot
// products (src/dotp.c); here every vector and every sum is double.
//
// Dot products are reduced in a fixed order (per-thread strided partial sums,
// a fixed-shape block tree, then one block over the block partials), so a
// result does not depend on scheduling: repeated calls give identical bits.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "denise_b200.h"
#include "dn_internal.h"

namespace {

constexpr int DOT_THREADS = 256;
constexpr int DOT_BLOCKS = 148 * 4;

__global__ void k_dot_partial(const double *__restrict__ a, const double *__restrict__ b, long long n,
                              double *__restrict__ part)
{
    __shared__ double sh[DOT_THREADS];
    double s = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride)
        s = __dadd_rn(s, __dmul_rn(a[k], b[k]));
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = DOT_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] = __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_dot_final(const double *__restrict__ part, int n, double *__restrict__ out)
{
    __shared__ double sh[DOT_THREADS];
    double s = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) s = __dadd_rn(s, part[k]);
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = DOT_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] = __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

// y += a * x
__global__ void k_axpy(double a, const double *__restrict__ x, double *__restrict__ y, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride)
        y[k] = __dadd_rn(y[k], __dmul_rn(a, x[k]));
}

// y = a * x
__global__ void k_scale(double a, const double *__restrict__ x, double *__restrict__ y, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride)
        y[k] = __dmul_rn(a, x[k]);
}

int dot_on(const double *a, const double *b, long long n, double *scratch, cudaStream_t st, double *out)
{
    k_dot_partial<<<DOT_BLOCKS, DOT_THREADS, 0, st>>>(a, b, n, scratch);
    k_dot_final<<<1, DOT_THREADS, 0, st>>>(scratch, DOT_BLOCKS, scratch + DOT_BLOCKS);
    cudaError_t e = cudaMemcpyAsync(out, scratch + DOT_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "dot product: %s", cudaGetErrorString(e));
    return DN_OK;
}

}   // namespace

struct dn_lbfgs {
    int device = 0, m = 0;
    long long n = 0;
    int count = 0, head = 0;      // pairs stored; slot of the next pair
    double *S = nullptr, *Y = nullptr, *scratch = nullptr;
    std::vector<double> rho;
    cudaStream_t stream = nullptr;
};

extern "C" int dn_dot(const double *a, const double *b, long long n, double *out)
{
    if (!a || !b || !out || n < 0) return dn_fail(DN_EINVAL, "dn_dot: bad arguments");
    double *scratch = nullptr;
    if (dn_malloc(&scratch, sizeof(double) * (DOT_BLOCKS + 1)) != cudaSuccess)
        return dn_fail(DN_ENOMEM, "dn_dot: scratch allocation failed");
    int st = dot_on(a, b, n, scratch, 0, out);
    dn_free(scratch);
    return st;
}

extern "C" int dn_lbfgs_create(long long n, int m, int device, dn_lbfgs **out)
{
    if (!out || n < 1 || m < 1 || m > 1000) return dn_fail(DN_EINVAL, "dn_lbfgs_create: bad arguments");
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
    dn_lbfgs *L = new dn_lbfgs();
    L->device = device;
    L->n = n;
    L->m = m;
    L->rho.assign(m, 0.0);
    if (dn_malloc(&L->S, sizeof(double) * n * m) != cudaSuccess ||
        dn_malloc(&L->Y, sizeof(double) * n * m) != cudaSuccess ||
        dn_malloc(&L->scratch, sizeof(double) * (DOT_BLOCKS + 1)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        dn_lbfgs_destroy(L);
        return dn_fail(DN_ENOMEM, "dn_lbfgs_create: %lld x %d history does not fit", n, m);
    }
    *out = L;
    return DN_OK;
}

extern "C" int dn_lbfgs_destroy(dn_lbfgs *L)
{
    if (!L) return DN_OK;
    cudaSetDevice(L->device);
    if (L->stream) cudaStreamSynchronize(L->stream);
    dn_free(L->S);
    dn_free(L->Y);
    dn_free(L->scratch);
    if (L->stream) cudaStreamDestroy(L->stream);
    delete L;
    return DN_OK;
}

// stores s = x_{k+1} - x_k and y = g_{k+1} - g_k (device vectors of length n); the oldest
// pair is dropped when m are held.  rho = 1 / (y . s), or 0 when y . s = 0 (LBFGS.c:40-49).
extern "C" int dn_lbfgs_push(dn_lbfgs *L, const double *d_s, const double *d_y)
{
    if (!L || !d_s || !d_y) return dn_fail(DN_EINVAL, "dn_lbfgs_push: null argument");
    CU(cudaSetDevice(L->device));
    double *s = L->S + (size_t)L->head * L->n, *y = L->Y + (size_t)L->head * L->n;
    CU(cudaMemcpyAsync(s, d_s, sizeof(double) * L->n, cudaMemcpyDeviceToDevice, L->stream));
    CU(cudaMemcpyAsync(y, d_y, sizeof(double) * L->n, cudaMemcpyDeviceToDevice, L->stream));
    double ys = 0.0;
    int st = dot_on(y, s, L->n, L->scratch, L->stream, &ys);
    if (st) return st;
    L->rho[L->head] = ys != 0.0 ? 1.0 / ys : 0.0;
    L->head = (L->head + 1) % L->m;
    if (L->count < L->m) L->count++;
    return DN_OK;
}

extern "C" int dn_lbfgs_count(const dn_lbfgs *L, int *count)
{
    if (!L || !count) return dn_fail(DN_EINVAL, "dn_lbfgs_count: null argument");
    *count = L->count;
    return DN_OK;
}

// r = H g: the two-loop recursion with H0 = gamma I, gamma = (s . y) / (y . y) of
// the newest pair (LBFGS.c:27-90); with no pair stored, r = g.  d_g and d_r are
// device vectors of length n; they may not alias the history.
extern "C" int dn_lbfgs_direction(dn_lbfgs *L, const double *d_g, double *d_r)
{
    if (!L || !d_g || !d_r) return dn_fail(DN_EINVAL, "dn_lbfgs_direction: null argument");
    CU(cudaSetDevice(L->device));
    const long long n = L->n;
    const int G = 148 * 8, T = 256;
    CU(cudaMemcpyAsync(d_r, d_g, sizeof(double) * n, cudaMemcpyDeviceToDevice, L->stream));
    if (L->count == 0) {
        CU(cudaStreamSynchronize(L->stream));
        return DN_OK;
    }
    std::vector<double> alpha(L->m, 0.0);
    // newest to oldest: alpha_k = rho_k s_k . q, q -= alpha_k y_k  (q lives in d_r)
    for (int c = 0; c < L->count; c++) {
        const int k = (L->head - 1 - c + 2 * L->m) % L->m;
        double sq = 0.0;
        int st = dot_on(L->S + (size_t)k * n, d_r, n, L->scratch, L->stream, &sq);
        if (st) return st;
        alpha[k] = L->rho[k] * sq;
        k_axpy<<<G, T, 0, L->stream>>>(-alpha[k], L->Y + (size_t)k * n, d_r, n);
    }
    const int newest = (L->head - 1 + L->m) % L->m;
    double sy = 0.0, yy = 0.0;
    int st = dot_on(L->S + (size_t)newest * n, L->Y + (size_t)newest * n, n, L->scratch, L->stream, &sy);
    if (!st) st = dot_on(L->Y + (size_t)newest * n, L->Y + (size_t)newest * n, n, L->scratch, L->stream, &yy);
    if (st) return st;
    const double gamma = yy != 0.0 ? sy / yy : 1.0;
    k_scale<<<G, T, 0, L->stream>>>(gamma, d_r, d_r, n);
    // oldest to newest: beta = rho_k y_k . r, r += s_k (alpha_k - beta)
    for (int c = L->count - 1; c >= 0; c--) {
        const int k = (L->head - 1 - c + 2 * L->m) % L->m;
        double yr = 0.0;
        st = dot_on(L->Y + (size_t)k * n, d_r, n, L->scratch, L->stream, &yr);
        if (st) return st;
        const double beta = L->rho[k] * yr;
        k_axpy<<<G, T, 0, L->stream>>>(alpha[k] - beta, L->S + (size_t)k * n, d_r, n);
    }
    CU(cudaStreamSynchronize(L->stream));
    CU(cudaGetLastError());
    return DN_OK;
}

// ===========================================================================
// The reference's optimisers on the device (FWI_PSV.c:637-676), applied to a
// model's stacked, conditioned gradient in place:
//  - GRAD_METHOD 2: the LBFGS_pointer rule of FWI_PSV.c:452-466,
//    store_LBFGS_PSV (src/PSV/store_LBFGS_PSV.c:37-206), LBFGS
//    (src/LBFGS.c:26-93) and extract_LBFGS_PSV (src/PSV/extract_LBFGS_PSV.c:
//    31-76);
//  - GRAD_METHOD 1: descent, store_PCG_PSV, PCG (src/PCG.c:23-100),
//    extract_PCG_PSV, descent.
// Vectors are float, as the reference's; every dot product sums the exact
// double products of its float operands in double (fixed reduction order)
// and is rounded to float where the reference keeps the sum in a float, so
// the only departure from the reference's arithmetic is the (more accurate)
// summation of the dot products.  Every elementwise float operation is an
// explicit round-to-nearest intrinsic in the reference's order.
// Internal vectors hold the classes vp, vs, rho, each [j][i] row-major like
// the model's stacked gradient; slots of the L-BFGS history that were never
// written since the last reset are skipped, which is exact (the reference's
// zero vectors give rho = alpha = beta = 0 and leave q and r unchanged).
// ===========================================================================
namespace {

constexpr int OPT_G = 148 * 8, OPT_T = 256;

// sum over k of a[k] * (b[k] (-) c[k]) with the difference rounded to float
// first (c == nullptr: a[k] * b[k]); products exact in double
__global__ void k_dotf_partial(const float *__restrict__ a, const float *__restrict__ b, const float *__restrict__ c,
                               long long n, double *__restrict__ part)
{
    __shared__ double sh[DOT_THREADS];
    double s = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        const float bb = c ? __fsub_rn(b[k], c[k]) : b[k];
        s = __dadd_rn(s, __dmul_rn((double)a[k], (double)bb));
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = DOT_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] = __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// element e of class c = e / nn, cell (j, i) = (e % nn) / nx + 1, (e % nn) % nx + 1
struct ModelPlanes {
    const float *cls[3];      // vp, vs, rho origin pointers
    int nx, pitch;
    long long nn;
};
__device__ __forceinline__ float model_at(const ModelPlanes &M, long long e)
{
    const int c = (int)(e / M.nn);
    const long long w = e - c * M.nn;
    const int j = (int)(w / M.nx) + 1, i = (int)(w % M.nx) + 1;
    return M.cls[c][(long long)j * M.pitch + i];
}
__device__ __forceinline__ float grad_at(const void *g, int g64, long long e)
{
    return g64 ? __double2float_rn(((const double *)g)[e]) : ((const float *)g)[e];
}
__device__ __forceinline__ void grad_put(void *g, int g64, long long e, float v)
{
    if (g64)
        ((double *)g)[e] = (double)v;
    else
        ((float *)g)[e] = v;
}

// store_LBFGS_PSV: gn = C g per class (the gradients the reference normalises and
// keeps as gradp); with a previous iteration y = gn - gold and s = m - mold into
// slot (y, s); q = gn; then gold = gn and mold = m (what extract_LBFGS_PSV writes
// to the JACOBIAN files)
__global__ void k_lbfgs_store(ModelPlanes M, const void *__restrict__ g, int g64, float c0, float c1, float c2,
                              int have_old, float *__restrict__ y, float *__restrict__ s, float *__restrict__ q,
                              float *__restrict__ gold, float *__restrict__ mold, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        const int c = (int)(e / M.nn);
        const float C = c == 0 ? c0 : (c == 1 ? c1 : c2);
        const float gn = __fmul_rn(C, grad_at(g, g64, e));
        const float m = model_at(M, e);
        if (have_old) {
            y[e] = __fsub_rn(gn, gold[e]);
            s[e] = __fsub_rn(m, mold[e]);
        }
        q[e] = gn;
        gold[e] = gn;
        mold[e] = m;
    }
}

// q = q - alpha y
__global__ void k_lbfgs_q(float alpha, const float *__restrict__ y, float *__restrict__ q, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride)
        q[e] = __fsub_rn(q[e], __fmul_rn(alpha, y[e]));
}

// r = gamma q
__global__ void k_lbfgs_r0(float gamma, const float *__restrict__ q, float *__restrict__ r, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) r[e] = __fmul_rn(gamma, q[e]);
}

// r = r + s (alpha - beta)
__global__ void k_lbfgs_r(float ab, const float *__restrict__ s, float *__restrict__ r, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride)
        r[e] = __fadd_rn(r[e], __fmul_rn(s[e], ab));
}

// extract_LBFGS_PSV: direction = r C per class (scale = 1: the normalised gradient itself)
__global__ void k_lbfgs_extract(const float *__restrict__ r, int scale, float c0, float c1, float c2, long long nn,
                                float *__restrict__ dir, void *__restrict__ g, int g64, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        const int c = (int)(e / nn);
        const float C = c == 0 ? c0 : (c == 1 ? c1 : c2);
        const float d = scale ? __fmul_rn(r[e], C) : r[e];
        dir[e] = d;
        grad_put(g, g64, e, d);
    }
}

// descent + store_PCG_PSV: pnew = -g
__global__ void k_pcg_new(const void *__restrict__ g, int g64, float *__restrict__ pnew, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) pnew[e] = -grad_at(g, g64, e);
}

// PCG direction per class dir = new + beta dir; then pold = pnew, and the
// gradient becomes -dir (extract_PCG_PSV, descent)
__global__ void k_pcg_dir(float b0, float b1, float b2, long long nn, const float *__restrict__ pnew,
                          float *__restrict__ pold, float *__restrict__ pdir, void *__restrict__ g, int g64, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        const int c = (int)(e / nn);
        const float b = c == 0 ? b0 : (c == 1 ? b1 : b2);
        const float d = __fadd_rn(pnew[e], __fmul_rn(b, pdir[e]));
        pdir[e] = d;
        pold[e] = pnew[e];
        grad_put(g, g64, e, -d);
    }
}

}   // namespace

struct dn_optim {
    int method = 2, nx = 0, ny = 0, nlbfgs = 0, pcg_beta = 2, device = 0;
    long long nn = 0, n = 0;
    int ptr = 1, have_old = 0;
    std::vector<char> filled;         // slot written since the last reset
    float *Y = nullptr, *S = nullptr;  // nlbfgs x n
    float *q = nullptr, *r = nullptr, *gold = nullptr, *mold = nullptr, *dir = nullptr;
    float *pold = nullptr, *pnew = nullptr, *pdir = nullptr;
    double *scratch = nullptr;
    cudaStream_t stream = nullptr;
};

static int dotf(dn_optim *o, const float *a, const float *b, const float *c, long long n, float *out)
{
    k_dotf_partial<<<DOT_BLOCKS, DOT_THREADS, 0, o->stream>>>(a, b, c, n, o->scratch);
    k_dot_final<<<1, DOT_THREADS, 0, o->stream>>>(o->scratch, DOT_BLOCKS, o->scratch + DOT_BLOCKS);
    double v = 0.0;
    cudaError_t e = cudaMemcpyAsync(&v, o->scratch + DOT_BLOCKS, sizeof(double), cudaMemcpyDeviceToHost, o->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(o->stream);
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "optimiser dot product: %s", cudaGetErrorString(e));
    *out = (float)v;
    return DN_OK;
}

extern "C" int dn_optim_destroy(dn_optim *o)
{
    if (!o) return DN_OK;
    cudaSetDevice(o->device);
    if (o->stream) cudaStreamSynchronize(o->stream);
    for (float *p : {o->Y, o->S, o->q, o->r, o->gold, o->mold, o->dir, o->pold, o->pnew, o->pdir}) dn_free(p);
    dn_free(o->scratch);
    if (o->stream) cudaStreamDestroy(o->stream);
    delete o;
    return DN_OK;
}

extern "C" int dn_optim_reset(dn_optim *o)
{
    if (!o) return dn_fail(DN_EINVAL, "dn_optim_reset: null optimiser");
    CU(cudaSetDevice(o->device));
    o->ptr = 1;
    std::fill(o->filled.begin(), o->filled.end(), 0);
    if (o->method == 1) {
        CU(cudaMemsetAsync(o->pold, 0, sizeof(float) * o->n, o->stream));
        CU(cudaMemsetAsync(o->pdir, 0, sizeof(float) * o->n, o->stream));
        CU(cudaStreamSynchronize(o->stream));
    }
    return DN_OK;
}

extern "C" int dn_optim_create(int grad_method, int nx, int ny, int nlbfgs, int pcg_beta, int device, dn_optim **out)
{
    if (!out || nx < 1 || ny < 1 || (grad_method != 1 && grad_method != 2) ||
        (grad_method == 2 && (nlbfgs < 1 || nlbfgs > 1000)) || (grad_method == 1 && (pcg_beta < 1 || pcg_beta > 4)))
        return dn_fail(DN_EINVAL, "dn_optim_create: GRAD_METHOD %d, NLBFGS %d, PCG_BETA %d, %d x %d", grad_method,
                       nlbfgs, pcg_beta, nx, ny);
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
    dn_optim *o = new dn_optim();
    o->method = grad_method;
    o->nx = nx;
    o->ny = ny;
    o->nlbfgs = grad_method == 2 ? nlbfgs : 0;
    o->pcg_beta = pcg_beta;
    o->device = device;
    o->nn = (long long)nx * ny;
    o->n = 3 * o->nn;
    o->filled.assign(o->nlbfgs, 0);
    const size_t v = sizeof(float) * o->n;
    bool ok = dn_malloc(&o->scratch, sizeof(double) * (DOT_BLOCKS + 1)) == cudaSuccess &&
              cudaStreamCreateWithFlags(&o->stream, cudaStreamNonBlocking) == cudaSuccess;
    if (ok && grad_method == 2)
        ok = dn_malloc(&o->Y, v * o->nlbfgs) == cudaSuccess && dn_malloc(&o->S, v * o->nlbfgs) == cudaSuccess &&
             dn_malloc(&o->q, v) == cudaSuccess && dn_malloc(&o->r, v) == cudaSuccess &&
             dn_malloc(&o->gold, v) == cudaSuccess && dn_malloc(&o->mold, v) == cudaSuccess &&
             dn_malloc(&o->dir, v) == cudaSuccess;
    if (ok && grad_method == 1)
        ok = dn_malloc(&o->pold, v) == cudaSuccess && dn_malloc(&o->pnew, v) == cudaSuccess &&
             dn_malloc(&o->pdir, v) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        dn_optim_destroy(o);
        return dn_fail(DN_ENOMEM, "dn_optim_create: %lld-element vectors (%d pairs) do not fit", o->n, nlbfgs);
    }
    int st = dn_optim_reset(o);
    if (st) {
        dn_optim_destroy(o);
        return st;
    }
    *out = o;
    return DN_OK;
}

extern "C" int dn_optim_step(dn_optim *o, dn_model *m, int iter, const float c[3])
{
    if (!o || !m || !c || iter < 1) return dn_fail(DN_EINVAL, "dn_optim_step: bad arguments");
    dn_model_view v;
    int st = dn_model_view_get(m, &v);
    if (st) return st;
    if (v.nx != o->nx || v.ny != o->ny || v.device != o->device)
        return dn_fail(DN_EINVAL, "dn_optim_step: model %d x %d on device %d, optimiser %d x %d on device %d", v.nx,
                       v.ny, v.device, o->nx, o->ny, o->device);
    CU(cudaSetDevice(o->device));
    CU(cudaDeviceSynchronize());   // the gradient's producers (runs, conditioning) are complete
    const long long n = o->n, nn = o->nn;
    if (o->method == 1) {
        k_pcg_new<<<OPT_G, OPT_T, 0, o->stream>>>(v.dgrad, v.grad64, o->pnew, n);
        float beta[3];
        for (int k = 0; k < 3; k++) {
            const float *a = o->pnew + k * nn, *old = o->pold + k * nn, *d = o->pdir + k * nn;
            float bz = 0.0f, bn = 0.0f;
            switch (o->pcg_beta) {
            case 1: st = dotf(o, a, a, nullptr, nn, &bz); if (!st) st = dotf(o, old, old, nullptr, nn, &bn); break;
            case 2: st = dotf(o, a, a, old, nn, &bz); if (!st) st = dotf(o, old, old, nullptr, nn, &bn); break;
            case 3: st = dotf(o, a, a, old, nn, &bz); bz = -bz; if (!st) st = dotf(o, d, a, old, nn, &bn); break;
            default: st = dotf(o, a, a, nullptr, nn, &bz); bz = -bz; if (!st) st = dotf(o, d, a, old, nn, &bn); break;
            }
            if (st) return st;
            beta[k] = bn != 0.0f ? bz / bn : 0.0f;
            if (beta[k] < 0.0f && o->pcg_beta == 2) beta[k] = 0.0f;
        }
        k_pcg_dir<<<OPT_G, OPT_T, 0, o->stream>>>(beta[0], beta[1], beta[2], nn, o->pnew, o->pold, o->pdir, v.dgrad,
                                                  v.grad64, n);
        CU(cudaStreamSynchronize(o->stream));
        CU(cudaGetLastError());
        return DN_OK;
    }
    if (iter > 2) o->ptr++;
    if (o->ptr > o->nlbfgs) o->ptr = 1;
    const int have_old = iter > 1 && o->have_old;
    const int cur = o->ptr - 1;
    float *Yc = o->Y + (size_t)cur * n, *Sc = o->S + (size_t)cur * n;
    ModelPlanes M;
    M.cls[0] = v.vp;
    M.cls[1] = v.vs;
    M.cls[2] = v.rho;
    M.nx = v.nx;
    M.pitch = v.pitch;
    M.nn = nn;
    k_lbfgs_store<<<OPT_G, OPT_T, 0, o->stream>>>(M, v.dgrad, v.grad64, c[0], c[1], c[2], have_old, Yc, Sc, o->q,
                                                  o->gold, o->mold, n);
    o->have_old = 1;
    if (!have_old) {
        // iteration 1 (or no stored pair): the direction is the normalised gradient
        k_lbfgs_extract<<<OPT_G, OPT_T, 0, o->stream>>>(o->q, 0, c[0], c[1], c[2], nn, o->dir, v.dgrad, v.grad64, n);
        CU(cudaStreamSynchronize(o->stream));
        CU(cudaGetLastError());
        return DN_OK;
    }
    o->filled[cur] = 1;
    float sn = 0.0f, sd = 0.0f;
    if ((st = dotf(o, Yc, Sc, nullptr, n, &sn)) || (st = dotf(o, Yc, Yc, nullptr, n, &sd))) return st;
    const float gamma = sn / sd;
    std::vector<float> rho(o->nlbfgs, 0.0f), alpha(o->nlbfgs, 0.0f);
    for (int k = 0; k < o->nlbfgs; k++) {
        if (!o->filled[k]) continue;
        float yk = 0.0f;
        if ((st = dotf(o, o->Y + (size_t)k * n, o->S + (size_t)k * n, nullptr, n, &yk))) return st;
        rho[k] = fabsf(yk) > 0.0f ? (float)(1.0 / (double)yk) : 0.0f;
    }
    for (int k = o->nlbfgs - 1; k >= 0; k--) {
        if (!o->filled[k]) continue;
        float sq = 0.0f;
        if ((st = dotf(o, o->S + (size_t)k * n, o->q, nullptr, n, &sq))) return st;
        alpha[k] = rho[k] * sq;
        k_lbfgs_q<<<OPT_G, OPT_T, 0, o->stream>>>(alpha[k], o->Y + (size_t)k * n, o->q, n);
    }
    k_lbfgs_r0<<<OPT_G, OPT_T, 0, o->stream>>>(gamma, o->q, o->r, n);
    for (int k = 0; k < o->nlbfgs; k++) {
        if (!o->filled[k]) continue;
        float yr = 0.0f;
        if ((st = dotf(o, o->Y + (size_t)k * n, o->r, nullptr, n, &yr))) return st;
        const float beta = rho[k] * yr;
        k_lbfgs_r<<<OPT_G, OPT_T, 0, o->stream>>>(alpha[k] - beta, o->S + (size_t)k * n, o->r, n);
    }
    k_lbfgs_extract<<<OPT_G, OPT_T, 0, o->stream>>>(o->r, 1, c[0], c[1], c[2], nn, o->dir, v.dgrad, v.grad64, n);
    CU(cudaStreamSynchronize(o->stream));
    CU(cudaGetLastError());
    return DN_OK;
}

extern "C" int dn_optim_get(const dn_optim *o, int which, float *out)
{
    if (!o || !out || which < 0 || which > 8) return dn_fail(DN_EINVAL, "dn_optim_get: bad arguments");
    if (o->method != 2) return dn_fail(DN_ESTATE, "dn_optim_get: the JACOBIAN vectors belong to L-BFGS");
    if (!o->have_old) return dn_fail(DN_ESTATE, "dn_optim_get: no step taken");
    CU(cudaSetDevice(o->device));
    // which: 0-2 gradp (vp, vs, rho) | 3-5 model (vp, vs, rho) | 6-8 direction (vp, vs, rho)
    const float *src = (which < 3 ? o->gold : which < 6 ? o->mold : o->dir) + (size_t)(which % 3) * o->nn;
    std::vector<float> h(o->nn);
    CU(cudaMemcpy(h.data(), src, sizeof(float) * o->nn, cudaMemcpyDeviceToHost));
    for (int j = 0; j < o->ny; j++)
        for (int i = 0; i < o->nx; i++) out[(size_t)i * o->ny + j] = h[(size_t)j * o->nx + i];
    return DN_OK;
}
