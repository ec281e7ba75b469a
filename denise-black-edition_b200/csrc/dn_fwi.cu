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
