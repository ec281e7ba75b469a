// L2 data residual and misfit on the device: calc_res() of the reference
// (src/calc_res.c:306-445 residual, :514-568 misfit) for LNORM = 2, the
// residual that becomes the adjoint source of the back-propagation.
//
// One thread per trace walks the trace in time: the first observed sample is
// replaced by the synthetic one (calc_res.c:419), the float difference is
// time-integrated (GRAD_FORM 1: intseis += DT*(syn-obs), calc_res.c:435) or
// taken as is (GRAD_FORM 2) and written time-reversed; the misfit
// 0.5*sum(r^2) is accumulated in double per trace into a scratch array of
// per-trace partial sums, which a second kernel adds up in trace order.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "dn_internal.h"

namespace {

// rtm = 1: the reverse-time-migration source of calc_res.c:436/441 (MODE 2): the
// observed trace itself (first sample replaced by the synthetic one), integrated
// for GRAD_FORM 1, instead of the difference
__global__ void k_residual_l2(const float *__restrict__ syn, const float *__restrict__ obs, float *__restrict__ res,
                              int ntr, int nt, float dt, int grad_form, int rtm, double *__restrict__ part)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= ntr) return;
    const float *ob = obs + (size_t)l * nt;
    float *rs = res + (size_t)l * nt;
    float intseis = 0.0f;
    double l2 = 0.0;
    for (int t = 0; t < nt; t++) {
        const float s = syn[(size_t)t * ntr + l];
        const float d = t == 0 ? s : ob[t];
        const float diff = rtm ? d : __fsub_rn(s, d);
        float r;
        if (grad_form == 1) {
            intseis = __fadd_rn(intseis, __fmul_rn(dt, diff));
            r = intseis;
        } else {
            r = diff;
        }
        rs[nt - 1 - t] = r;
        l2 = __dadd_rn(l2, __dmul_rn(__dmul_rn(0.5, (double)r), (double)r));
    }
    part[l] = l2;
}

__global__ void k_sum_partials(const double *__restrict__ part, int n, double *__restrict__ out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double s = 0.0;
    for (int l = 0; l < n; l++) s = __dadd_rn(s, part[l]);
    *out = s;
}

}   // namespace

// Launches the two kernels on `stream` with `scratch` holding ntr + 1 doubles.
extern "C" int dn_adjoint_source_launch(const float *syn_tm, const float *obs, float *res, int ntr, int nt, float dt,
                                        int grad_form, int rtm, double *scratch, cudaStream_t stream)
{
    k_residual_l2<<<(ntr + 127) / 128, 128, 0, stream>>>(syn_tm, obs, res, ntr, nt, dt, grad_form, rtm, scratch);
    k_sum_partials<<<1, 1, 0, stream>>>(scratch, ntr, scratch + ntr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "residual kernels: %s", cudaGetErrorString(e));
    return DN_OK;
}

extern "C" int dn_residual_l2_launch(const float *syn_tm, const float *obs, float *res, int ntr, int nt, float dt,
                                     int grad_form, double *scratch, cudaStream_t stream)
{
    return dn_adjoint_source_launch(syn_tm, obs, res, ntr, nt, dt, grad_form, 0, scratch, stream);
}

extern "C" int dn_residual_l2(const float *syn_tm, const float *obs, float *res, int ntr, int nt, float dt,
                              int grad_form, double *l2)
{
    if (!syn_tm || !obs || !res || ntr < 1 || nt < 1)
        return dn_fail(DN_EINVAL, "dn_residual_l2: bad arguments");
    if (grad_form != 1 && grad_form != 2) return dn_fail(DN_EINVAL, "dn_residual_l2: GRAD_FORM must be 1 or 2");
    double *scratch = nullptr;
    cudaError_t e = cudaMalloc(&scratch, sizeof(double) * ((size_t)ntr + 1));
    if (e != cudaSuccess) return dn_fail(DN_ENOMEM, "dn_residual_l2: scratch allocation failed");
    int st = dn_residual_l2_launch(syn_tm, obs, res, ntr, nt, dt, grad_form, scratch, 0);
    double h = 0.0;
    if (!st) {
        e = cudaMemcpy(&h, scratch + ntr, sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = dn_fail(DN_EDEVICE, "dn_residual_l2: %s", cudaGetErrorString(e));
    }
    cudaFree(scratch);
    if (!st && l2) *l2 = h;
    return st;
}

// ---------------------------------------------------------------------------
// dn_residual_l2_noalloc: the same residual and misfit for callers that must
// not allocate device memory on the call, e.g. an inversion loop that runs
// under a fixed device-memory budget (every byte pre-reserved for shots and
// snapshots) or code that must not synchronise the device through
// cudaMalloc/cudaFree between shots.  The per-trace partial sums live in a
// file-scope device array of DN_RESIDUAL_NOALLOC_MAX_TRACES + 1 doubles
// (128 KiB + 8 B per device); larger trace counts are rejected.
//
// Set-up: the first call on each device looks up the array's address with that
// device current (cudaGetSymbolAddress, which may load this module on the
// device) and caches it; make that first call before any stream capture.
// Nothing in the scratch has to start at zero: k_residual_l2 writes every
// partial sum k_sum_partials reads, and the misfit slot is written, not added
// to.  There is one scratch array per device, so calls that overlap on the
// same device (from several host threads at once) race on it and may return
// each other's misfit; serialise them.  Each call returns only after its
// kernels and the copy of the misfit have finished.
// ---------------------------------------------------------------------------
#define DN_RESIDUAL_NOALLOC_MAX_TRACES 16384
#define DN_RESIDUAL_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) double g_residual_scratch[DN_RESIDUAL_NOALLOC_MAX_TRACES + 1];

namespace {

std::mutex g_scratch_mutex;
double *g_scratch_ptr[DN_RESIDUAL_NOALLOC_MAX_DEVICES];

// Address of this device's scratch array; looked up once per device.
int residual_scratch(double **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "dn_residual_l2_noalloc: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= DN_RESIDUAL_NOALLOC_MAX_DEVICES)
        return dn_fail(DN_ENOTSUP, "dn_residual_l2_noalloc: device %d beyond the %d supported", dev,
                       DN_RESIDUAL_NOALLOC_MAX_DEVICES);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        double *p = nullptr;
        e = cudaGetSymbolAddress((void **)&p, g_residual_scratch);
        if (e != cudaSuccess || !p)
            return dn_fail(DN_EDEVICE, "dn_residual_l2_noalloc: scratch address lookup on device %d: %s", dev,
                           cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return DN_OK;
}

}   // namespace

extern "C" int dn_residual_l2_noalloc(const float *syn_tm, const float *obs, float *res, int ntr, int nt, float dt,
                                      int grad_form, double *l2)
{
    if (!syn_tm || !obs || !res || ntr < 1 || nt < 1)
        return dn_fail(DN_EINVAL, "dn_residual_l2_noalloc: bad arguments");
    if (grad_form != 1 && grad_form != 2)
        return dn_fail(DN_EINVAL, "dn_residual_l2_noalloc: GRAD_FORM must be 1 or 2");
    if (ntr > DN_RESIDUAL_NOALLOC_MAX_TRACES)
        return dn_fail(DN_EINVAL, "dn_residual_l2_noalloc: %d traces exceed the static scratch of %d traces "
                       "(use dn_residual_l2)", ntr, DN_RESIDUAL_NOALLOC_MAX_TRACES);
    double *scratch = nullptr;
    int st = residual_scratch(&scratch);
    if (st) return st;
    st = dn_residual_l2_launch(syn_tm, obs, res, ntr, nt, dt, grad_form, scratch, 0);
    if (st) return st;
    double h = 0.0;
    cudaError_t e = cudaMemcpy(&h, scratch + ntr, sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "dn_residual_l2_noalloc: %s", cudaGetErrorString(e));
    if (l2) *l2 = h;
    return DN_OK;
}
