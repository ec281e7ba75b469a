// Time-domain Butterworth filtering of traces: apply_tdfilt (src/apply_tdfilt.c)
// -> timedomain_filt (src/timedomain_filt.c) -> seife_lpb / seife_hpb of the
// libcseife library in the reference tree.  The filter is E. Wielandt's
// recursive Butterworth of seife: an order-m filter is one first-order section
// (m odd) and m/2 second-order sections, each the recursion
//     y_k = f0 x_k + f1 x_{k-1} + f2 x_{k-2} + g1 y_{k-1} + g2 y_{k-2}
// from rest with bilinear-transform coefficients.  The reference runs the
// sections one after another over the whole trace; since each section's
// output at sample k depends only on its input up to k, running all sections
// per sample gives the same double values, so one pass per trace suffices.
// timedomain_filt converts to double, filters and converts back to float for
// the low-pass and again for the high-pass, and leaves the last sample of each
// trace unfiltered (it hands the filter a vector whose index 0 is a zero and
// copies back indices 1..ns); both are kept.
#include <cuda_runtime.h>

#include <cmath>

#include "denise_b200.h"
#include "dn_internal.h"

namespace {

constexpr int MAX_SEC = 9;   // order <= 16: one first-order and eight second-order sections

struct Sections {
    int n;
    double c[MAX_SEC][5];    // f0, f1, f2, g1, g2
};

// seife_butterworth: coefficients for period t0 (in samples) of an order-m low- or high-pass
Sections butterworth(int m, double t0, bool highpass)
{
    Sections s = {};
    const double one = 1.0, two = 2.0, four = 4.0;
    const double eps = 8.0 * atan(one) / t0;
    const int mm = m / 2;
    if (m > 2 * mm) {   // first-order section
        const double g1 = (two - eps) / (two + eps);
        const double f0 = highpass ? two / (two + eps) : eps / (two + eps);
        const double c[5] = {f0, highpass ? -f0 : f0, 0.0, g1, 0.0};
        for (int k = 0; k < 5; k++) s.c[s.n][k] = c[k];
        s.n++;
    }
    const double pih = 2.0 * atan(1.0);
    for (int j = 1; j <= mm; j++) {
        const double h = sin(pih * (2 * j - 1) / m);
        const double epsq = eps * eps;
        const double a = one - eps * h + epsq / four;
        const double b = -two + epsq / two;
        const double c = one + eps * h + epsq / four;
        const double f0 = highpass ? one / c : epsq / four / c;
        const double cc[5] = {f0, highpass ? -f0 - f0 : f0 + f0, f0, -b / c, -a / c};
        for (int k = 0; k < 5; k++) s.c[s.n][k] = cc[k];
        s.n++;
    }
    return s;
}

__device__ __forceinline__ double cascade(double x, const Sections &S, double (*st)[4])
{
    for (int q = 0; q < S.n; q++) {
        const double *c = S.c[q];
        double *z = st[q];   // xa, xaa, ya, yaa
        double y = __dmul_rn(c[0], x);
        y = __dadd_rn(y, __dmul_rn(c[1], z[0]));
        y = __dadd_rn(y, __dmul_rn(c[2], z[1]));
        y = __dadd_rn(y, __dmul_rn(c[3], z[2]));
        y = __dadd_rn(y, __dmul_rn(c[4], z[3]));
        z[1] = z[0];
        z[0] = x;
        z[3] = z[2];
        z[2] = y;
        x = y;
    }
    return x;
}

__global__ void k_tdfilt(float *tr, int ntr, int ns, Sections lp, Sections hp, int has_hp)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= ntr) return;
    float *r = tr + (size_t)l * ns;
    double sl[MAX_SEC][4] = {}, sh[MAX_SEC][4] = {};
    for (int t = 0; t + 1 < ns; t++) {
        float v = __double2float_rn(cascade((double)r[t], lp, sl));
        if (has_hp) v = __double2float_rn(cascade((double)v, hp, sh));
        r[t] = v;
    }
}

int check_args(int ntr, int ns, float dt, int order, float fc_low, float fc_high)
{
    if (ntr < 1 || ns < 1 || !(dt > 0.0f)) return dn_fail(DN_EINVAL, "dn_tdfilt: %d traces of %d samples, DT %g", ntr, ns, dt);
    if (order < 1 || order > 16) return dn_fail(DN_EINVAL, "dn_tdfilt: filter order %d (1..16)", order);
    if (!(fc_low > 0.0f)) return dn_fail(DN_EINVAL, "dn_tdfilt: low-pass corner %g must be positive", fc_low);
    // apply_tdfilt.c high-passes only for fc1 > 0: zero or negative corners (the
    // FC_SPIKE_1 = -5 of the reference's example files) mean no high-pass
    if (fc_high != fc_high) return dn_fail(DN_EINVAL, "dn_tdfilt: high-pass corner %g", fc_high);
    return DN_OK;
}

int launch(float *d, int ntr, int ns, float dt, int order, float fc_low, float fc_high, cudaStream_t st)
{
    // timedomain_filt.c: T0 = 1.0 / fc in double, the period in samples T0 / DT
    const Sections lp = butterworth(order, (1.0 / fc_low) / dt, false);
    const Sections hp = fc_high > 0.0f ? butterworth(order, (1.0 / fc_high) / dt, true) : Sections{};
    k_tdfilt<<<(ntr + 63) / 64, 64, 0, st>>>(d, ntr, ns, lp, hp, fc_high > 0.0f);
    CU(cudaGetLastError());
    return DN_OK;
}

}   // namespace

extern "C" int dn_tdfilt(float *traces, int ntr, int ns, float dt, int order, float fc_low, float fc_high)
{
    if (!traces) return dn_fail(DN_EINVAL, "dn_tdfilt: null traces");
    int st = check_args(ntr, ns, dt, order, fc_low, fc_high);
    if (st) return st;
    st = launch(traces, ntr, ns, dt, order, fc_low, fc_high, 0);
    if (st) return st;
    CU(cudaStreamSynchronize(0));
    return DN_OK;
}

extern "C" int dn_tdfilt_host(float *traces, int ntr, int ns, float dt, int order, float fc_low, float fc_high,
                              int device)
{
    if (!traces) return dn_fail(DN_EINVAL, "dn_tdfilt_host: null traces");
    int st = check_args(ntr, ns, dt, order, fc_low, fc_high);
    if (st) return st;
    CU(cudaSetDevice(device));
    const size_t bytes = sizeof(float) * (size_t)ntr * ns;
    float *d = nullptr;
    if (dn_malloc(&d, bytes) != cudaSuccess) {
        cudaGetLastError();
        return dn_fail(DN_ENOMEM, "dn_tdfilt_host: %zu bytes", bytes);
    }
    cudaError_t e = cudaMemcpy(d, traces, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        st = launch(d, ntr, ns, dt, order, fc_low, fc_high, 0);
        if (!st) e = cudaMemcpy(traces, d, bytes, cudaMemcpyDeviceToHost);
    }
    dn_free(d);
    if (!st && e != cudaSuccess) st = dn_fail(DN_EDEVICE, "dn_tdfilt_host: %s", cudaGetErrorString(e));
    return st;
}
