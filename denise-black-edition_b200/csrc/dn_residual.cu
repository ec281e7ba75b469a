// Data residual and misfit on the device: calc_res() of the reference
// (src/calc_res.c:7-640) for the objective functions that need no Fourier
// transform (LNORM 1, 2, 3, 4, 5, 7, 8); the residual becomes the adjoint
// source of the back-propagation.
//
// One thread per trace walks the trace in time: the first observed sample is
// replaced by the synthetic one (calc_res.c:419), the residual of the chosen
// norm is written time-reversed, and the trace's share of the misfit is
// accumulated in double into a scratch array of per-trace partial sums, which
// a second kernel adds up in trace order.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "dn_internal.h"

namespace {

// Options of calc_res as the kernel reads them (device pointers).
struct ResArgs {
    int lnorm, grad_form, mode, n_order, comp_weight;
    float wscale;                    // c_vp * c_rho (COMP_WEIGHT)
    float dt, dh;
    int nagc;                        // LNORM 8 half window
    const int *kill;                 // per trace, or null
    int offset_mute, timewin;
    float offsetc, gamma, twl;
    const int *rec_i, *rec_j;        // per trace, or null (no offsets needed)
    float src_x, src_z;
    float *s1, *s2;                  // LNORM 7: two [ntr][nt] scratch arrays
};

constexpr int MAX_NORDER = 8;

// One trace of calc_res (src/calc_res.c:306-600).  syn is time-major
// [nt][ntr]; obs and res [ntr][nt]; the first observed sample is replaced by
// the synthetic one (:419) after the N_ORDER integrations; float operations
// with explicit rounding, the reference's double terms in double; the trace's
// share of the misfit goes to part[l].
__global__ void k_residual(const float *__restrict__ syn, const float *__restrict__ obs, float *__restrict__ res,
                           int ntr, int nt, ResArgs a, double *__restrict__ part)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= ntr) return;
    const float *ob = obs + (size_t)l * nt;
    float *rs = res + (size_t)l * nt;
    const float dt = a.dt;
    double L2 = 0.0;
    auto S = [&](int t) { return a.comp_weight ? __fmul_rn(syn[(size_t)t * ntr + l], a.wscale) : syn[(size_t)t * ntr + l]; };
    auto D = [&](int t) { return a.comp_weight ? __fmul_rn(ob[t], a.wscale) : ob[t]; };
    float offset = 0.0f;
    bool skip = a.kill && a.kill[l] == 1;
    if (!skip && (a.offset_mute || a.timewin == 5)) {
        const float xr = __fmul_rn((float)a.rec_i[l], a.dh), yr = __fmul_rn((float)a.rec_j[l], a.dh);
        const float dx = __fsub_rn(a.src_x, xr), dy = __fsub_rn(a.src_z, yr);
        offset = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
        if (a.offset_mute == 1 && offset >= a.offsetc) skip = true;
        if (a.offset_mute == 2 && offset <= a.offsetc) skip = true;
    }
    if (skip) {   // calc_res zeroes the whole residual first (:44)
        for (int t = 0; t < nt; t++) rs[t] = 0.0f;
        part[l] = 0.0;
        return;
    }
    const int ln = a.lnorm, gf = a.grad_form;
    if (ln == 7) {
        // :240-303 and :362-382; scratch s1 = integrated synthetic, s2 = running Qmod then dQ
        float *is = a.s1 + (size_t)l * nt, *q = a.s2 + (size_t)l * nt;
        float cs = 0.0f, cd = 0.0f, Qm = 0.0f, Qt = 0.0f;
        for (int t = 0; t < nt; t++) {
            float xs = S(t), xd = D(t);
            if (gf == 1) {
                cs = __fadd_rn(cs, xs);
                cd = __fadd_rn(cd, xd);
                xs = __fmul_rn(dt, cs);
                xd = __fmul_rn(dt, cd);
            }
            is[t] = xs;
            Qm = __fadd_rn(Qm, __fmul_rn(xs, xs));
            Qt = __fadd_rn(Qt, __fmul_rn(xd, xd));
            q[t] = Qm;
            rs[t] = Qt;   // running Qtrue, consumed below
        }
        float Q1 = 0.0f, Q2 = 0.0f;
        for (int t = 0; t < nt; t++) {
            const float qm = __fdiv_rn(q[t], Qm), qt = __fdiv_rn(rs[t], Qt);
            const float dq = __fsub_rn(qm, qt);
            Q1 = __fadd_rn(Q1, __fmul_rn(dq, qm));
            Q2 = __fadd_rn(Q2, qm);
            q[t] = dq;
        }
        float Q3 = 0.0f;
        for (int t = nt - 1, h = 0; t >= 0; t--, h++) {
            Q3 = __fadd_rn(Q3, q[t]);
            const double v = __ddiv_rn(__dmul_rn(__dmul_rn(-2.0, (double)is[t]), (double)__fsub_rn(-Q3, Q1)), (double)Q2);
            rs[h] = __double2float_rn(v);
        }
        for (int t = nt - 1; t >= 0; t--) L2 = __dadd_rn(L2, __dmul_rn(__dmul_rn(0.5, (double)q[t]), (double)q[t]));
        part[l] = L2;
        return;
    }
    // LNORM 5: norms of the (integrated) traces before the main loop (:331-360)
    float ad = 0.0f, asn = 0.0f, dms = 0.0f;
    if (ln == 5) {
        float cs = 0.0f, cd = 0.0f;
        for (int t = 0; t < nt; t++) {
            float xs = S(t), xd = D(t);
            if (gf == 1) {
                cs = __fadd_rn(cs, xs);
                cd = __fadd_rn(cd, xd);
                xs = __fmul_rn(dt, cs);
                xd = __fmul_rn(dt, cd);
            }
            ad = __fadd_rn(ad, __fmul_rn(xd, xd));
            asn = __fadd_rn(asn, __fmul_rn(xs, xs));
            dms = __fadd_rn(dms, __fmul_rn(xs, xd));
        }
        ad = __fsqrt_rn(ad);
        asn = __fsqrt_rn(asn);
    }
    const float tmp5 = __fmul_rn(__fmul_rn(__fmul_rn(asn, asn), asn), ad), tmp15 = __fmul_rn(asn, ad);
    const float t0 = fabsf(__fdiv_rn(offset, a.twl));
    // N_ORDER integrations (:400-414) run along the trace with one accumulator per order
    float ps[MAX_NORDER], pd[MAX_NORDER];
    float cs5 = 0.0f, cd5 = 0.0f;        // LNORM 5, GRAD_FORM 1: the integration of :134-148
    float intseis = 0.0f, sign = 0.0f;
    for (int t = 0; t < nt; t++) {
        float xs = S(t), xd = D(t);
        const float rawd = xd;
        for (int k = 0; k < a.n_order; k++) {
            if (t == 0) {
                xs = __fmul_rn(xs, dt);
                xd = __fmul_rn(xd, dt);
            } else {
                xs = __fadd_rn(ps[k], __fmul_rn(xs, dt));
                xd = __fadd_rn(pd[k], __fmul_rn(xd, dt));
            }
            ps[k] = xs;
            pd[k] = xd;
        }
        if (t == 0) xd = xs;
        float r = 0.0f;
        if (ln == 1) {
            const float df = __fsub_rn(xd, xs);
            if (df > 0.0f) sign = 1.0f;
            if (df < 0.0f) sign = -1.0f;
            if (df == 0.0f) sign = 0.0f;
            r = sign;
        } else if (ln == 2) {
            const float v = a.mode == 2 ? xd : __fsub_rn(xs, xd);
            intseis = gf == 1 ? __fadd_rn(intseis, __fmul_rn(dt, v)) : v;
            r = intseis;
            if (a.timewin == 5) {
                const float tj = __fmul_rn((float)(t + 1), dt);
                if (tj >= t0) {
                    const double u = (double)__fsub_rn(tj, t0);
                    r = __double2float_rn(__dmul_rn((double)r, exp(__dmul_rn(-(double)a.gamma, __dmul_rn(u, u)))));
                }
            }
            L2 = __dadd_rn(L2, __dmul_rn(__dmul_rn(0.5, (double)r), (double)r));
        } else if (ln == 3) {
            const float df = __fsub_rn(xd, xs);
            r = __fdiv_rn(df, __fadd_rn(1.0f, __fmul_rn(df, df)));
        } else if (ln == 4) {
            r = __double2float_rn(tanh((double)__fsub_rn(xd, xs)));
        } else if (ln == 5) {
            float ys = xs, yd = xd;
            if (gf == 1) {   // the integrated traces, computed before the replacement of sample 1
                cs5 = __fadd_rn(cs5, S(t));
                cd5 = __fadd_rn(cd5, D(t));
                ys = __fmul_rn(dt, cs5);
                yd = __fmul_rn(dt, cd5);
            }
            r = __fsub_rn(__fdiv_rn(__fmul_rn(ys, dms), __fadd_rn(tmp5, 0.0f)), __fdiv_rn(yd, __fadd_rn(tmp15, 0.0f)));
            L2 = __dadd_rn(L2, -(double)__fdiv_rn(__fmul_rn(yd, ys), __fadd_rn(__fmul_rn(ad, asn), 0.0f)));
        } else if (ln == 8) {
            // AGC of the observed trace before N_ORDER (:388-396), recomputed per sample in the reference's order
            float acc = 0.0f;
            for (int h = max(t - a.nagc, 0); h <= min(t + a.nagc, nt - 1); h++) {
                const float dh_ = D(h);
                acc = __fadd_rn(acc, __fmul_rn(dh_, dh_));
            }
            const float agc = __fsqrt_rn(acc);
            r = 0.0f;
            if (fabsf(agc) > 0.0f) {
                const float df = __fsub_rn(xs, xd);
                r = __fdiv_rn(df, agc);
                L2 = __dadd_rn(L2, __ddiv_rn(__dmul_rn(__dmul_rn(0.5, (double)df), (double)df), (double)agc));
            }
            (void)rawd;
        }
        rs[nt - 1 - t] = r;
    }
    part[l] = L2;
}

// The misfit: the per-trace double sums added in a fixed order by one block of
// SUM_THREADS threads (thread t adds traces t, t + SUM_THREADS, ... in order, then a
// shared-memory tree), so repeated calls give the same bits.
constexpr int SUM_THREADS = 1024;
__global__ void __launch_bounds__(SUM_THREADS) k_sum_partials(const double *__restrict__ part, int n,
                                                              double *__restrict__ out)
{
    __shared__ double sh[SUM_THREADS];
    double s = 0.0;
    for (int l = threadIdx.x; l < n; l += SUM_THREADS) s = __dadd_rn(s, part[l]);
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = SUM_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] = __dadd_rn(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

}   // namespace

// Validates the options; returns the AGC half window in *nagc.
extern "C" int dn_residual_check(const dn_residual_opts *o, float dt, int *nagc)
{
    if (!o) return dn_fail(DN_EINVAL, "residual: null options");
    if (o->lnorm == 6) return dn_fail(DN_ENOTSUP, "LNORM 6 (envelope misfit) needs a Hilbert transform (FFTW)");
    if (o->lnorm < 1 || o->lnorm > 8) return dn_fail(DN_EINVAL, "LNORM %d", o->lnorm);
    if (o->grad_form != 1 && o->grad_form != 2) return dn_fail(DN_EINVAL, "GRAD_FORM must be 1 or 2");
    if (o->lnorm == 8 && o->grad_form != 2) return dn_fail(DN_EINVAL, "LNORM 8 needs GRAD_FORM 2");
    if (o->mode == 2 && o->lnorm != 2) return dn_fail(DN_EINVAL, "the RTM source (MODE 2) is defined for LNORM 2");
    if (o->n_order < 0 || o->n_order > MAX_NORDER) return dn_fail(DN_EINVAL, "N_ORDER %d (0..%d)", o->n_order, MAX_NORDER);
    if (o->timewin != 0 && o->timewin != 5)
        return dn_fail(DN_ENOTSUP, "TIMEWIN %d (picked-time windows) is not supported; 0 or 5", o->timewin);
    if (o->timewin == 5 && o->lnorm != 2) return dn_fail(DN_EINVAL, "TIMEWIN 5 applies to LNORM 2");
    if (o->offset_mute < 0 || o->offset_mute > 2) return dn_fail(DN_EINVAL, "OFFSET_MUTE %d", o->offset_mute);
    *nagc = 0;
    if (o->lnorm == 8) {
        const float den = (o->fc_start + o->fc_end) * dt;
        const double w = 2.0 / den;
        if (!(w >= 0.0 && w < 1e7)) return dn_fail(DN_EINVAL, "LNORM 8: FC_START + FC_END must be positive");
        *nagc = (int)floor(w + 0.5);
    }
    return DN_OK;
}

// Launches the residual on `stream`: scratch holds ntr + 1 doubles; s1/s2 two
// [ntr][nt] float arrays (LNORM 7 only); kill/rec_i/rec_j device arrays or null.
extern "C" int dn_residual_launch_ex(const float *syn_tm, const float *obs, float *res, int ntr, int nt, float dt,
                                     float dh, const dn_residual_opts *o, int nagc, const int *kill, const int *rec_i,
                                     const int *rec_j, float *s1, float *s2, double *scratch, cudaStream_t stream)
{
    ResArgs a = {};
    a.lnorm = o->lnorm;
    a.grad_form = o->grad_form;
    a.mode = o->mode;
    a.n_order = o->n_order;
    a.comp_weight = o->comp_weight > 0;
    a.wscale = o->c_vp * o->c_rho;
    a.dt = dt;
    a.dh = dh;
    a.nagc = nagc;
    a.kill = kill;
    a.offset_mute = o->offset_mute;
    a.timewin = o->timewin;
    a.offsetc = o->offsetc;
    a.gamma = o->gamma;
    a.twl = o->twlength_minus;
    a.rec_i = rec_i;
    a.rec_j = rec_j;
    a.src_x = o->src_x;
    a.src_z = o->src_z;
    a.s1 = s1;
    a.s2 = s2;
    k_residual<<<(ntr + 127) / 128, 128, 0, stream>>>(syn_tm, obs, res, ntr, nt, a, scratch);
    k_sum_partials<<<1, SUM_THREADS, 0, stream>>>(scratch, ntr, scratch + ntr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "residual kernels: %s", cudaGetErrorString(e));
    return DN_OK;
}

// Launches the L2 residual (LNORM 2, no trace selection) or, with rtm, the RTM
// source on `stream` with `scratch` holding ntr + 1 doubles.
extern "C" int dn_adjoint_source_launch(const float *syn_tm, const float *obs, float *res, int ntr, int nt, float dt,
                                        int grad_form, int rtm, double *scratch, cudaStream_t stream)
{
    dn_residual_opts o = {};
    o.lnorm = 2;
    o.grad_form = grad_form;
    o.mode = rtm ? 2 : 1;
    return dn_residual_launch_ex(syn_tm, obs, res, ntr, nt, dt, 0.0f, &o, 0, nullptr, nullptr, nullptr, nullptr,
                                 nullptr, scratch, stream);
}

extern "C" int dn_residual_l2_launch(const float *syn_tm, const float *obs, float *res, int ntr, int nt, float dt,
                                     int grad_form, double *scratch, cudaStream_t stream)
{
    return dn_adjoint_source_launch(syn_tm, obs, res, ntr, nt, dt, grad_form, 0, scratch, stream);
}

// Device buffers for one generalized residual call (scratch, LNORM 7 arrays,
// per-trace tables), freed by residual_bufs_free.
struct ResBufs {
    char *buf = nullptr;
    double *scratch = nullptr;
    float *s1 = nullptr, *s2 = nullptr;
    int *kill = nullptr, *ri = nullptr, *rj = nullptr;
};
static int residual_bufs(ResBufs &b, int ntr, int nt, const dn_residual_opts *o, const int *rec_i, const int *rec_j,
                         cudaStream_t st)
{
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const bool pos = o->offset_mute || o->timewin == 5;
    if (pos && (!rec_i || !rec_j)) return dn_fail(DN_EINVAL, "residual: OFFSET_MUTE / TIMEWIN 5 need receiver positions");
    size_t off_s1 = up(sizeof(double) * (ntr + 1)), n7 = o->lnorm == 7 ? (size_t)ntr * nt : 0;
    size_t off_s2 = off_s1 + up(4 * n7), off_k = off_s2 + up(4 * n7);
    size_t off_i = off_k + (o->kill ? up(4 * (size_t)ntr) : 0), off_j = off_i + (pos ? up(4 * (size_t)ntr) : 0);
    size_t total = off_j + (pos ? up(4 * (size_t)ntr) : 0);
    if (dn_malloc(&b.buf, total) != cudaSuccess) {
        cudaGetLastError();
        return dn_fail(DN_ENOMEM, "residual: %zu bytes of device scratch", total);
    }
    b.scratch = (double *)b.buf;
    if (n7) {
        b.s1 = (float *)(b.buf + off_s1);
        b.s2 = (float *)(b.buf + off_s2);
    }
    if (o->kill) {
        b.kill = (int *)(b.buf + off_k);
        CU(cudaMemcpyAsync(b.kill, o->kill, 4 * (size_t)ntr, cudaMemcpyHostToDevice, st));
    }
    if (pos) {
        b.ri = (int *)(b.buf + off_i);
        b.rj = (int *)(b.buf + off_j);
        CU(cudaMemcpyAsync(b.ri, rec_i, 4 * (size_t)ntr, cudaMemcpyHostToDevice, st));
        CU(cudaMemcpyAsync(b.rj, rec_j, 4 * (size_t)ntr, cudaMemcpyHostToDevice, st));
    }
    return DN_OK;
}

extern "C" int dn_residual_run_ex(const float *syn_tm, const float *obs, float *res, int ntr, int nt, float dt, float dh,
                                  const int *rec_i, const int *rec_j, const dn_residual_opts *o, double *misfit,
                                  cudaStream_t st)
{
    int nagc;
    int rc = dn_residual_check(o, dt, &nagc);
    if (rc) return rc;
    ResBufs b;
    rc = residual_bufs(b, ntr, nt, o, rec_i, rec_j, st);
    if (!rc)
        rc = dn_residual_launch_ex(syn_tm, obs, res, ntr, nt, dt, dh, o, nagc, b.kill, b.ri, b.rj, b.s1, b.s2,
                                   b.scratch, st);
    double h = 0.0;
    if (!rc) {
        cudaError_t e = cudaMemcpyAsync(&h, b.scratch + ntr, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = dn_fail(DN_EDEVICE, "residual: %s", cudaGetErrorString(e));
    } else {
        cudaStreamSynchronize(st);
    }
    dn_free(b.buf);
    if (!rc && misfit) *misfit = h;
    return rc;
}

extern "C" int dn_residual_ex(const float *syn_tm, const float *obs, float *res, int ntr, int nt, float dt, float dh,
                              const int *rec_i, const int *rec_j, const dn_residual_opts *o, double *misfit)
{
    if (!syn_tm || !obs || !res || ntr < 1 || nt < 1) return dn_fail(DN_EINVAL, "dn_residual_ex: bad arguments");
    return dn_residual_run_ex(syn_tm, obs, res, ntr, nt, dt, dh, rec_i, rec_j, o, misfit, 0);
}

extern "C" int dn_residual_l2(const float *syn_tm, const float *obs, float *res, int ntr, int nt, float dt,
                              int grad_form, double *l2)
{
    if (!syn_tm || !obs || !res || ntr < 1 || nt < 1)
        return dn_fail(DN_EINVAL, "dn_residual_l2: bad arguments");
    if (grad_form != 1 && grad_form != 2) return dn_fail(DN_EINVAL, "dn_residual_l2: GRAD_FORM must be 1 or 2");
    double *scratch = nullptr;
    cudaError_t e = dn_malloc(&scratch, sizeof(double) * ((size_t)ntr + 1));
    if (e != cudaSuccess) return dn_fail(DN_ENOMEM, "dn_residual_l2: scratch allocation failed");
    int st = dn_residual_l2_launch(syn_tm, obs, res, ntr, nt, dt, grad_form, scratch, 0);
    double h = 0.0;
    if (!st) {
        e = cudaMemcpy(&h, scratch + ntr, sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = dn_fail(DN_EDEVICE, "dn_residual_l2: %s", cudaGetErrorString(e));
    }
    dn_free(scratch);
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
// device) and caches it; make that first call before any stream capture.  The
// cached address belongs to the device's current context: after a
// cudaDeviceReset of that device it would point at freed memory, so a device
// reset between calls is not supported (as for every other object of this
// library).  The kernels run on the legacy default stream, which does not wait
// for work on non-blocking streams: the caller makes sure the producers of
// syn_tm and obs have finished (e.g. synchronises their stream) before the call.
// Nothing in the scratch has to start at zero: k_residual writes every
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
