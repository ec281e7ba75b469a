// Engine of the B200 P-SV propagator: device-resident models and shots,
// batched time loop (one launch per operation for all shots of a batch,
// captured in a CUDA graph), plain single-shot loop, gradient assembly and the
// C ABI declared in include/denise_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "dn_internal.h"
#include "dn_precond.h"
#include "dn_launch.cuh"
#include "dn_materials.cuh"

using namespace dn;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local char g_err[512] = "";

extern "C" int dn_fail(int code, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

extern "C" const char *dn_last_error(void) { return g_err; }

extern "C" int dn_version(int *major, int *minor)
{
    if (major) *major = DN_VERSION_MAJOR;
    if (minor) *minor = DN_VERSION_MINOR;
    return DN_OK;
}


extern "C" int dn_device_count(int *count)
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) n = 0;
    if (count) *count = n;
    return DN_OK;
}

extern "C" int dn_device_memory(int device, size_t *free_bytes, size_t *total_bytes)
{
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
    size_t f = 0, t = 0;
    e = cudaMemGetInfo(&f, &t);
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "cudaMemGetInfo: %s", cudaGetErrorString(e));
    f += dn_pool_idle_bytes(device);   // cached by the library, free for its next allocation
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return DN_OK;
}

// ---------------------------------------------------------------------------
// per-device state: one stream, a zero step counter for direct launches
// ---------------------------------------------------------------------------
struct DevState {
    cudaStream_t stream = nullptr;
    int *d_zero = nullptr;     // 0, used as the step base of direct launches
    int *d_step = nullptr;     // step base advanced by graph replays
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};
static std::mutex g_dev_mu;
static std::map<int, DevState> g_dev;
static thread_local double g_last_ms = 0.0;
static thread_local long long g_last_launches = 0;

static int dev_state(int device, DevState **out)
{
    std::lock_guard<std::mutex> lk(g_dev_mu);
    auto it = g_dev.find(device);
    if (it == g_dev.end()) {
        DevState st;
        CU(cudaSetDevice(device));
        CU(cudaStreamCreateWithFlags(&st.stream, cudaStreamNonBlocking));
        CU(dn_malloc(&st.d_zero, 2 * sizeof(int)));
        CU(cudaMemset(st.d_zero, 0, 2 * sizeof(int)));
        st.d_step = st.d_zero + 1;
        CU(cudaEventCreate(&st.ev0));
        CU(cudaEventCreate(&st.ev1));
        it = g_dev.emplace(device, st).first;
    }
    *out = &it->second;
    return DN_OK;
}

// ---------------------------------------------------------------------------
// model / shot objects
// ---------------------------------------------------------------------------
struct Layout {
    int nx, ny, pitch, rows;
    long long plane;   // floats per padded field
    long long origin;  // offset of the origin pointer inside a padded field
};

static Layout make_layout(int nx, int ny)
{
    Layout L;
    L.nx = nx;
    L.ny = ny;
    L.pitch = ((nx + 2 * DN_HX) + 31) / 32 * 32;
    L.rows = ny + 2 * DN_HZ;
    L.plane = (long long)L.pitch * L.rows;
    L.origin = (long long)(DN_HZ - 1) * L.pitch + (DN_HX - 1);
    return L;
}

enum { MF_RIP, MF_RJP, MF_UIPJP, MF_MU, MF_LAM, MF_RHO, MF_VP, MF_VS, MF_GMUSS, MF_GLAMSS,
       MF_CMUIPJP, MF_CTAUSIPJP, MF_CMU, MF_CTAUS, MF_CPI, MF_CTAUP, MF_COUNT };

struct dn_model {
    dn_params p;
    int device;
    float hc[7];
    Layout lay;
    int nfields;
    float *dmat = nullptr;         // nfields padded planes
    float *dpml = nullptr;         // 12 CPML vectors of 2 fw
    float *dsurf = nullptr;        // visco surface constants: 4 x nx
    float eta[DN_MAX_L], bip[DN_MAX_L], cip[DN_MAX_L], s_bjm[DN_MAX_L];
    void *dgrad = nullptr;         // stacked gradient: 3 x nx*ny (float or double), row-major [j][i]
    int grad64;
    int nshots = 0;
    float rdh = 0.0f;              // RN(1 / DH)
    int fastdiv = 0;               // div_markstein verified for DH on this device
    float *field(int f) const { return dmat + (long long)f * lay.plane + lay.origin; }
};

struct dn_shot {
    dn_model *m;
    dn_params p;                   // copy of the model parameters at creation
    // acquisition (host copies)
    int nsrc, ntr;
    std::vector<int> src_i, src_j, src_type, rec_i, rec_j;
    std::vector<float> src_azi, signals;
    int quelltyp_last;
    // device state
    char *dstate = nullptr;        // fields + psi + rpq, zeroed per run
    size_t state_bytes = 0;
    float *f[7];                   // vx vy sxx syy sxy vxp1 vyp1 (origin pointers)
    float *r = nullptr, *pmv = nullptr, *q = nullptr;
    float *psi[9];
    char *dacq = nullptr;          // source / receiver tables + signals
    int nsrc_cells;
    int *d_cell_i, *d_cell_j, *d_cell_start, *d_cell_count, *d_perm, *d_src_type, *d_rec_i, *d_rec_j;
    double *d_nsin, *d_cos;
    float *d_signals;
    float *d_sec = nullptr;        // [ncomp=5][nt][ntr]
    float *d_res = nullptr;        // [3][ntr][nt]
    int has_res[3] = {0, 0, 0};
    void *d_snap = nullptr;
    float *d_snap_scale = nullptr;
    int nsnap = 0, zch = 16, bx = 128, tiles_x = 0, tiles = 0;
    int kern = DN_KERN_PAIRED;     // stencil kernel variant (the batch runs its first shot's)
    bool auto_rows = false;        // tile rows chosen per batch (batch_rows)
    bool rec_dup = false;          // two receivers share a cell
    // fused elastic step (DN_KERN_FUSED on an eligible shot): the second set of fields and
    // velocity CPML memory (inside dstate, so zeroed with it) and the tile rows
    bool fz = false;
    int fzc = 0;
    float *fb[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    float *fpsi[4] = {nullptr, nullptr, nullptr, nullptr};
    void *d_acc = nullptr;         // wc, wcu, wcrho (float or double) + Ws, Wr
    int acc64;
    int *d_flag = nullptr;
    int stored = 0;                // a mode-0 run with snapshots completed
    int correlated = 0;            // a mode-1 run completed
    // checkpointed adjoint (ckpt_steps > 0): full states at segment starts, and the
    // adjoint's own wavefield state (the forward state is recomputed per segment)
    int nseg = 0;
    char *dckpt = nullptr;         // nseg x state_bytes
    char *dstate2 = nullptr;       // adjoint state, state_bytes
};

static size_t snap_elem_bytes(int prec) { return prec == DN_SNAP_F32 ? 4 : 2; }

static int validate_params(const dn_params *p)
{
    if (!p) return dn_fail(DN_EINVAL, "null params");
    if (p->nx < 1 || p->ny < 1) return dn_fail(DN_EINVAL, "NX and NY must be positive (got %d x %d)", p->nx, p->ny);
    if (p->fdorder < 2 || p->fdorder > 12 || (p->fdorder & 1))
        return dn_fail(DN_EINVAL, "Error in selection of FD coefficients: wrong FDORDER (%d)", p->fdorder);
    if (p->maxrelerror < 0 || p->maxrelerror > 4)
        return dn_fail(DN_EINVAL, "Error in selection of FD coefficients: wrong choice of maximum relative error (%d)",
                       p->maxrelerror);
    if (p->nt < 2) return dn_fail(DN_EINVAL, "NT must be at least 2 (got %d)", p->nt);
    if (!(p->dt > 0.0f) || !(p->dh > 0.0f)) return dn_fail(DN_EINVAL, "DT and DH must be positive");
    if (p->fw < 0) return dn_fail(DN_EINVAL, "FW must be >= 0");
    if (p->boundary != 0) return dn_fail(DN_ENOTSUP, "BOUNDARY=%d (periodic edges) is not built; use 0", p->boundary);
    if (p->L < 0 || p->L > DN_MAX_L) return dn_fail(DN_EINVAL, "L must be in 0..%d", DN_MAX_L);
    if (p->invmat1 != 1) return dn_fail(DN_ENOTSUP, "INVMAT1=%d is not built; use 1 (vp, vs, rho)", p->invmat1);
    if (p->grad_form != 1) return dn_fail(DN_ENOTSUP, "GRAD_FORM=%d is not built; use 1", p->grad_form);
    if (p->store_snapshots && p->dtinv < 1) return dn_fail(DN_EINVAL, "DTINV must be >= 1");
    if (p->ckpt_steps < 0 || (p->ckpt_steps > 0 && (!p->store_snapshots || p->ckpt_steps % p->dtinv)))
        return dn_fail(DN_EINVAL, "ckpt_steps must be 0 or a positive multiple of DTINV with snapshots stored");
    if (p->snap_precision < 0 || p->snap_precision > 2) return dn_fail(DN_EINVAL, "bad snapshot precision");
    if (p->seismo < 0 || p->seismo > 4) return dn_fail(DN_EINVAL, "SEISMO must be 0..4");
    if (p->L > 0 && !(p->ts > 0.0f) && p->free_surf)
        return dn_fail(DN_EINVAL, "TS (1 / max source frequency) is needed by the viscoelastic free surface");
    for (int l = 0; l < p->L; l++)
        if (!(p->fl[l] > 0.0f)) return dn_fail(DN_EINVAL, "relaxation frequency FL[%d] must be positive", l + 1);
    return DN_OK;
}

static void file_to_padded(const Layout &L, const float *file, std::vector<float> &pad, long long plane_off)
{
    // x-major file order to the padded [z][x] plane, in 32 x 32 blocks so that
    // both sides of the transposition stay in cache
    float *dst = pad.data() + plane_off + L.origin;
    for (int i0 = 1; i0 <= L.nx; i0 += 32)
        for (int j0 = 1; j0 <= L.ny; j0 += 32)
            for (int i = i0; i < i0 + 32 && i <= L.nx; i++)
                for (int j = j0; j < j0 + 32 && j <= L.ny; j++)
                    dst[(long long)j * L.pitch + i] = file[(size_t)(i - 1) * L.ny + (j - 1)];
}

extern "C" int dn_model_footprint(const dn_params *p, size_t *bytes)
{
    int st = validate_params(p);
    if (st) return st;
    Layout L = make_layout(p->nx, p->ny);
    int nf = p->L > 0 ? MF_COUNT : MF_CMUIPJP;
    size_t b = (size_t)nf * L.plane * 4 + 12 * 2 * (size_t)std::max(p->fw, 1) * 4 + 4 * (size_t)p->nx * 4;
    b += 3 * (size_t)p->nx * p->ny * (p->grad_accum == DN_ACC_F64 ? 8 : 4);
    if (bytes) *bytes = b;
    return DN_OK;
}

// ---------------------------------------------------------------------------
// Exhaustive check of the fast division by DH (div_markstein) against
// __fdiv_rn over all 2^32 float dividends; ~5 ms once per distinct DH and
// device.  DN_FASTDIV=0 skips it and keeps the general division.
// ---------------------------------------------------------------------------
__global__ void k_fastdiv_check(float d, unsigned long long n, unsigned long long *bad, float *y_out)
{
    const float y = __frcp_rn(d);
    if (blockIdx.x == 0 && threadIdx.x == 0) *y_out = y;
    unsigned long long nbad = 0;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        const float a = __uint_as_float((unsigned)k);
        const float q0 = __fdiv_rn(a, d), q1 = div_markstein(a, d, y);
        if (__float_as_uint(q0) != __float_as_uint(q1) && !(q0 != q0 && q1 != q1)) nbad++;
    }
    if (nbad) atomicAdd(bad, nbad);
}

static std::mutex g_fastdiv_mu;
static std::map<std::pair<int, unsigned>, std::pair<int, float>> g_fastdiv;   // (device, DH bits) -> (ok, y)

static int fastdiv_setup(int device, float dh, int *ok, float *y)
{
    unsigned bits;
    memcpy(&bits, &dh, 4);
    std::lock_guard<std::mutex> lk(g_fastdiv_mu);
    auto it = g_fastdiv.find({device, bits});
    if (it != g_fastdiv.end()) {
        *ok = it->second.first;
        *y = it->second.second;
        return DN_OK;
    }
    const char *ev = getenv("DN_FASTDIV");
    const bool enabled = !(ev && ev[0] == '0');
    char *buf = nullptr;
    if (dn_malloc(&buf, 16) != cudaSuccess) return dn_fail(DN_ENOMEM, "fast division check: allocation failed");
    unsigned long long hbad = 0;
    float hy = 0.0f;
    cudaError_t e = cudaMemset(buf, 0, 16);
    if (e == cudaSuccess) {
        // disabled: n = 0 computes y only
        k_fastdiv_check<<<148 * 8, 256>>>(dh, enabled ? (1ull << 32) : 0ull, (unsigned long long *)buf,
                                          (float *)(buf + 8));
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(&hbad, buf, 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&hy, buf + 8, 4, cudaMemcpyDeviceToHost);
    dn_free(buf);
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "fast division check: %s", cudaGetErrorString(e));
    *ok = enabled && hbad == 0;
    *y = hy;
    g_fastdiv[{device, bits}] = {*ok, hy};
    return DN_OK;
}

// The material planes of m from the model files on the device (k_file_to_plane, k_materials),
// enqueued on stream cs; the staging of the files is released in stream order.
static cudaError_t device_materials(dn_model *m, const float *vp, const float *vs, const float *rho, const float *qp,
                                    const float *qs, cudaStream_t cs)
{
    const dn_params &p = m->p;
    const Layout &L = m->lay;
    const size_t n = (size_t)p.nx * p.ny;
    const bool visc = p.L > 0, q = visc && p.honor_q;
    const int nraw = q ? 5 : 3;
    cudaError_t e = cudaMemsetAsync(m->dmat, 0, (size_t)m->nfields * L.plane * 4, cs);
    float *raw = nullptr, *qpl = nullptr;
    if (e == cudaSuccess) e = cudaMallocAsync((void **)&raw, n * nraw * 4, cs);
    if (e == cudaSuccess && q) e = cudaMallocAsync((void **)&qpl, (size_t)2 * L.plane * 4, cs);
    if (e == cudaSuccess && q) e = cudaMemsetAsync(qpl, 0, (size_t)2 * L.plane * 4, cs);
    const float *src[5] = {rho, vs, vp, qs, qp};
    for (int k = 0; k < nraw && e == cudaSuccess; k++)
        e = cudaMemcpyAsync(raw + k * n, src[k], n * 4, cudaMemcpyHostToDevice, cs);
    if (e == cudaSuccess) {
        const dim3 tg((p.ny + 31) / 32, (p.nx + 31) / 32), tb(32, 8);
        float *dst[5] = {m->field(MF_RHO), m->field(MF_VS), m->field(MF_VP), q ? qpl + L.origin : nullptr,
                         q ? qpl + L.plane + L.origin : nullptr};
        for (int k = 0; k < nraw; k++) k_file_to_plane<<<tg, tb, 0, cs>>>(raw + k * n, dst[k], p.nx, p.ny, L.pitch);
        MatPlanes M;
        M.rho = m->field(MF_RHO);
        M.vs = m->field(MF_VS);
        M.vp = m->field(MF_VP);
        M.qs = q ? dst[3] : nullptr;
        M.qp = q ? dst[4] : nullptr;
        M.rip = m->field(MF_RIP);
        M.rjp = m->field(MF_RJP);
        M.uipjp = m->field(MF_UIPJP);
        M.mu = m->field(MF_MU);
        M.lam = m->field(MF_LAM);
        M.gmuss = m->field(MF_GMUSS);
        M.glamss = m->field(MF_GLAMSS);
        M.c_muipjp = visc ? m->field(MF_CMUIPJP) : nullptr;
        M.c_tausipjp = visc ? m->field(MF_CTAUSIPJP) : nullptr;
        M.c_mu = visc ? m->field(MF_CMU) : nullptr;
        M.c_taus = visc ? m->field(MF_CTAUS) : nullptr;
        M.c_pi = visc ? m->field(MF_CPI) : nullptr;
        M.c_taup = visc ? m->field(MF_CTAUP) : nullptr;
        M.pitch = L.pitch;
        M.nx = p.nx;
        M.ny = p.ny;
        M.visc = visc;
        M.sumu = visc ? dn_visc_sumu(&p) : 0.0f;
        k_materials<<<dim3((p.nx + 127) / 128, p.ny), 128, 0, cs>>>(M);
        e = cudaGetLastError();
    }
    if (raw) cudaFreeAsync(raw, cs);
    if (qpl) cudaFreeAsync(qpl, cs);
    return e;
}

extern "C" int dn_model_create(const dn_params *p, const float *vp, const float *vs, const float *rho,
                               const float *qp, const float *qs, int device, dn_model **out)
{
    if (!out) return dn_fail(DN_EINVAL, "dn_model_create: null out");
    *out = nullptr;
    int st = validate_params(p);
    if (st) return st;
    if (!vp || !vs || !rho) return dn_fail(DN_EINVAL, "dn_model_create: vp, vs and rho are required");
    if (p->L > 0 && p->honor_q && (!qp || !qs)) return dn_fail(DN_EINVAL, "dn_model_create: honor_q needs qp and qs");
    dn_model *m = new dn_model();
    m->p = *p;
    m->device = device;
    m->lay = make_layout(p->nx, p->ny);
    m->nfields = p->L > 0 ? MF_COUNT : MF_CMUIPJP;
    m->grad64 = p->grad_accum == DN_ACC_F64;
    st = dn_holbergcoeff(p->fdorder, p->maxrelerror, m->hc);
    if (st) {
        delete m;
        return st;
    }
    const Layout &L = m->lay;
    const size_t n = (size_t)p->nx * p->ny;
    // the material planes come from the device (k_materials) unless DN_HOST_MATERIALS=1 asks
    // for the host set-up below; both give the same bits
    const char *hm = getenv("DN_HOST_MATERIALS");
    const bool host_mat = hm && strcmp(hm, "0") != 0;
    std::vector<float> host;
    std::vector<float> uipjp, rip, rjp, mu, lam, gmuss, glamss;
    if (host_mat) {
        host.assign((size_t)m->nfields * L.plane, 0.0f);
        uipjp.resize(n), rip.resize(n), rjp.resize(n), mu.resize(n), lam.resize(n), gmuss.resize(n), glamss.resize(n);
        st = dn_average_materials(p, vp, vs, rho, uipjp.data(), rip.data(), rjp.data());
        if (st) {
            delete m;
            return st;
        }
        for (size_t k = 0; k < n; k++) {
            // update_s_elastic_PML_PSV.c:442-444 and psv.c:333-334 (float, with the 2.0 promotion)
            float u = vs[k], pi = vp[k], r = rho[k];
            mu[k] = r * u * u;
            lam[k] = r * ((pi * pi) - 2 * u * u);
            float muss = r * u * u;
            gmuss[k] = muss;
            glamss[k] = (float)((double)(r * pi * pi) - 2.0 * (double)muss);
        }
        file_to_padded(L, rip.data(), host, MF_RIP * L.plane);
        file_to_padded(L, rjp.data(), host, MF_RJP * L.plane);
        file_to_padded(L, uipjp.data(), host, MF_UIPJP * L.plane);
        file_to_padded(L, mu.data(), host, MF_MU * L.plane);
        file_to_padded(L, lam.data(), host, MF_LAM * L.plane);
        file_to_padded(L, rho, host, MF_RHO * L.plane);
        file_to_padded(L, vp, host, MF_VP * L.plane);
        file_to_padded(L, vs, host, MF_VS * L.plane);
        file_to_padded(L, gmuss.data(), host, MF_GMUSS * L.plane);
        file_to_padded(L, glamss.data(), host, MF_GLAMSS * L.plane);
    }
    std::vector<float> surf;
    if (p->L > 0) {
        if (host_mat) {
            std::vector<float> a(n), b(n), c(n), d(n), e(n), f(n);
            st = dn_visc_cell_factors(p, vp, vs, rho, qp, qs, a.data(), b.data(), c.data(), d.data(), e.data(),
                                      f.data());
            if (st) {
                delete m;
                return st;
            }
            file_to_padded(L, a.data(), host, MF_CMUIPJP * L.plane);
            file_to_padded(L, b.data(), host, MF_CTAUSIPJP * L.plane);
            file_to_padded(L, c.data(), host, MF_CMU * L.plane);
            file_to_padded(L, d.data(), host, MF_CTAUS * L.plane);
            file_to_padded(L, e.data(), host, MF_CPI * L.plane);
            file_to_padded(L, f.data(), host, MF_CTAUP * L.plane);
        }
        float eta[DN_MAX_L];
        dn_visc_eta(p, eta, nullptr);
        for (int l = 0; l < p->L; l++) {
            m->eta[l] = eta[l];
            m->bip[l] = 1.0 / (1.0 + (eta[l] * 0.5));
            m->cip[l] = 1.0 - (eta[l] * 0.5);
            m->s_bjm[l] = eta[l] / (1.0 + (eta[l] * 0.5));   // surface_visc_PML_PSV.c:158
        }
        // surface row j = 1 (surface_visc_PML_PSV.c:34-49, 136-143): ws = 2 pi / TS
        surf.assign(4 * (size_t)p->nx, 0.0f);
        if (p->free_surf) {
            float ws = 2.0 * 3.141592653589793 * (1.0 / p->ts);
            float sumu = dn_visc_sum(p, ws), sumpi = sumu;
            for (int i = 1; i <= p->nx; i++) {
                size_t o = (size_t)(i - 1) * p->ny;   // j = 1
                float qsv = p->honor_q ? qs[o] : 30.0f, qpv = p->honor_q ? qp[o] : 30.0f;
                float taus = dn_visc_tau_from_q(qsv), taup = dn_visc_tau_from_q(qpv);
                float pu = vs[o], ppi = vp[o], prho = rho[o];
                float smu = (pu * pu * prho) / (1.0 + sumu * taus);
                float spi = (ppi * ppi * prho) / (1.0 + sumpi * taup);
                surf[0 * p->nx + i - 1] = smu;
                surf[1 * p->nx + i - 1] = spi;
                surf[2 * p->nx + i - 1] = taus;
                surf[3 * p->nx + i - 1] = taup;
            }
        }
    }
    std::vector<float> pml(12 * 2 * (size_t)std::max(p->fw, 1), 0.0f);
    if (p->fw > 0) {
        const size_t w = 2 * (size_t)p->fw;
        std::vector<float> scratch(8 * w);
        dn_pml P;
        P.d_x = &scratch[0 * w];
        P.alpha_prime_x = &scratch[1 * w];
        P.d_x_half = &scratch[2 * w];
        P.alpha_prime_x_half = &scratch[3 * w];
        P.d_y = &scratch[4 * w];
        P.alpha_prime_y = &scratch[5 * w];
        P.d_y_half = &scratch[6 * w];
        P.alpha_prime_y_half = &scratch[7 * w];
        P.K_x = &pml[0 * w];
        P.a_x = &pml[1 * w];
        P.b_x = &pml[2 * w];
        P.K_x_half = &pml[3 * w];
        P.a_x_half = &pml[4 * w];
        P.b_x_half = &pml[5 * w];
        P.K_y = &pml[6 * w];
        P.a_y = &pml[7 * w];
        P.b_y = &pml[8 * w];
        P.K_y_half = &pml[9 * w];
        P.a_y_half = &pml[10 * w];
        P.b_y_half = &pml[11 * w];
        st = dn_pml_profiles(p, &P);
        if (st) {
            delete m;
            return st;
        }
    }
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        delete m;
        return dn_fail(DN_EDEVICE, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
    }
    size_t gbytes = 3 * n * (m->grad64 ? 8 : 4);
    const size_t mat_bytes = (size_t)m->nfields * L.plane * 4;
    if (dn_malloc(&m->dmat, mat_bytes) != cudaSuccess || dn_malloc(&m->dpml, pml.size() * 4) != cudaSuccess ||
        dn_malloc(&m->dgrad, gbytes) != cudaSuccess ||
        (!surf.empty() && dn_malloc(&m->dsurf, surf.size() * 4) != cudaSuccess)) {
        cudaGetLastError();
        dn_model_destroy(m);
        return dn_fail(DN_ENOMEM, "dn_model_create: device allocation failed");
    }
    // uploads on a private stream, so that creating a model does not wait for runs in flight
    cudaStream_t cs = nullptr;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
        dn_model_destroy(m);
        return dn_fail(DN_EDEVICE, "dn_model_create: stream creation failed");
    }
    bool up = cudaMemcpyAsync(m->dpml, pml.data(), pml.size() * 4, cudaMemcpyHostToDevice, cs) == cudaSuccess &&
              cudaMemsetAsync(m->dgrad, 0, gbytes, cs) == cudaSuccess &&
              (surf.empty() ||
               cudaMemcpyAsync(m->dsurf, surf.data(), surf.size() * 4, cudaMemcpyHostToDevice, cs) == cudaSuccess);
    if (up && host_mat) up = cudaMemcpyAsync(m->dmat, host.data(), mat_bytes, cudaMemcpyHostToDevice, cs) == cudaSuccess;
    if (up && !host_mat) up = device_materials(m, vp, vs, rho, qp, qs, cs) == cudaSuccess;
    const bool done = up && cudaStreamSynchronize(cs) == cudaSuccess;
    cudaStreamDestroy(cs);
    if (!done) {
        cudaGetLastError();
        dn_model_destroy(m);
        return dn_fail(DN_EDEVICE, "dn_model_create: upload failed");
    }
    st = fastdiv_setup(device, p->dh, &m->fastdiv, &m->rdh);
    if (st) {
        dn_model_destroy(m);
        return st;
    }
    *out = m;
    return DN_OK;
}

extern "C" int dn_model_destroy(dn_model *m)
{
    if (!m) return DN_OK;
    cudaSetDevice(m->device);
    dn_free(m->dmat);
    dn_free(m->dpml);
    dn_free(m->dsurf);
    dn_free(m->dgrad);
    delete m;
    return DN_OK;
}

extern "C" int dn_model_params(const dn_model *m, dn_params *out)
{
    if (!m || !out) return dn_fail(DN_EINVAL, "null argument");
    *out = m->p;
    return DN_OK;
}

extern "C" int dn_model_get_material(const dn_model *m, int which, float *out)
{
    if (!m || !out) return dn_fail(DN_EINVAL, "null argument");
    if (which < 0 || which >= m->nfields)
        return dn_fail(DN_EINVAL, "dn_model_get_material: plane %d of %d", which, m->nfields);
    const Layout &L = m->lay;
    std::vector<float> h(L.plane);
    CU(cudaSetDevice(m->device));
    CU(cudaMemcpy(h.data(), m->dmat + (long long)which * L.plane, L.plane * 4, cudaMemcpyDeviceToHost));
    for (int i = 1; i <= L.nx; i++)
        for (int j = 1; j <= L.ny; j++) out[(size_t)(i - 1) * L.ny + (j - 1)] = h[L.origin + (size_t)j * L.pitch + i];
    return DN_OK;
}

// ---------------------------------------------------------------------------
// shots
// ---------------------------------------------------------------------------
// Tile shapes and kernel variants of new shots: rules set by dn_set_tile_shape /
// dn_set_kernel_rule (the autotuner of denise_b200/tune.py measures them per
// FDORDER, L, snapshot class and grid size on the device) after the built-in
// ones below, the last matching rule winning; DN_TILE="WxZ" overrides the tile.
struct TileRule {
    int fdorder, L;
    long long cells_min, cells_max;
    int bx, zch;
    int store;     // -1: any shot; 0 / 1: shots that do not / do store snapshots
    int variant;   // DN_KERN_* stencil kernels (register blocking); -1: the default
};
static std::mutex g_tile_mu;
// Built-in rules: none.  The table denise_b200.tune measured on a B200
// (denise_b200/tiles_b200.json: FDORDER 4, 8, 12 x L 0, 3 x snapshot class x
// grids of 0.18 M and 1.2 M cells; forward batches of 32 shots, storing batches
// of 8) picks the default of tile_choice in 16 of its 18 classes and beats it by
// 1.0 % and 0.4 % in the other two, within the run-to-run spread.
static std::vector<TileRule> g_tile_rules;

static bool tile_ok(int bx, int zch) { return bx >= 32 && bx <= 256 && (bx % 32) == 0 && zch >= 1 && zch <= 256; }

static void tile_choice(const dn_params *p, int &bx, int &zch, int &variant, bool *deflt = nullptr)
{
    variant = DN_KERN_PAIRED;
    bool from_rule = false;
    // default tiles: 128 x 8 for forward shots of 480 k cells and more (batches
    // of 32 and 64 shots of 2000 x 600 cells step 2.3-4.1 % faster than at
    // 128 x 4), 128 x 4 for smaller forward grids (32 shots of 600 x 300: 3-8 %
    // faster than 128 x 8 for FDORDER 4, 8, 12 and L 0, 3) and for
    // snapshot-storing shots, whose batches the snapshots keep small (the 7-shot
    // 1700 x 500 FP16 forward + adjoint ran 449 ms per 1000 steps at 128 x 8 and
    // 416 ms at 128 x 4)
    bx = 128;
    zch = (p->store_snapshots || (long long)p->nx * p->ny < 480000) ? 4 : 8;
    const long long cells = (long long)p->nx * p->ny;
    {
        std::lock_guard<std::mutex> lk(g_tile_mu);
        for (const TileRule &r : g_tile_rules)
            if (r.fdorder == p->fdorder && r.L == p->L && cells >= r.cells_min && cells <= r.cells_max &&
                (r.store < 0 || r.store == (p->store_snapshots ? 1 : 0))) {
                bx = r.bx;
                zch = r.zch;
                if (r.variant >= 0) variant = r.variant;
                from_rule = true;
            }
    }
    const char *ev = getenv("DN_TILE");
    if (ev) {
        int a = 0, b = 0;
        if (sscanf(ev, "%dx%d", &a, &b) == 2 && tile_ok(a, b)) {
            bx = a;
            zch = b;
            from_rule = true;
        }
    }
    if (deflt) *deflt = !from_rule;
}

// Rows per tile of a batch of shots that keep their tiles open (no snapshots, no
// rule, no DN_TILE): the best of 1, 2, 4, 8 rows depends on the cells of the whole
// batch, not of one shot.  Measured on a B200 (600 x 300 and 2000 x 600 grids, 1-32
// shots, forward): one row up to 1.3 M cells (one 600 x 300 shot: 24.0 us a step
// against 40.8 at 4 rows), two up to 5 M, four up to 16 M (viscoelastic: 30 M), eight
// above (64 shots of 2000 x 600).  DN_AUTO_ROWS=0 keeps each shot's own tile.
static int batch_rows(long long cells, int L)
{
    const char *ev = getenv("DN_AUTO_ROWS");
    if (ev && strcmp(ev, "0") == 0) return 0;
    if (cells < 1300000) return 1;
    if (cells < 5000000) return 2;
    if (cells < (L > 0 ? 30000000LL : 16000000LL)) return 4;
    return 8;
}

static void tile_shape(const dn_params *p, int &bx, int &zch)
{
    int v;
    tile_choice(p, bx, zch, v);
}

extern "C" int dn_set_kernel_rule(int fdorder, int L, int store, long long cells_min, long long cells_max, int bx,
                                  int zch, int variant)
{
    if (fdorder < 2 || fdorder > 12 || (fdorder % 2) || L < 0 || L > DN_MAX_L || cells_min > cells_max ||
        store < -1 || store > 1)
        return dn_fail(DN_EINVAL, "dn_set_kernel_rule: bad class");
    if (!tile_ok(bx, zch))
        return dn_fail(DN_EINVAL, "dn_set_kernel_rule: %d x %d (width a multiple of 32 up to 256, 1-256 rows)", bx,
                       zch);
    if (variant < -1 || variant > DN_KERN_FUSED) return dn_fail(DN_EINVAL, "dn_set_kernel_rule: variant %d", variant);
    std::lock_guard<std::mutex> lk(g_tile_mu);
    for (TileRule &r : g_tile_rules)
        if (r.fdorder == fdorder && r.L == L && r.cells_min == cells_min && r.cells_max == cells_max &&
            r.store == store) {
            r.bx = bx;
            r.zch = zch;
            r.variant = variant;
            return DN_OK;
        }
    g_tile_rules.push_back({fdorder, L, cells_min, cells_max, bx, zch, store, variant});
    return DN_OK;
}

extern "C" int dn_set_tile_shape(int fdorder, int L, long long cells_min, long long cells_max, int bx, int zch)
{
    return dn_set_kernel_rule(fdorder, L, -1, cells_min, cells_max, bx, zch, -1);
}

extern "C" int dn_clear_tile_shapes(void)
{
    std::lock_guard<std::mutex> lk(g_tile_mu);
    g_tile_rules.clear();
    return DN_OK;
}

extern "C" int dn_get_tile_shape(const dn_params *p, int *bx, int *zch)
{
    if (!p || !bx || !zch) return dn_fail(DN_EINVAL, "dn_get_tile_shape: null argument");
    tile_shape(p, *bx, *zch);
    return DN_OK;
}

extern "C" int dn_get_kernel_choice(const dn_params *p, int *bx, int *zch, int *variant)
{
    if (!p || !bx || !zch || !variant) return dn_fail(DN_EINVAL, "dn_get_kernel_choice: null argument");
    tile_choice(p, *bx, *zch, *variant);
    return DN_OK;
}

static int shot_counts(const dn_params *p, int bx, int zch, int &tiles_x, int &tiles, int &nsnap)
{
    tiles_x = (p->nx + bx - 1) / bx;
    tiles = tiles_x * ((p->ny + zch - 1) / zch);
    nsnap = p->store_snapshots ? (int)ceil((float)p->nt / (float)p->dtinv) : 0;   // FD_PSV.c:82
    if (p->store_snapshots && p->ckpt_steps > 0) nsnap = std::min(nsnap, p->ckpt_steps / p->dtinv);   // one segment
    return DN_OK;
}

// shots of this class run the fused elastic step (k_step_el_fused) in their forward runs:
// elastic, no snapshots, variant DN_KERN_FUSED (a rule, or DN_FUSED=1 / 0 in the environment)
static bool fused_class(const dn_params *p, int variant)
{
    if (p->L != 0 || p->store_snapshots) return false;
    const char *ev = getenv("DN_FUSED");
    if (ev) return strcmp(ev, "0") != 0;
    return variant == DN_KERN_FUSED;
}

// rows per tile of the fused step: about DN_FUSED_ROWS (default 96) in equal chunks,
// at least R + 1 so that the top tile holds the rows the free surface reads
static int fused_rows(const dn_params *p)
{
    const char *ev = getenv("DN_FUSED_ROWS");
    int z = ev && atoi(ev) > 0 ? atoi(ev) : 96;
    z = std::max(z, p->fdorder / 2 + 1);
    const int chunks = std::max(1, (p->ny + z - 1) / z);
    return std::max((p->ny + chunks - 1) / chunks, std::min(p->ny, p->fdorder / 2 + 1));
}

extern "C" int dn_shot_footprint(const dn_params *p, int ntr, int store, size_t *bytes)
{
    int st = validate_params(p);
    if (st) return st;
    Layout L = make_layout(p->nx, p->ny);
    int bx, zch, tx, tiles, nsnap;
    dn_params q = *p;
    q.store_snapshots = store;
    tile_shape(&q, bx, zch);
    shot_counts(&q, bx, zch, tx, tiles, nsnap);
    size_t b = (size_t)(7 + 3 * p->L) * L.plane * 4;
    b += (size_t)9 * 2 * std::max(p->fw, 1) * std::max(p->nx, p->ny) * 4;
    b += (size_t)5 * p->nt * std::max(ntr, 1) * 4 + (size_t)3 * p->nt * std::max(ntr, 1) * 4;
    b += (size_t)nsnap * 5 * tiles * bx * zch * snap_elem_bytes(p->snap_precision);
    if (store && p->ckpt_steps > 0) {   // checkpoints and the adjoint state
        const size_t nseg = (p->nt + p->ckpt_steps - 1) / p->ckpt_steps;
        b += (nseg + 1) * ((size_t)(7 + 3 * p->L) * L.plane * 4 + (size_t)9 * 2 * std::max(p->fw, 1) *
                           std::max(p->nx, p->ny) * 4);
    }
    b += (size_t)p->nx * p->ny * (3 * (p->grad_accum == DN_ACC_F64 ? 8 : 4) + 8);
    int variant;
    tile_choice(&q, bx, zch, variant);
    if (fused_class(&q, variant))   // the fused step's second set of fields and CPML memory
        b += (size_t)5 * L.plane * 4 + (size_t)4 * 2 * std::max(p->fw, 1) * std::max(p->nx, p->ny) * 4;
    if (bytes) *bytes = b;
    return DN_OK;
}

template <typename T> static T *carve(char *&cur, size_t count)
{
    T *r = (T *)cur;
    size_t b = (count * sizeof(T) + 255) & ~(size_t)255;
    cur += b;
    return r;
}
static size_t carve_size(size_t count, size_t elem) { return (count * elem + 255) & ~(size_t)255; }

extern "C" int dn_shot_create(dn_model *m, const dn_acq *acq, dn_shot **out)
{
    if (!m || !acq || !out) return dn_fail(DN_EINVAL, "dn_shot_create: null argument");
    *out = nullptr;
    const dn_params *p = &m->p;
    if (acq->nsrc < 0 || acq->ntr < 0) return dn_fail(DN_EINVAL, "negative source/receiver count");
    if (acq->nsrc > 0 && (!acq->src_i || !acq->src_j || !acq->signals))
        return dn_fail(DN_EINVAL, "sources need src_i, src_j and signals");
    if (acq->ntr > 0 && (!acq->rec_i || !acq->rec_j)) return dn_fail(DN_EINVAL, "receivers need rec_i and rec_j");
    for (int l = 0; l < acq->nsrc; l++) {
        if (acq->src_i[l] < 1 || acq->src_i[l] > p->nx || acq->src_j[l] < 1 || acq->src_j[l] > p->ny)
            return dn_fail(DN_EINVAL, "source %d at grid point (%d,%d) lies outside the %d x %d grid", l + 1,
                           acq->src_i[l], acq->src_j[l], p->nx, p->ny);
        int ty = acq->src_type ? acq->src_type[l] : 1;
        if (ty < 1 || ty > 5) return dn_fail(DN_ENOTSUP, "source type QUELLTYP=%d is not built", ty);
        if (ty == 5 && (acq->src_i[l] < 2 || acq->src_j[l] < 2))
            return dn_fail(DN_EINVAL, "moment-tensor source %d needs i, j >= 2", l + 1);
    }
    for (int l = 0; l < acq->ntr; l++)
        if (acq->rec_i[l] < 1 || acq->rec_i[l] > p->nx || acq->rec_j[l] < 1 || acq->rec_j[l] > p->ny)
            return dn_fail(DN_EINVAL, "receiver %d at grid point (%d,%d) lies outside the grid", l + 1, acq->rec_i[l],
                           acq->rec_j[l]);
    dn_shot *s = new dn_shot();
    s->m = m;
    m->nshots++;
    s->p = *p;
    s->nsrc = acq->nsrc;
    s->ntr = acq->ntr;
    s->src_i.assign(acq->src_i, acq->src_i + acq->nsrc);
    s->src_j.assign(acq->src_j, acq->src_j + acq->nsrc);
    s->src_type.resize(acq->nsrc);
    s->src_azi.resize(acq->nsrc);
    for (int l = 0; l < acq->nsrc; l++) {
        s->src_type[l] = acq->src_type ? acq->src_type[l] : 1;
        s->src_azi[l] = acq->src_azi ? acq->src_azi[l] : 0.0f;
    }
    s->signals.assign(acq->signals, acq->signals + (size_t)acq->nsrc * p->nt);
    s->rec_i.assign(acq->rec_i, acq->rec_i + acq->ntr);
    s->rec_j.assign(acq->rec_j, acq->rec_j + acq->ntr);
    {
        std::vector<long long> cells(acq->ntr);
        for (int l = 0; l < acq->ntr; l++) cells[l] = (long long)acq->rec_j[l] * (p->nx + 2) + acq->rec_i[l];
        std::sort(cells.begin(), cells.end());
        s->rec_dup = std::adjacent_find(cells.begin(), cells.end()) != cells.end();
    }
    s->quelltyp_last = acq->nsrc > 0 ? s->src_type[acq->nsrc - 1] : 0;
    bool deflt = false;
    tile_choice(p, s->bx, s->zch, s->kern, &deflt);
    s->auto_rows = deflt && !p->store_snapshots;
    shot_counts(p, s->bx, s->zch, s->tiles_x, s->tiles, s->nsnap);
    s->acc64 = p->grad_accum == DN_ACC_F64;

    // unique source cells, list order kept inside a cell
    std::vector<int> perm(acq->nsrc);
    for (int l = 0; l < acq->nsrc; l++) perm[l] = l;
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) {
        if (s->src_j[a] != s->src_j[b]) return s->src_j[a] < s->src_j[b];
        return s->src_i[a] < s->src_i[b];
    });
    std::vector<int> ci, cj, cs, cc;
    for (int k = 0; k < acq->nsrc; k++) {
        int l = perm[k];
        if (ci.empty() || ci.back() != s->src_i[l] || cj.back() != s->src_j[l]) {
            ci.push_back(s->src_i[l]);
            cj.push_back(s->src_j[l]);
            cs.push_back(k);
            cc.push_back(0);
        }
        cc.back()++;
    }
    s->nsrc_cells = (int)ci.size();
    std::vector<double> nsin(acq->nsrc), cosv(acq->nsrc);
    for (int l = 0; l < acq->nsrc; l++) {
        float azi_rad = s->src_azi[l] * 3.141592653589793 / 180;   // update_v_PML_PSV.c:743
        nsin[l] = -sin((double)azi_rad);   // C promotes the float argument to double
        cosv[l] = cos((double)azi_rad);
    }

    const Layout &L = m->lay;
    const int fw = p->fw;
    const size_t xf = (size_t)p->ny * 2 * std::max(fw, 1), zf = (size_t)2 * std::max(fw, 1) * p->nx;
    s->state_bytes = carve_size(L.plane, 4) * (7 + 3 * p->L) + carve_size(xf, 4) * 5 + carve_size(zf, 4) * 4;
    // the fused step takes shots with at most FZ_MAXSRC source cells and no moment-tensor source
    s->fz = fused_class(p, s->kern) && s->nsrc_cells <= FZ_MAXSRC;
    for (int l = 0; l < acq->nsrc; l++)
        if (s->src_type[l] == 5) s->fz = false;
    if (s->fz) {
        s->fzc = fused_rows(p);
        s->state_bytes += carve_size(L.plane, 4) * 5 + carve_size(xf, 4) * 2 + carve_size(zf, 4) * 2;
    }
    size_t acq_bytes = carve_size(std::max((size_t)s->nsrc_cells, (size_t)1), 4) * 4 +
                       carve_size(std::max((size_t)acq->nsrc, (size_t)1), 4) * 2 +
                       carve_size(std::max((size_t)acq->ntr, (size_t)1), 4) * 2 +
                       carve_size(std::max((size_t)acq->nsrc, (size_t)1), 8) * 2 +
                       carve_size(std::max((size_t)acq->nsrc * p->nt, (size_t)1), 4) + carve_size(1, 4);
    const size_t sec_n = (size_t)5 * p->nt * std::max(acq->ntr, 1);
    const size_t res_n = (size_t)3 * std::max(acq->ntr, 1) * p->nt;
    const size_t ncell = (size_t)p->nx * p->ny;
    const size_t acc_bytes = carve_size(ncell, s->acc64 ? 8 : 4) * 3 + carve_size(ncell, 4) * 2;
    const size_t snap_n = (size_t)s->nsnap * 5 * s->tiles * s->bx * s->zch;

    cudaError_t e = cudaSetDevice(m->device);
    if (e != cudaSuccess) {
        delete s;
        return dn_fail(DN_EDEVICE, "cudaSetDevice: %s", cudaGetErrorString(e));
    }
    bool ok = dn_malloc(&s->dstate, s->state_bytes) == cudaSuccess && dn_malloc(&s->dacq, acq_bytes) == cudaSuccess &&
              dn_malloc(&s->d_sec, sec_n * 4) == cudaSuccess && dn_malloc(&s->d_res, res_n * 4) == cudaSuccess &&
              dn_malloc(&s->d_acc, acc_bytes) == cudaSuccess;
    if (ok && s->nsnap > 0) {
        ok = dn_malloc(&s->d_snap, std::max(snap_n, (size_t)1) * snap_elem_bytes(p->snap_precision)) == cudaSuccess &&
             dn_malloc(&s->d_snap_scale, std::max((size_t)s->nsnap * 5 * s->tiles, (size_t)1) * 4) == cudaSuccess;
    }
    if (ok && p->store_snapshots && p->ckpt_steps > 0) {
        s->nseg = (p->nt + p->ckpt_steps - 1) / p->ckpt_steps;
        ok = dn_malloc(&s->dckpt, s->state_bytes * s->nseg) == cudaSuccess &&
             dn_malloc(&s->dstate2, s->state_bytes) == cudaSuccess;
    }
    if (!ok) {
        cudaGetLastError();
        dn_shot_destroy(s);
        return dn_fail(DN_ENOMEM, "dn_shot_create: device allocation failed (%.1f MB of snapshots)",
                       snap_n * snap_elem_bytes(p->snap_precision) / 1e6);
    }
    char *cur = s->dstate;
    for (int k = 0; k < 7; k++) s->f[k] = carve<float>(cur, L.plane) + L.origin;
    if (p->L > 0) {
        s->r = carve<float>(cur, L.plane * p->L) + L.origin;
        s->pmv = carve<float>(cur, L.plane * p->L) + L.origin;
        s->q = carve<float>(cur, L.plane * p->L) + L.origin;
        // carve reserved one plane per array above; the remaining planes follow contiguously
    }
    for (int k = 0; k < 5; k++) s->psi[k] = carve<float>(cur, xf);
    for (int k = 5; k < 9; k++) s->psi[k] = carve<float>(cur, zf);
    if (s->fz) {
        for (int k = 0; k < 5; k++) s->fb[k] = carve<float>(cur, L.plane) + L.origin;
        for (int k = 0; k < 2; k++) s->fpsi[k] = carve<float>(cur, xf);
        for (int k = 2; k < 4; k++) s->fpsi[k] = carve<float>(cur, zf);
    }
    // (the visco planes were carved with their full size)
    char *ac = s->dacq;
    s->d_cell_i = carve<int>(ac, std::max(s->nsrc_cells, 1));
    s->d_cell_j = carve<int>(ac, std::max(s->nsrc_cells, 1));
    s->d_cell_start = carve<int>(ac, std::max(s->nsrc_cells, 1));
    s->d_cell_count = carve<int>(ac, std::max(s->nsrc_cells, 1));
    s->d_perm = carve<int>(ac, std::max(acq->nsrc, 1));
    s->d_src_type = carve<int>(ac, std::max(acq->nsrc, 1));
    s->d_rec_i = carve<int>(ac, std::max(acq->ntr, 1));
    s->d_rec_j = carve<int>(ac, std::max(acq->ntr, 1));
    s->d_nsin = carve<double>(ac, std::max(acq->nsrc, 1));
    s->d_cos = carve<double>(ac, std::max(acq->nsrc, 1));
    s->d_signals = carve<float>(ac, std::max((size_t)acq->nsrc * p->nt, (size_t)1));
    s->d_flag = carve<int>(ac, 1);
    ok = true;
    // uploads on a private stream, so that creating a shot does not wait for runs in flight
    cudaStream_t us = nullptr;
    if (cudaStreamCreateWithFlags(&us, cudaStreamNonBlocking) != cudaSuccess) {
        dn_shot_destroy(s);
        return dn_fail(DN_EDEVICE, "dn_shot_create: stream creation failed");
    }
    auto up = [&](void *dst, const void *src, size_t b) {
        if (b && ok) ok = cudaMemcpyAsync(dst, src, b, cudaMemcpyHostToDevice, us) == cudaSuccess;
    };
    up(s->d_cell_i, ci.data(), ci.size() * 4);
    up(s->d_cell_j, cj.data(), cj.size() * 4);
    up(s->d_cell_start, cs.data(), cs.size() * 4);
    up(s->d_cell_count, cc.data(), cc.size() * 4);
    up(s->d_perm, perm.data(), perm.size() * 4);
    up(s->d_src_type, s->src_type.data(), s->src_type.size() * 4);
    up(s->d_rec_i, s->rec_i.data(), s->rec_i.size() * 4);
    up(s->d_rec_j, s->rec_j.data(), s->rec_j.size() * 4);
    up(s->d_nsin, nsin.data(), nsin.size() * 8);
    up(s->d_cos, cosv.data(), cosv.size() * 8);
    up(s->d_signals, s->signals.data(), s->signals.size() * 4);
    if (ok) ok = cudaMemsetAsync(s->d_flag, 0, 4, us) == cudaSuccess &&
                 cudaMemsetAsync(s->d_sec, 0, sec_n * 4, us) == cudaSuccess &&
                 cudaMemsetAsync(s->d_res, 0, res_n * 4, us) == cudaSuccess &&
                 cudaMemsetAsync(s->d_acc, 0, acc_bytes, us) == cudaSuccess &&
                 cudaMemsetAsync(s->dstate, 0, s->state_bytes, us) == cudaSuccess;
    const bool done = ok && cudaStreamSynchronize(us) == cudaSuccess;
    cudaStreamDestroy(us);
    if (!done) {
        cudaGetLastError();
        dn_shot_destroy(s);
        return dn_fail(DN_EDEVICE, "dn_shot_create: upload failed");
    }
    *out = s;
    return DN_OK;
}

extern "C" int dn_shot_kernel(const dn_shot *s, int *variant, int *fused)
{
    if (!s || !variant || !fused) return dn_fail(DN_EINVAL, "dn_shot_kernel: null argument");
    *variant = s->kern;
    *fused = s->fz ? 1 : 0;
    return DN_OK;
}

static void forget_shot(const dn_shot *s);

extern "C" int dn_shot_destroy(dn_shot *s)
{
    if (!s) return DN_OK;
    forget_shot(s);
    cudaSetDevice(s->m->device);
    dn_free(s->dstate);
    dn_free(s->dacq);
    dn_free(s->d_sec);
    dn_free(s->d_res);
    dn_free(s->d_snap);
    dn_free(s->d_snap_scale);
    dn_free(s->d_acc);
    dn_free(s->dckpt);
    dn_free(s->dstate2);
    s->m->nshots--;
    delete s;
    return DN_OK;
}

// accumulator views
static void *acc_ptr(const dn_shot *s, int k)
{
    const size_t ncell = (size_t)s->p.nx * s->p.ny;
    const size_t a = carve_size(ncell, s->acc64 ? 8 : 4);
    const size_t w = carve_size(ncell, 4);
    char *b = (char *)s->d_acc;
    if (k < 3) return b + k * a;
    return b + 3 * a + (k - 3) * w;
}

// source cells per shot up to which the stencil kernels apply the forward sources themselves
constexpr int SRC_IN_KERNEL = 8;

// a forward run (mode 0 or 2) of a shot with the second field set takes the fused step
static bool runs_fused(const dn_shot *s, int mode) { return s->fz && (mode == 0 || mode == 2); }

// rows per tile of shot s in a batch configured as c
static int eff_rows(const dn_shot *s, const LaunchCfg *c)
{
    return (c && c->auto_zch > 0 && s->auto_rows) ? c->auto_zch : s->zch;
}
static int eff_tiles(const dn_shot *s, const LaunchCfg *c)
{
    const int z = eff_rows(s, c);
    return ((s->p.nx + s->bx - 1) / s->bx) * ((s->p.ny + z - 1) / z);
}

// the descriptor of shot s in mode `mode` for a batch configured as c (the configuration the
// batch's kernels are launched with: tile rows, in-kernel sources)
static Inst make_inst(const dn_shot *s, int mode, const LaunchCfg *c)
{
    const dn_model *m = s->m;
    const dn_params &p = s->p;
    Inst I;
    memset(&I, 0, sizeof(I));
    I.nx = p.nx;
    I.ny = p.ny;
    I.nt = p.nt;
    I.pitch = m->lay.pitch;
    I.fw = p.fw;
    I.free_surf = p.free_surf;
    I.L = p.L;
    I.mode = mode;
    I.zch = eff_rows(s, c);
    I.tiles_x = s->tiles_x;
    I.tiles = eff_tiles(s, c);
    I.store = (mode == 0) && p.store_snapshots && s->nsnap > 0;
    I.dtinv = std::max(p.dtinv, 1);
    I.nsnap = s->nsnap;
    I.snap_prec = p.snap_precision;
    I.acc64 = s->acc64;
    I.eprecond = p.eprecond;
    I.seismo = p.seismo;
    I.DT = p.dt;
    I.DH = p.dh;
    I.rdh = m->rdh;
    I.fastdiv = m->fastdiv;
    I.dhi_el = p.dt / p.dh;
    I.dhi_vi = 1.0 / p.dh;
    I.dh1 = 1.0 / p.dh;
    I.dthalbe = p.dt / 2.0;
    for (int k = 0; k < 7; k++) I.hc[k] = m->hc[k];
    I.vx = s->f[0];
    I.vy = s->f[1];
    I.sxx = s->f[2];
    I.syy = s->f[3];
    I.sxy = s->f[4];
    I.vxp1 = s->f[5];
    I.vyp1 = s->f[6];
    I.r = s->r;
    I.p = s->pmv;
    I.q = s->q;
    I.plane = m->lay.plane;
    I.rip = m->field(MF_RIP);
    I.rjp = m->field(MF_RJP);
    I.uipjp = m->field(MF_UIPJP);
    I.mu = m->field(MF_MU);
    I.lam = m->field(MF_LAM);
    I.rho = m->field(MF_RHO);
    I.vp = m->field(MF_VP);
    I.vs = m->field(MF_VS);
    I.gmuss = m->field(MF_GMUSS);
    I.glamss = m->field(MF_GLAMSS);
    if (p.L > 0) {
        I.c_muipjp = m->field(MF_CMUIPJP);
        I.c_tausipjp = m->field(MF_CTAUSIPJP);
        I.c_mu = m->field(MF_CMU);
        I.c_taus = m->field(MF_CTAUS);
        I.c_pi = m->field(MF_CPI);
        I.c_taup = m->field(MF_CTAUP);
        for (int l = 0; l < p.L; l++) {
            I.eta[l] = m->eta[l];
            I.bip[l] = m->bip[l];
            I.cip[l] = m->cip[l];
            I.s_bjm[l] = m->s_bjm[l];
        }
        if (m->dsurf) {
            I.s_mu = m->dsurf;
            I.s_pi = m->dsurf + p.nx;
            I.s_taus = m->dsurf + 2 * p.nx;
            I.s_taup = m->dsurf + 3 * p.nx;
        }
    }
    const size_t w = 2 * (size_t)std::max(p.fw, 1);
    I.K_x = m->dpml + 0 * w;
    I.a_x = m->dpml + 1 * w;
    I.b_x = m->dpml + 2 * w;
    I.K_xh = m->dpml + 3 * w;
    I.a_xh = m->dpml + 4 * w;
    I.b_xh = m->dpml + 5 * w;
    I.K_y = m->dpml + 6 * w;
    I.a_y = m->dpml + 7 * w;
    I.b_y = m->dpml + 8 * w;
    I.K_yh = m->dpml + 9 * w;
    I.a_yh = m->dpml + 10 * w;
    I.b_yh = m->dpml + 11 * w;
    I.psi_sxx_x = s->psi[0];
    I.psi_sxy_x = s->psi[1];
    I.psi_vxx = s->psi[2];
    I.psi_vyx = s->psi[3];
    I.psi_vxxs = s->psi[4];
    I.psi_syy_y = s->psi[5];
    I.psi_sxy_y = s->psi[6];
    I.psi_vyy = s->psi[7];
    I.psi_vxy = s->psi[8];
    I.nsrc_cells = s->nsrc_cells;
    I.src_cell_i = s->d_cell_i;
    I.src_cell_j = s->d_cell_j;
    I.src_cell_start = s->d_cell_start;
    I.src_cell_count = s->d_cell_count;
    I.src_perm = s->d_perm;
    I.src_type = s->d_src_type;
    I.src_nsin = s->d_nsin;
    I.src_cos = s->d_cos;
    I.signals = s->d_signals;
    I.quelltyp_last = s->quelltyp_last;
    I.nsrc = s->nsrc;
    I.quelltypb = p.quelltypb;
    const size_t rs = (size_t)std::max(s->ntr, 1) * p.nt;
    I.res_vx = s->d_res;
    I.res_vy = s->d_res + rs;
    I.res_p = s->d_res + 2 * rs;
    I.ntr = s->ntr;
    I.rec_dup = s->rec_dup;
    I.rec_i = s->d_rec_i;
    I.rec_j = s->d_rec_j;
    I.sec = s->d_sec;
    I.snap = s->d_snap;
    I.snap_scale = s->d_snap_scale;
    I.wc = acc_ptr(s, 0);
    I.wcu = acc_ptr(s, 1);
    I.wcrho = acc_ptr(s, 2);
    I.Ws = (float *)acc_ptr(s, 3);
    I.Wr = (float *)acc_ptr(s, 4);
    I.flag = s->d_flag;
    if (c && c->fuse_src && mode != 1 && !runs_fused(s, mode)) {
        I.fsrc_v = 1;
        I.fsrc_s = s->quelltyp_last == 1;
    }
    if (runs_fused(s, mode)) {
        const int R = p.fdorder / 2;
        I.pp = 1;
        I.f_w = fz_width(R);
        I.f_tiles_x = (p.nx + I.f_w - 1) / I.f_w;
        I.f_zc = s->fzc;
        I.f_tiles = I.f_tiles_x * ((p.ny + s->fzc - 1) / s->fzc);
        I.vx_b = s->fb[0];
        I.vy_b = s->fb[1];
        I.sxx_b = s->fb[2];
        I.syy_b = s->fb[3];
        I.sxy_b = s->fb[4];
        I.psi_sxx_x_b = s->fpsi[0];
        I.psi_sxy_x_b = s->fpsi[1];
        I.psi_syy_y_b = s->fpsi[2];
        I.psi_sxy_y_b = s->fpsi[3];
    }
    return I;
}

// ---------------------------------------------------------------------------
// kernel dispatch (per-order launch functions in dn_launch_impl.cuh)
// ---------------------------------------------------------------------------
template <bool X>
static int set_smem_attrs_X(int R)
{
    switch (R) {
    case 1: return set_smem_attrs_R<1, X>();
    case 2: return set_smem_attrs_R<2, X>();
    case 3: return set_smem_attrs_R<3, X>();
    case 4: return set_smem_attrs_R<4, X>();
    case 5: return set_smem_attrs_R<5, X>();
    default: return set_smem_attrs_R<6, X>();
    }
}

template <bool X>
static int set_vpipe_attr_X(int R)
{
    switch (R) {
    case 1: return set_vpipe_attr_R<1, X>();
    case 2: return set_vpipe_attr_R<2, X>();
    case 3: return set_vpipe_attr_R<3, X>();
    case 4: return set_vpipe_attr_R<4, X>();
    case 5: return set_vpipe_attr_R<5, X>();
    default: return set_vpipe_attr_R<6, X>();
    }
}

static int prepare_launch(const LaunchCfg &c)
{
    if (c.vpipe) {
        int e = c.exact ? set_vpipe_attr_X<true>(c.R) : set_vpipe_attr_X<false>(c.R);
        if (e) return dn_fail(DN_EDEVICE, "cudaFuncSetAttribute (dynamic shared memory) failed");
    }
    if (!c.tma) return DN_OK;
    int e = c.exact ? set_smem_attrs_X<true>(c.R) : set_smem_attrs_X<false>(c.R);
    if (e) return dn_fail(DN_EDEVICE, "cudaFuncSetAttribute (dynamic shared memory) failed");
    return DN_OK;
}

template <bool X>
static void launch_step_X(const LaunchCfg &c, cudaStream_t st, const Inst *d, const int *ntb, int off, long long &nl,
                          cudaEvent_t *marks)
{
    switch (c.R) {
    case 1: launch_step_R<1, X>(c, st, d, ntb, off, nl, marks); break;
    case 2: launch_step_R<2, X>(c, st, d, ntb, off, nl, marks); break;
    case 3: launch_step_R<3, X>(c, st, d, ntb, off, nl, marks); break;
    case 4: launch_step_R<4, X>(c, st, d, ntb, off, nl, marks); break;
    case 5: launch_step_R<5, X>(c, st, d, ntb, off, nl, marks); break;
    default: launch_step_R<6, X>(c, st, d, ntb, off, nl, marks); break;
    }
}

static void launch_step(const LaunchCfg &c, cudaStream_t st, const Inst *d, const int *ntb, int off, long long &nl,
                        cudaEvent_t *marks = nullptr)
{
    if (c.exact) launch_step_X<true>(c, st, d, ntb, off, nl, marks);
    else launch_step_X<false>(c, st, d, ntb, off, nl, marks);
}

__global__ void k_advance(int *ntb, int by) { *ntb += by; }

// ---------------------------------------------------------------------------
// batch runner
// ---------------------------------------------------------------------------
struct Batch {
    int device;
    std::vector<const dn_shot *> shots;
    int mode;
    Inst *d_insts = nullptr;
    std::vector<Inst> h_insts;
    cudaGraphExec_t exec = nullptr;
    int chunk = 0;
    long long launches_per_chunk = 0;
};
static std::mutex g_batch_mu;
static std::vector<Batch *> g_batches;   // small cache of captured graphs

static void batch_free(Batch *b)
{
    cudaSetDevice(b->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    dn_free(b->d_insts);
    delete b;
}

static void forget_shot(const dn_shot *s)
{
    std::lock_guard<std::mutex> lk(g_batch_mu);
    for (size_t k = 0; k < g_batches.size();) {
        Batch *b = g_batches[k];
        if (std::find(b->shots.begin(), b->shots.end(), s) != b->shots.end()) {
            batch_free(b);
            g_batches.erase(g_batches.begin() + k);
        } else {
            k++;
        }
    }
}

// modes: per-shot modes of a mixed batch (a run queue), or null: every shot runs `mode`
static int check_batch(dn_shot *const *shots, int n, int mode, LaunchCfg &c, const int *modes = nullptr)
{
    if (!shots || n < 1) return dn_fail(DN_EINVAL, "dn_run: empty batch");
    if (!modes && (mode < 0 || mode > 2)) return dn_fail(DN_EINVAL, "dn_run: bad mode %d", mode);
    const dn_params &p0 = shots[0]->p;
    c.R = p0.fdorder / 2;
    c.L = p0.L;
    c.exact = p0.arith == DN_ARITH_EXACT;
    c.bx = shots[0]->bx;
    // stencil kernels of the batch: the variant of its first shot (tile rules, measured by
    // the autotuner; results do not depend on it); environment overrides: DN_KERNEL=tma the
    // bulk-copy row pipeline of dn_kernels_tma.cuh, DN_PACK=0 the one-column kernels,
    // DN_VPIPE=1 / 0 the pipelined velocity kernel on / off
    const char *kern = getenv("DN_KERNEL");
    c.tma = c.bx == TMA_W && kern && strcmp(kern, "tma") == 0;
    const char *pk = getenv("DN_PACK");
    c.pack = !c.tma && shots[0]->kern != DN_KERN_COLUMN;
    if (pk) c.pack = !c.tma && strcmp(pk, "0") != 0;
    c.any_surf = c.any_src_s = c.any_store = c.any_adj = c.any_rec = false;
    c.any_fused = c.any_plain = false;
    int maxtiles = 0, maxsrc = 1, maxnx = 1, maxtr = 1, maxft = 1;
    {
        long long cells = 0;
        for (int k = 0; k < n; k++)
            if (shots[k]) cells += (long long)shots[k]->p.nx * shots[k]->p.ny;
        c.auto_zch = c.tma ? 0 : batch_rows(cells, p0.L);   // the row pipeline keeps its measured tiles
    }
    for (int k = 0; k < n; k++) {
        const dn_shot *s = shots[k];
        if (!s) return dn_fail(DN_EINVAL, "dn_run: null shot %d", k);
        const int m = modes ? modes[k] : mode;
        if (m < 0 || m > 2) return dn_fail(DN_EINVAL, "dn_run: bad mode %d", m);
        if (s->m->device != shots[0]->m->device) return dn_fail(DN_EINVAL, "dn_run: shots on different devices");
        if (s->p.fdorder != p0.fdorder || s->p.L != p0.L)
            return dn_fail(DN_EINVAL, "dn_run: a batch must share FDORDER and L (shot %d differs)", k);
        if (s->p.arith != p0.arith || s->bx != c.bx) return dn_fail(DN_EINVAL, "dn_run: mixed arithmetic/tile width");
        if (m == 1) {
            if (!s->stored) return dn_fail(DN_ESTATE, "dn_run: adjoint run of shot %d without a stored forward run", k);
            for (int l = 0; l < s->nsrc; l++)
                if (s->src_type[l] == 5)
                    return dn_fail(DN_ENOTSUP, "moment-tensor sources are not supported in the adjoint pass");
        }
        maxtiles = std::max(maxtiles, eff_tiles(s, &c));
        if (runs_fused(s, m)) {
            c.any_fused = true;
            const int fwd = fz_width(s->p.fdorder / 2);
            maxft = std::max(maxft, ((s->p.nx + fwd - 1) / fwd) * ((s->p.ny + s->fzc - 1) / s->fzc));
        } else {
            c.any_plain = true;
        }
        maxsrc = std::max(maxsrc, std::max(s->nsrc_cells, m == 1 ? s->ntr : 0));
        maxnx = std::max(maxnx, s->p.nx);
        maxtr = std::max(maxtr, s->ntr);
        if (s->p.free_surf) c.any_surf = true;
        if (m == 1 ? s->p.quelltypb >= 4 : (s->quelltyp_last == 1 || s->quelltyp_last == 5)) c.any_src_s = true;
        if (m == 0 && s->p.store_snapshots && s->nsnap > 0) c.any_store = true;
        if (m == 1) c.any_adj = true;
    }
    c.tile_grid = dim3(maxtiles, n);
    c.fgrid = dim3(maxft, n);
    // pipelined velocity kernel (DN_VPIPE=1): strips of VP_W columns, about four CTAs per
    // resident slot (148 SMs x 3) over the batch, at least 32 rows tall (DN_VPIPE_ROWS sets it)
    const char *vp = getenv("DN_VPIPE");
    c.vpipe = !c.tma && shots[0]->kern == DN_KERN_VPIPE;
    if (vp) c.vpipe = !c.tma && strcmp(vp, "1") == 0;
    c.vsh = 0;
    c.vgrid = dim3(1, n);
    if (c.vpipe) {
        int sum_tx = 0, maxny = 1;
        for (int k = 0; k < n; k++) {
            sum_tx += (shots[k]->p.nx + VP_W - 1) / VP_W;
            maxny = std::max(maxny, shots[k]->p.ny);
        }
        const int strips = std::max(1, (4 * 148 * 3 + sum_tx - 1) / sum_tx);
        c.vsh = std::max(32, (maxny + strips - 1) / strips);
        const char *vr = getenv("DN_VPIPE_ROWS");
        if (vr && atoi(vr) > 0) c.vsh = atoi(vr);
        int maxc = 1;
        for (int k = 0; k < n; k++)
            maxc = std::max(maxc, ((shots[k]->p.nx + VP_W - 1) / VP_W) * ((shots[k]->p.ny + c.vsh - 1) / c.vsh));
        c.vgrid = dim3(maxc, n);
    }
    // forward sources inside the paired velocity kernel and the stress kernels (their SRC
    // variants), for batches whose step is bound by launches (below 5 M cells: a 600 x 300
    // shot steps in 20.4 instead of 24.0 us; the 64-shot batches were 3 % slower with the
    // sources in the kernels) and whose shots have at most SRC_IN_KERNEL source cells each;
    // DN_SRC_IN_KERNEL=0 / 1 turns them off / on for every batch
    {
        const char *fs = getenv("DN_SRC_IN_KERNEL");
        long long cells = 0;
        for (int k = 0; k < n; k++) cells += (long long)shots[k]->p.nx * shots[k]->p.ny;
        c.fuse_src = c.pack && !c.tma && !c.vpipe && (fs ? strcmp(fs, "0") != 0 : cells < 5000000);
        for (int k = 0; k < n; k++)
            if (shots[k]->nsrc_cells > SRC_IN_KERNEL) c.fuse_src = false;
        c.need_inject_v = false;
        c.any_src_s = false;
        for (int k = 0; k < n; k++) {
            const dn_shot *s = shots[k];
            const int m = modes ? modes[k] : mode;
            if (runs_fused(s, m)) continue;   // the fused step injects its own sources
            if (m == 1) {
                c.need_inject_v = true;
                if (s->p.quelltypb >= 4) c.any_src_s = true;
            } else {
                if (!c.fuse_src) c.need_inject_v = true;
                if (s->quelltyp_last == 5 || (s->quelltyp_last == 1 && !c.fuse_src)) c.any_src_s = true;
            }
        }
    }
    c.src_grid = dim3((maxsrc + 127) / 128, n);
    c.surf_grid = dim3((maxnx + 127) / 128, n);
    c.rec_grid = dim3((maxtr + 127) / 128, n);
    return DN_OK;
}

static int zero_for_run(dn_shot *s, int mode, cudaStream_t st)
{
    CU(cudaMemsetAsync(s->dstate, 0, s->state_bytes, st));   // zero_denise_*_PSV
    CU(cudaMemsetAsync(s->d_flag, 0, 4, st));
    if (mode == 0 && s->p.store_snapshots) {
        // init_grad of the per-shot accumulators and Ws/Wr (grad_obj_psv.c:61-70)
        const size_t ncell = (size_t)s->p.nx * s->p.ny;
        CU(cudaMemsetAsync(s->d_acc, 0, carve_size(ncell, s->acc64 ? 8 : 4) * 3 + carve_size(ncell, 4) * 2, st));
    }
    return DN_OK;
}

static int finish_run(dn_shot *const *shots, int n, int mode, cudaStream_t st)
{
    CU(cudaStreamSynchronize(st));
    CU(cudaGetLastError());
    int bad = -1;
    for (int k = 0; k < n; k++) {
        int f = 0;
        CU(cudaMemcpy(&f, shots[k]->d_flag, 4, cudaMemcpyDeviceToHost));
        if (f & 2) return dn_fail(DN_ETIMEDOUT, "a pipelined stencil kernel gave up waiting for its row copies (shot %d)", k);
        if (f & 1) bad = k;
        if (mode == 0 && shots[k]->p.store_snapshots) shots[k]->stored = 1;
        if (mode == 1) shots[k]->correlated = 1;
    }
    if (bad >= 0) return dn_fail(DN_EUNSTABLE, " Simulation is unstable ! (NaN in shot %d of the batch)", bad);
    return DN_OK;
}

static int graph_chunk(int maxnt)
{
    const char *ev = getenv("DN_GRAPH_CHUNK");
    int k = ev ? atoi(ev) : 50;
    if (k < 1) k = 1;
    return std::min(k, maxnt);
}

// ---------------------------------------------------------------------------
// checkpointed adjoint (ckpt_steps > 0)
//
// Forward (mode 0): the full state (fields, memory variables, CPML memory) is
// copied aside at the start of every segment of ckpt_steps steps; no snapshot
// is kept.  Adjoint (mode 1): for the segments from last to first, the forward
// state is restored from the segment's checkpoint and the segment is recomputed
// with its snapshots stored (slots relative to the segment), then the adjoint
// steps whose mirrored forward steps lie in the segment run, in their own state.
// The adjoint steps still run in increasing order and the recomputed forward
// states are bit-identical, so the gradient equals the one with every snapshot
// stored.  Direct launches: the grids that need checkpoints are large.
// ---------------------------------------------------------------------------
static Inst make_inst_state2(const dn_shot *s, int mode, const LaunchCfg *c)
{
    Inst I = make_inst(s, mode, c);
    const ptrdiff_t d = s->dstate2 - s->dstate;
    auto mv = [d](float *&p) {
        if (p) p = (float *)((char *)p + d);
    };
    mv(I.vx), mv(I.vy), mv(I.sxx), mv(I.syy), mv(I.sxy), mv(I.vxp1), mv(I.vyp1);
    mv(I.r), mv(I.p), mv(I.q);
    mv(I.psi_sxx_x), mv(I.psi_sxy_x), mv(I.psi_syy_y), mv(I.psi_sxy_y);
    mv(I.psi_vxx), mv(I.psi_vyx), mv(I.psi_vyy), mv(I.psi_vxy), mv(I.psi_vxxs);
    return I;
}

// Checkpointed shots (params.ckpt_steps > 0) of one batch: they share NT, DTINV and
// the segment length, so the segments line up and every launch covers all of them.
// Forward (mode 0/2): before each segment every shot's full state is copied to its
// checkpoint slot, then the segment's steps run for the whole batch.  Adjoint: the
// segments from last to first; per segment every shot's state is restored from its
// checkpoint, the segment is recomputed for the batch with its snapshots into the
// one-segment buffers, and the adjoint steps that correlate with it run for the batch.
static int run_ckpt(dn_shot *const *shots, int n, int mode, double &ms_total, long long &nl)
{
    LaunchCfg c, cf;
    int st = check_batch(shots, n, mode, c);
    if (!st && mode == 1) st = check_batch(shots, n, 0, cf);
    if (st) return st;
    const dn_shot *s0 = shots[0];
    for (int k = 1; k < n; k++)
        if (shots[k]->p.nt != s0->p.nt || shots[k]->p.ckpt_steps != s0->p.ckpt_steps ||
            shots[k]->p.dtinv != s0->p.dtinv || shots[k]->nseg != s0->nseg || shots[k]->nsnap != s0->nsnap)
            return dn_fail(DN_EINVAL, "dn_run: checkpointed shots of one batch must share NT, DTINV and ckpt_steps");
    DevState *ds;
    st = dev_state(s0->m->device, &ds);
    if (st) return st;
    CU(cudaSetDevice(s0->m->device));
    st = prepare_launch(c);
    if (st) return st;
    const int Ls = s0->p.ckpt_steps, nt = s0->p.nt, nseg = s0->nseg, per = Ls / s0->p.dtinv;
    cudaStream_t sm = ds->stream;
    std::vector<Inst> h;
    if (mode != 1) {
        for (int k = 0; k < n; k++) {
            h.push_back(make_inst(shots[k], mode, &c));
            h.back().store = 0;
        }
    } else {
        // segment g: n recompute instances, then n adjoint instances
        for (int g = 0; g < nseg; g++) {
            for (int k = 0; k < n; k++) {
                Inst f = make_inst(shots[k], 0, &cf);
                f.snap_base = g * per;
                f.nsnap = shots[k]->nsnap;   // the segment buffer's slots (fewer than per when NT < ckpt_steps)
                h.push_back(f);
            }
            for (int k = 0; k < n; k++) {
                Inst a = make_inst_state2(shots[k], 1, &c);
                a.snap_base = g * per;
                a.nsnap = shots[k]->nsnap;
                h.push_back(a);
            }
        }
    }
    Inst *d = nullptr;
    CU(dn_malloc(&d, sizeof(Inst) * h.size()));
    cudaError_t e = cudaMemcpyAsync(d, h.data(), sizeof(Inst) * h.size(), cudaMemcpyHostToDevice, sm);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sm);
    if (e != cudaSuccess) {
        dn_free(d);
        return dn_fail(DN_EDEVICE, "checkpointed run: %s", cudaGetErrorString(e));
    }
    for (int k = 0; k < n && !st; k++) {
        dn_shot *s = shots[k];
        if (mode != 1) {
            st = zero_for_run(s, mode, sm);
        } else if (cudaMemsetAsync(s->dstate2, 0, s->state_bytes, sm) != cudaSuccess ||
                   cudaMemsetAsync(s->d_flag, 0, 4, sm) != cudaSuccess) {
            st = dn_fail(DN_EDEVICE, "checkpointed adjoint: state reset failed");
        }
    }
    if (st) {
        dn_free(d);
        return st;
    }
    cudaEventRecord(ds->ev0, sm);
    if (mode != 1) {
        for (int g = 0; g < nseg; g++) {
            if (mode == 0)
                for (int k = 0; k < n; k++)
                    cudaMemcpyAsync(shots[k]->dckpt + shots[k]->state_bytes * g, shots[k]->dstate,
                                    shots[k]->state_bytes, cudaMemcpyDeviceToDevice, sm);
            for (int t = g * Ls + 1; t <= std::min((g + 1) * Ls, nt); t++) launch_step(c, sm, d, ds->d_zero, t, nl);
        }
    } else {
        for (int g = nseg - 1; g >= 0; g--) {
            const int a = g * Ls + 1, b = std::min((g + 1) * Ls, nt);
            for (int k = 0; k < n; k++)
                cudaMemcpyAsync(shots[k]->dstate, shots[k]->dckpt + shots[k]->state_bytes * g, shots[k]->state_bytes,
                                cudaMemcpyDeviceToDevice, sm);
            for (int t = a; t <= b; t++) launch_step(cf, sm, d + (size_t)2 * n * g, ds->d_zero, t, nl);
            for (int t = nt - b + 1; t <= nt - a + 1; t++)
                launch_step(c, sm, d + (size_t)2 * n * g + n, ds->d_zero, t, nl);
        }
    }
    cudaEventRecord(ds->ev1, sm);
    cudaError_t le = cudaGetLastError();
    st = finish_run(shots, n, mode, sm);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ds->ev0, ds->ev1);
    ms_total += ms;
    dn_free(d);
    if (le != cudaSuccess) return dn_fail(DN_EDEVICE, "kernel launch failed: %s", cudaGetErrorString(le));
    return st;
}

extern "C" int dn_run(dn_shot *const *shots, int n, int mode)
{
    DnRange range(mode == 0 ? "dn_run forward" : mode == 1 ? "dn_run adjoint" : "dn_run objective");
    if (shots && n > 0 && shots[0] && shots[0]->nseg > 0) {
        // checkpointed shots run as one batch
        double ms = 0.0;
        long long nl = 0;
        for (int k = 0; k < n; k++)
            if (!shots[k] || shots[k]->nseg == 0)
                return dn_fail(DN_EINVAL, "dn_run: checkpointed and stored-snapshot shots cannot share a batch");
        int st = run_ckpt(shots, n, mode, ms, nl);
        if (st) return st;
        g_last_ms = ms;
        g_last_launches = nl;
        return DN_OK;
    }
    LaunchCfg c;
    int st = check_batch(shots, n, mode, c);
    if (st) return st;
    for (int k = 0; k < n; k++)
        if (shots[k]->nseg > 0) return dn_fail(DN_EINVAL, "dn_run: checkpointed and stored-snapshot shots cannot share a batch");
    const int device = shots[0]->m->device;
    DevState *ds;
    st = dev_state(device, &ds);
    if (st) return st;
    CU(cudaSetDevice(device));
    st = prepare_launch(c);
    if (st) return st;
    int maxnt = 0;
    for (int k = 0; k < n; k++) maxnt = std::max(maxnt, shots[k]->p.nt);

    // find or build the captured batch
    Batch *b = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_batch_mu);
        for (Batch *x : g_batches) {
            if (x->mode == mode && x->device == device && (int)x->shots.size() == n &&
                std::equal(x->shots.begin(), x->shots.end(), shots)) {
                b = x;
                break;
            }
        }
    }
    if (!b) {
        b = new Batch();
        b->device = device;
        b->mode = mode;
        b->shots.assign(shots, shots + n);
        for (int k = 0; k < n; k++) b->h_insts.push_back(make_inst(shots[k], mode, &c));
        if (dn_malloc(&b->d_insts, sizeof(Inst) * n) != cudaSuccess) {
            delete b;
            return dn_fail(DN_ENOMEM, "dn_run: descriptor allocation failed");
        }
        CU(cudaMemcpyAsync(b->d_insts, b->h_insts.data(), sizeof(Inst) * n, cudaMemcpyHostToDevice, ds->stream));
        CU(cudaStreamSynchronize(ds->stream));
        b->chunk = graph_chunk(maxnt);
        cudaGraph_t g;
        CU(cudaStreamBeginCapture(ds->stream, cudaStreamCaptureModeThreadLocal));
        long long nl = 0;
        for (int k = 0; k < b->chunk; k++) launch_step(c, ds->stream, b->d_insts, ds->d_step, k + 1, nl);
        k_advance<<<1, 1, 0, ds->stream>>>(ds->d_step, b->chunk);
        nl++;
        cudaError_t e = cudaStreamEndCapture(ds->stream, &g);
        if (e != cudaSuccess) {
            batch_free(b);
            return dn_fail(DN_EDEVICE, "graph capture failed: %s", cudaGetErrorString(e));
        }
        e = cudaGraphInstantiate(&b->exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            b->exec = nullptr;
            batch_free(b);
            return dn_fail(DN_EDEVICE, "graph instantiate failed: %s", cudaGetErrorString(e));
        }
        b->launches_per_chunk = nl;
        std::lock_guard<std::mutex> lk(g_batch_mu);
        if (g_batches.size() >= 8) {
            batch_free(g_batches.front());
            g_batches.erase(g_batches.begin());
        }
        g_batches.push_back(b);
    }
    for (int k = 0; k < n; k++) {
        st = zero_for_run(shots[k], mode, ds->stream);
        if (st) return st;
    }
    CU(cudaMemsetAsync(ds->d_step, 0, sizeof(int), ds->stream));
    const int nchunks = (maxnt + b->chunk - 1) / b->chunk;
    CU(cudaEventRecord(ds->ev0, ds->stream));
    for (int k = 0; k < nchunks; k++) CU(cudaGraphLaunch(b->exec, ds->stream));
    CU(cudaEventRecord(ds->ev1, ds->stream));
    st = finish_run(shots, n, mode, ds->stream);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ds->ev0, ds->ev1);
    g_last_ms = ms;
    g_last_launches = b->launches_per_chunk * nchunks;
    return st;
}

static int run_direct(dn_shot *s, int mode, int nt0, int nt1, bool zero)
{
    LaunchCfg c;
    dn_shot *arr[1] = {s};
    int st = check_batch(arr, 1, mode, c);
    if (st) return st;
    DevState *ds;
    st = dev_state(s->m->device, &ds);
    if (st) return st;
    CU(cudaSetDevice(s->m->device));
    st = prepare_launch(c);
    if (st) return st;
    Inst h = make_inst(s, mode, &c);
    if (h.pp && (nt0 != 1 || nt1 != s->p.nt)) {
        // a partial range runs the separate kernels on the primary buffers, so that the state
        // between calls stays where dn_shot_get_field and the next range read it
        h.pp = 0;
        c.any_fused = false;
        c.any_plain = true;
        if (c.fuse_src && mode != 1) {   // its sources then come from the stencil kernels
            h.fsrc_v = 1;
            h.fsrc_s = s->quelltyp_last == 1;
        } else {
            c.need_inject_v = true;
            if (s->quelltyp_last == 1) c.any_src_s = true;
        }
    }
    Inst *d = nullptr;
    CU(dn_malloc(&d, sizeof(Inst)));
    CU(cudaMemcpyAsync(d, &h, sizeof(Inst), cudaMemcpyHostToDevice, ds->stream));
    CU(cudaStreamSynchronize(ds->stream));
    if (zero) {
        st = zero_for_run(s, mode, ds->stream);
        if (st) {
            dn_free(d);
            return st;
        }
    }
    long long nl = 0;
    cudaEventRecord(ds->ev0, ds->stream);
    for (int nt = nt0; nt <= nt1; nt++) launch_step(c, ds->stream, d, ds->d_zero, nt, nl);
    cudaEventRecord(ds->ev1, ds->stream);
    cudaError_t le = cudaGetLastError();
    st = finish_run(arr, 1, mode, ds->stream);
    if (nt1 < s->p.nt) {
        if (mode == 0 && s->p.store_snapshots) s->stored = 0;
        if (mode == 1) s->correlated = 0;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ds->ev0, ds->ev1);
    g_last_ms = ms;
    g_last_launches = nl;
    dn_free(d);
    if (le != cudaSuccess) return dn_fail(DN_EDEVICE, "kernel launch failed: %s", cudaGetErrorString(le));
    return st;
}

extern "C" int dn_run_plain(dn_shot *s, int mode)
{
    if (!s) return dn_fail(DN_EINVAL, "null shot");
    if (s->nseg > 0) return dn_run(&s, 1, mode);
    return run_direct(s, mode, 1, s->p.nt, true);
}

extern "C" int dn_run_steps(dn_shot *s, int mode, int nt0, int nt1)
{
    if (!s) return dn_fail(DN_EINVAL, "null shot");
    if (nt0 < 1 || nt1 > s->p.nt || nt0 > nt1) return dn_fail(DN_EINVAL, "bad step range %d..%d", nt0, nt1);
    if (s->nseg > 0) return dn_fail(DN_ENOTSUP, "dn_run_steps: not for checkpointed shots");
    return run_direct(s, mode, nt0, nt1, nt0 == 1);
}

extern "C" int dn_last_run_stats(double *ms, long long *launches)
{
    if (ms) *ms = g_last_ms;
    if (launches) *launches = g_last_launches;
    return DN_OK;
}

// ---------------------------------------------------------------------------
// run queues: continuous batching
//
// A queue runs shots that share FDORDER, L and arithmetic, each at its own
// time step: an instance that joined when the queue's step counter stood at t0
// computes step *ntb + off - t0.  Membership changes only between chunks of
// `chunk` time steps: dn_queue_step waits for the chunk in flight, retires the
// shots it finished, admits the shots added since, re-captures the chunk graph
// if the membership changed and enqueues the next chunk without waiting for
// it.  Each queue owns a stream, so chunks of different queues overlap.
// ---------------------------------------------------------------------------
struct QSlot {
    dn_shot *s;
    int mode;
    long long t0;
};

struct dn_queue {
    int device = 0, chunk = 50;
    cudaStream_t stream = nullptr;
    int *d_step = nullptr;
    // up to two chunks in flight: while the host retires, admits and re-captures, the
    // GPU runs the newer one; ev[head] marks the end of the older
    cudaEvent_t ev[2] = {nullptr, nullptr};
    long long ev_gstep[2] = {0, 0};
    int nflight = 0, head = 0;
    bool dirty = true;
    long long gstep = 0;                 // value of *d_step once the enqueued chunks have run
    long long gstep_done = 0;            // value of *d_step after the chunks known to have completed
    std::vector<QSlot> active, pending;
    std::vector<Inst> h_insts;
    Inst *d_insts = nullptr;
    int cap_insts = 0;
    // pinned staging of the descriptors, two buffers in turn: a pageable source could make the
    // asynchronous copy wait for the chunk in flight, and the copy enqueued by the previous call
    // may still be pending behind it
    Inst *h_pin[2] = {nullptr, nullptr};
    int pin_cap[2] = {0, 0};
    int pin_k = 0;
    cudaGraphExec_t exec = nullptr;
    long long launches_per_chunk = 0;
};

extern "C" int dn_queue_create(int device, int chunk, dn_queue **out)
{
    if (!out) return dn_fail(DN_EINVAL, "dn_queue_create: null out");
    *out = nullptr;
    if (chunk < 1 || chunk > 4096) return dn_fail(DN_EINVAL, "dn_queue_create: chunk %d outside 1..4096", chunk);
    CU(cudaSetDevice(device));
    dn_queue *q = new dn_queue();
    q->device = device;
    q->chunk = chunk;
    if (cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking) != cudaSuccess ||
        dn_malloc(&q->d_step, sizeof(int)) != cudaSuccess ||
        cudaEventCreateWithFlags(&q->ev[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&q->ev[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaMemset(q->d_step, 0, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        dn_queue_destroy(q);
        return dn_fail(DN_EDEVICE, "dn_queue_create: stream/counter set-up failed");
    }
    *out = q;
    return DN_OK;
}

extern "C" int dn_queue_destroy(dn_queue *q)
{
    if (!q) return DN_OK;
    cudaSetDevice(q->device);
    if (q->stream) cudaStreamSynchronize(q->stream);
    if (q->exec) cudaGraphExecDestroy(q->exec);
    for (int k = 0; k < 2; k++)
        if (q->h_pin[k]) cudaFreeHost(q->h_pin[k]);
    dn_free(q->d_insts);
    dn_free(q->d_step);
    for (int k = 0; k < 2; k++)
        if (q->ev[k]) cudaEventDestroy(q->ev[k]);
    if (q->stream) cudaStreamDestroy(q->stream);
    delete q;
    return DN_OK;
}

extern "C" int dn_queue_add(dn_queue *q, dn_shot *s, int mode)
{
    if (!q || !s) return dn_fail(DN_EINVAL, "dn_queue_add: null argument");
    if (mode < 0 || mode > 2) return dn_fail(DN_EINVAL, "dn_queue_add: bad mode %d", mode);
    if (s->m->device != q->device) return dn_fail(DN_EINVAL, "dn_queue_add: shot on device %d, queue on %d",
                                                  s->m->device, q->device);
    const dn_shot *ref = !q->active.empty() ? q->active[0].s : !q->pending.empty() ? q->pending[0].s : nullptr;
    if (ref && (ref->p.fdorder != s->p.fdorder || ref->p.L != s->p.L || ref->p.arith != s->p.arith ||
                ref->bx != s->bx))
        return dn_fail(DN_EINVAL, "dn_queue_add: a queue runs one FDORDER, L and arithmetic");
    for (const QSlot &x : q->active)
        if (x.s == s) return dn_fail(DN_ESTATE, "dn_queue_add: shot already running in this queue");
    for (const QSlot &x : q->pending)
        if (x.s == s) return dn_fail(DN_ESTATE, "dn_queue_add: shot already waiting in this queue");
    if (mode == 1 && !s->stored) return dn_fail(DN_ESTATE, "dn_queue_add: adjoint run without a stored forward run");
    if (s->nseg > 0) return dn_fail(DN_ENOTSUP, "dn_queue_add: checkpointed shots run through dn_run");
    q->pending.push_back({s, mode, 0});
    return DN_OK;
}

extern "C" int dn_queue_count(const dn_queue *q, int *running, int *waiting)
{
    if (!q) return dn_fail(DN_EINVAL, "dn_queue_count: null queue");
    if (running) *running = (int)q->active.size();
    if (waiting) *waiting = (int)q->pending.size();
    return DN_OK;
}

static int queue_capture(dn_queue *q)
{
    const int n = (int)q->active.size();
    std::vector<dn_shot *> shots(n);
    std::vector<int> modes(n);
    q->h_insts.clear();
    for (int k = 0; k < n; k++) {
        shots[k] = q->active[k].s;
        modes[k] = q->active[k].mode;
    }
    LaunchCfg c;
    int st = check_batch(shots.data(), n, 0, c, modes.data());
    if (st) return st;
    for (int k = 0; k < n; k++) {
        Inst I = make_inst(shots[k], modes[k], &c);
        I.t0 = (int)q->active[k].t0;
        q->h_insts.push_back(I);
    }
    st = prepare_launch(c);
    if (st) return st;
    if (n > q->cap_insts) {
        dn_free(q->d_insts);
        q->d_insts = nullptr;
        q->cap_insts = 0;
        if (dn_malloc(&q->d_insts, sizeof(Inst) * n) != cudaSuccess)
            return dn_fail(DN_ENOMEM, "dn_queue_step: descriptor allocation failed");
        q->cap_insts = n;
    }
    q->pin_k ^= 1;
    const int pk = q->pin_k;
    if (n > q->pin_cap[pk]) {
        if (q->h_pin[pk]) cudaFreeHost(q->h_pin[pk]);
        q->h_pin[pk] = nullptr;
        q->pin_cap[pk] = 0;
        if (cudaMallocHost(&q->h_pin[pk], sizeof(Inst) * n) != cudaSuccess) {
            cudaGetLastError();
            q->h_pin[pk] = nullptr;
            return dn_fail(DN_ENOMEM, "dn_queue_step: pinned descriptor allocation failed");
        }
        q->pin_cap[pk] = n;
    }
    memcpy(q->h_pin[pk], q->h_insts.data(), sizeof(Inst) * n);
    CU(cudaMemcpyAsync(q->d_insts, q->h_pin[pk], sizeof(Inst) * n, cudaMemcpyHostToDevice, q->stream));
    if (q->exec) {
        cudaGraphExecDestroy(q->exec);
        q->exec = nullptr;
    }
    cudaGraph_t g;
    CU(cudaStreamBeginCapture(q->stream, cudaStreamCaptureModeThreadLocal));
    long long nl = 0;
    for (int k = 0; k < q->chunk; k++) launch_step(c, q->stream, q->d_insts, q->d_step, k + 1, nl);
    k_advance<<<1, 1, 0, q->stream>>>(q->d_step, q->chunk);
    nl++;
    cudaError_t e = cudaStreamEndCapture(q->stream, &g);
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "queue graph capture failed: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&q->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        q->exec = nullptr;
        return dn_fail(DN_EDEVICE, "queue graph instantiate failed: %s", cudaGetErrorString(e));
    }
    q->launches_per_chunk = nl;
    q->dirty = false;
    return DN_OK;
}

extern "C" int dn_queue_step(dn_queue *q, dn_shot **done, int *status, int cap, int *ndone)
{
    if (!q || !ndone || (cap > 0 && (!done || !status))) return dn_fail(DN_EINVAL, "dn_queue_step: bad arguments");
    *ndone = 0;
    CU(cudaSetDevice(q->device));
    // wait for the older of two chunks in flight; take the newer too if it has finished
    if (q->nflight == 2) {
        CU(cudaEventSynchronize(q->ev[q->head]));
        q->gstep_done = q->ev_gstep[q->head];
        q->head ^= 1;
        q->nflight = 1;
        CU(cudaGetLastError());
    }
    if (q->nflight == 1) {
        const cudaError_t r = cudaEventQuery(q->ev[q->head]);
        if (r == cudaSuccess) {
            q->gstep_done = q->ev_gstep[q->head];
            q->head ^= 1;
            q->nflight = 0;
        } else if (r != cudaErrorNotReady) {
            return dn_fail(DN_EDEVICE, "dn_queue_step: %s", cudaGetErrorString(r));
        }
        cudaGetLastError();   // a chunk still running is not an error
    }
    // retire the shots whose last step has run in a completed chunk (as many as `done` holds);
    // their descriptors stay in the chunk in flight, where every kernel skips them (step > NT)
    for (size_t k = 0; k < q->active.size() && *ndone < cap;) {
        QSlot &x = q->active[k];
        if (x.t0 + x.s->p.nt > q->gstep_done) {
            k++;
            continue;
        }
        int f = 0;
        CU(cudaMemcpy(&f, x.s->d_flag, 4, cudaMemcpyDeviceToHost));
        int st = DN_OK;
        if (f & 2) st = DN_ETIMEDOUT;
        else if (f & 1) st = DN_EUNSTABLE;
        if (x.mode == 0 && x.s->p.store_snapshots) x.s->stored = st == DN_OK;
        if (x.mode == 1) x.s->correlated = st == DN_OK;
        done[*ndone] = x.s;
        status[*ndone] = st;
        (*ndone)++;
        q->active.erase(q->active.begin() + k);
        q->dirty = true;
    }
    // admit the shots added since the last chunk: their step 1 is the next one
    for (QSlot &x : q->pending) {
        int st = zero_for_run(x.s, x.mode, q->stream);
        if (st) return st;
        x.t0 = q->gstep;
        q->active.push_back(x);
        q->dirty = true;
    }
    q->pending.clear();
    if (q->active.empty()) return DN_OK;
    if (q->gstep + q->chunk > INT32_MAX - 1) return dn_fail(DN_ENOTSUP, "dn_queue_step: step counter range exhausted");
    if (q->dirty) {
        int st = queue_capture(q);
        if (st) return st;
    }
    CU(cudaGraphLaunch(q->exec, q->stream));
    const int slot = (q->head + q->nflight) & 1;
    CU(cudaEventRecord(q->ev[slot], q->stream));
    q->gstep += q->chunk;
    q->ev_gstep[slot] = q->gstep;
    q->nflight++;
    return DN_OK;
}

// ---------------------------------------------------------------------------
// results
// ---------------------------------------------------------------------------
struct SecScratch {
    float *d = nullptr, *h = nullptr;   // device and pinned host buffers of n floats
    size_t n = 0;
};
static std::mutex g_sec_mu;
static std::map<int, SecScratch> g_sec_scratch;

// [nt][ntr] (the order the receiver kernel writes) to [ntr][nt] (trace order), 32 x 32 tiles
__global__ void k_sec_transpose(const float *__restrict__ in, float *__restrict__ out, int nt, int ntr)
{
    __shared__ float tile[32][33];
    const int r0 = blockIdx.x * 32, t0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int t = t0 + k, r = r0 + threadIdx.x;
        if (t < nt && r < ntr) tile[k][threadIdx.x] = in[(size_t)t * ntr + r];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, t = t0 + threadIdx.x;
        if (r < ntr && t < nt) out[(size_t)r * nt + t] = tile[threadIdx.x][k];
    }
}

extern "C" int dn_shot_get_sections(const dn_shot *s, int comp, float *out)
{
    if (!s || !out) return dn_fail(DN_EINVAL, "null argument");
    if (comp < 0 || comp > 4) return dn_fail(DN_EINVAL, "bad section component %d", comp);
    const int nt = s->p.nt, ntr = s->ntr;
    if (ntr == 0) return DN_OK;
    const int device = s->m->device;
    CU(cudaSetDevice(device));
    // transposed on the device into a per-device scratch buffer (kept between calls: a
    // release would wait for the whole device, run queues in flight included), then one
    // contiguous copy; the legacy default stream orders both after the runs, which end
    // with a stream synchronisation, and does not wait for the library's other streams
    const size_t n = (size_t)nt * ntr;
    std::lock_guard<std::mutex> lk(g_sec_mu);
    SecScratch &sc = g_sec_scratch[device];
    if (sc.n < n) {
        // grown, never shrunk: one transposed section on the device and its pinned host copy
        if (sc.d) cudaFree(sc.d);
        if (sc.h) cudaFreeHost(sc.h);
        sc = SecScratch();
        if (cudaMalloc(&sc.d, n * 4) != cudaSuccess || cudaMallocHost(&sc.h, n * 4) != cudaSuccess) {
            cudaGetLastError();
            if (sc.d) cudaFree(sc.d);
            sc = SecScratch();
            return dn_fail(DN_ENOMEM, "dn_shot_get_sections: scratch allocation failed");
        }
        sc.n = n;
    }
    k_sec_transpose<<<dim3((ntr + 31) / 32, (nt + 31) / 32), dim3(32, 8)>>>(s->d_sec + (size_t)comp * n, sc.d, nt, ntr);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(sc.h, sc.d, n * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "dn_shot_get_sections: %s", cudaGetErrorString(e));
    memcpy(out, sc.h, n * 4);
    return DN_OK;
}

extern "C" int dn_shot_set_residuals(dn_shot *s, const float *vxd, const float *vyd, const float *pd)
{
    if (!s) return dn_fail(DN_EINVAL, "null shot");
    CU(cudaSetDevice(s->m->device));
    const size_t rs = (size_t)std::max(s->ntr, 1) * s->p.nt;
    const float *src[3] = {vxd, vyd, pd};
    for (int k = 0; k < 3; k++) {
        if (src[k] && s->ntr > 0) {
            CU(cudaMemcpy(s->d_res + k * rs, src[k], (size_t)s->ntr * s->p.nt * 4, cudaMemcpyHostToDevice));
            s->has_res[k] = 1;
        } else {
            CU(cudaMemset(s->d_res + k * rs, 0, rs * 4));
            s->has_res[k] = 0;
        }
    }
    return DN_OK;
}

extern "C" int dn_shot_get_field(const dn_shot *s, int field, float *out)
{
    if (!s || !out) return dn_fail(DN_EINVAL, "null argument");
    const dn_params &p = s->p;
    const Layout &L = s->m->lay;
    CU(cudaSetDevice(s->m->device));
    if (field >= 0 && field < 7) {
        std::vector<float> h(L.plane);
        CU(cudaMemcpy(h.data(), s->f[field] - L.origin, L.plane * 4, cudaMemcpyDeviceToHost));
        for (int i = 1; i <= p.nx; i++)
            for (int j = 1; j <= p.ny; j++)
                out[(size_t)(i - 1) * p.ny + (j - 1)] = h[L.origin + (long long)j * L.pitch + i];
        return DN_OK;
    }
    if (field >= 7 && field <= 11) {
        const size_t ncell = (size_t)p.nx * p.ny;
        const bool dbl = field <= 9 && s->acc64;
        std::vector<char> h(ncell * (dbl ? 8 : 4));
        CU(cudaMemcpy(h.data(), acc_ptr(s, field - 7), h.size(), cudaMemcpyDeviceToHost));
        for (int j = 1; j <= p.ny; j++)
            for (int i = 1; i <= p.nx; i++) {
                size_t w = (size_t)(j - 1) * p.nx + (i - 1);
                out[(size_t)(i - 1) * p.ny + (j - 1)] = dbl ? (float)((double *)h.data())[w] : ((float *)h.data())[w];
            }
        return DN_OK;
    }
    return dn_fail(DN_EINVAL, "bad field id %d", field);
}

extern "C" int dn_shot_get_snapshot(const dn_shot *s, int k, int field, float *out)
{
    if (!s || !out) return dn_fail(DN_EINVAL, "null argument");
    if (s->nseg > 0) return dn_fail(DN_ENOTSUP, "dn_shot_get_snapshot: a checkpointed shot keeps no snapshot set");
    if (k < 0 || k >= s->nsnap || field < 0 || field > 4) return dn_fail(DN_EINVAL, "bad snapshot index");
    const dn_params &p = s->p;
    const size_t tc = (size_t)s->bx * s->zch;
    const size_t eb = snap_elem_bytes(p.snap_precision);
    std::vector<char> h((size_t)s->tiles * tc * eb);
    std::vector<float> sc(s->tiles, 1.0f);
    CU(cudaSetDevice(s->m->device));
    const size_t slot0 = ((size_t)k * 5 + field) * s->tiles;
    CU(cudaMemcpy(h.data(), (char *)s->d_snap + slot0 * tc * eb, h.size(), cudaMemcpyDeviceToHost));
    if (p.snap_precision != DN_SNAP_F32)
        CU(cudaMemcpy(sc.data(), s->d_snap_scale + slot0, s->tiles * 4, cudaMemcpyDeviceToHost));
    for (int b = 0; b < s->tiles; b++) {
        int tx = b % s->tiles_x, tz = b / s->tiles_x;
        for (int r = 0; r < s->zch; r++)
            for (int c = 0; c < s->bx; c++) {
                int i = tx * s->bx + c + 1, j = tz * s->zch + r + 1;
                if (i > p.nx || j > p.ny) continue;
                size_t e = (size_t)b * tc + (size_t)r * s->bx + c;
                float v;
                if (p.snap_precision == DN_SNAP_F32) {
                    v = ((float *)h.data())[e];
                } else {
                    uint16_t bits = ((uint16_t *)h.data())[e];
                    if (p.snap_precision == DN_SNAP_F16) {
                        __half_raw hr;
                        hr.x = bits;
                        v = __half2float(__half(hr)) * sc[b];
                    } else {
                        uint32_t u = (uint32_t)bits << 16;
                        float f;
                        memcpy(&f, &u, 4);
                        v = f * sc[b];
                    }
                }
                out[(size_t)(i - 1) * p.ny + (j - 1)] = v;
            }
    }
    return DN_OK;
}

// ---------------------------------------------------------------------------
// gradient assembly: ass_gradPSV.c:29-150 (INVMAT1 1, GRAD_FORM 1) + stacking
// ---------------------------------------------------------------------------
// Energy weight of a shot (eprecond1.c): EPRECOND 1, We = sqrt(Ws Wr); EPRECOND 3,
// We = sqrt(Ws) (asinh((xmax - x) / y) - asinh((xmin - x) / y)) with x = i DH,
// y = j DH, xmin = DH, xmax = NX DH (the receiver Green's function approximation
// of Plessix and Mulder 2004); its maximum is kept as float bits (We >= 0, so
// the bit patterns order like the values).
__global__ void k_energy_weight(int nx, int ny, int ep, float dh, const float *Ws, const float *Wr, float *We,
                                unsigned *maxbits)
{
    const long long n = (long long)nx * ny;
    const float xmin = dh, xmax = __fmul_rn((float)nx, dh);
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n; w += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(w / nx) + 1, i = (int)(w % nx) + 1;
        float we;
        if (ep == 1) {
            we = (float)sqrt((double)__fmul_rn(Ws[w], Wr[w]));
        } else {
            const float x = __fmul_rn((float)i, dh), y = __fmul_rn((float)j, dh);
            const double a = asinh((double)__fdiv_rn(__fsub_rn(xmax, x), y));
            const double b = asinh((double)__fdiv_rn(__fsub_rn(xmin, x), y));
            we = (float)(sqrt((double)Ws[w]) * (a - b));
        }
        We[w] = we;
        atomicMax(maxbits, __float_as_uint(we));
    }
}

// We: energy weights (or null: no preconditioning); we_add = EPSILON_WE max(We);
// c: the C_vp, C_vs, C_rho of grad_obj_psv.c:230-236
// Per-shot circular taper of taper_grad_shot.c: coefficient (msum - minm) / maxm
// with msum = m inside the G x G box at grid column x0, row z0 and 1 elsewhere,
// then the cells of zc (0-based row-major, rows zr0..zr1) set to zero.
struct ShotTaperArgs {
    int on, G, x0, z0;
    const float *m;
    float minm, maxm;
    const int *zc;
    int nz, zr0, zr1;
};

__global__ void k_ass_grad(int nx, int ny, int pitch, const float *rho, const float *vp, const float *vs,
                           const float *gmuss, const float *glamss, const void *wc, const void *wcu, const void *wcr,
                           int acc64, float DT, void *gsum, int out64, const float *We, const unsigned *maxbits,
                           float cvp, float cvs, float crho, ShotTaperArgs tp)
{
    const long long n = (long long)nx * ny;
    for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n; w += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(w / nx) + 1, i = (int)(w % nx) + 1;
        const long long o = (long long)j * pitch + i;
        const float r = rho[o], pi = vp[o], u = vs[o], muss = gmuss[o], lamss = glamss[o];
        double gvp, gvs, grho;
        if (!acc64) {
            const float ws = ((const float *)wc)[w], wus = ((const float *)wcu)[w], wrs = ((const float *)wcr)[w];
            float lam = __fmul_rn(-DT, ws);
            if (muss > 0.0f || lamss > 0.0f) {
                const float lm = __fadd_rn(lamss, muss);
                lam = F(DMUL(DDIV(1.0, DMUL(DMUL(4.0, (double)lm), (double)lm)), (double)lam));
            }
            const float fvp = F(DMUL(DMUL(DMUL(2.0, (double)pi), (double)r), (double)lam));
            const float mu = __fmul_rn(-DT, wus);
            const float fvs = F(DADD(DMUL(DMUL(DMUL(-4.0, (double)r), (double)u), (double)lam),
                                     DMUL(DMUL(DMUL(2.0, (double)r), (double)u), (double)mu)));
            const float rs = __fmul_rn(-DT, wrs);
            const double a = DSUB((double)__fmul_rn(pi, pi), DMUL(DMUL(2.0, (double)u), (double)u));
            const float frho = F(DADD(DADD(DMUL(a, (double)lam), (double)__fmul_rn(__fmul_rn(u, u), mu)), (double)rs));
            gvp = fvp;
            gvs = fvs;
            grho = frho;
            if (We) {   // grad_obj_psv.c:230-236, float
                const float wr = __fadd_rn(We[w], __fmul_rn(0.005f, __uint_as_float(*maxbits)));
                gvp = __fdiv_rn(fvp, __fmul_rn(__fmul_rn(wr, cvp), cvp));
                gvs = cvs == 0.0f ? 0.0f : __fdiv_rn(fvs, __fmul_rn(__fmul_rn(wr, cvs), cvs));
                grho = __fdiv_rn(frho, __fmul_rn(__fmul_rn(wr, crho), crho));
            }
        } else {
            const double ws = ((const double *)wc)[w], wus = ((const double *)wcu)[w], wrs = ((const double *)wcr)[w];
            double lam = -(double)DT * ws;
            if (muss > 0.0f || lamss > 0.0f) {
                const double lm = (double)lamss + (double)muss;
                lam = lam / (4.0 * lm * lm);
            }
            gvp = 2.0 * (double)pi * (double)r * lam;
            const double mu = -(double)DT * wus;
            gvs = -4.0 * (double)r * (double)u * lam + 2.0 * (double)r * (double)u * mu;
            const double rs = -(double)DT * wrs;
            grho = ((double)pi * pi - 2.0 * (double)u * u) * lam + (double)u * u * mu + rs;
            if (We) {
                const double wr = (double)We[w] + 0.005 * (double)__uint_as_float(*maxbits);
                gvp /= wr * cvp * cvp;
                gvs = cvs == 0.0f ? 0.0 : gvs / (wr * cvs * cvs);
                grho /= wr * crho * crho;
            }
        }
        if (tp.on) {   // taper_grad_shot.c, applied to the three shot gradients alike
            const int bi = i - tp.x0, bj = j - tp.z0;
            const float b = (bi >= 0 && bi < tp.G && bj >= 0 && bj < tp.G) ? tp.m[bj * tp.G + bi] : 1.0f;
            const float c = __fdiv_rn(__fsub_rn(b, tp.minm), tp.maxm);
            if (!acc64) {
                gvp = __fmul_rn((float)gvp, c);
                gvs = __fmul_rn((float)gvs, c);
                grho = __fmul_rn((float)grho, c);
            } else {
                gvp *= c;
                gvs *= c;
                grho *= c;
            }
            if (j >= tp.zr0 && j <= tp.zr1)
                for (int k = 0; k < tp.nz; k++)
                    if (tp.zc[k] == (int)w) gvp = gvs = grho = 0.0;
        }
        if (out64) {
            double *g = (double *)gsum;
            g[w] += gvp;
            g[n + w] += gvs;
            g[2 * n + w] += grho;
        } else {
            float *g = (float *)gsum;
            g[w] = __fadd_rn(g[w], (float)gvp);
            g[n + w] = __fadd_rn(g[n + w], (float)gvs);
            g[2 * n + w] = __fadd_rn(g[2 * n + w], (float)grho);
        }
    }
}

static int accumulate(dn_shot *s, const dn_accum_opts *o)
{
    DnRange range("gradient assembly");
    if (!s) return dn_fail(DN_EINVAL, "null shot");
    if (!s->correlated) return dn_fail(DN_ESTATE, "dn_shot_accumulate_gradient: no completed adjoint run");
    const bool precond = o && o->energy;
    const int ep = s->p.eprecond;
    if (precond && ep != 1 && ep != 3)
        return dn_fail(DN_EINVAL, "energy preconditioning needs EPRECOND 1 or 3 in the shot's parameters (got %d)", ep);
    const bool taper = o && o->circular_taper;
    if (taper && (o->srtshape != 1 && o->srtshape != 2))
        return dn_fail(DN_EINVAL, "circular taper: SRTSHAPE must be 1 or 2 (got %d)", o->srtshape);
    if (taper && (!(o->srtradius >= 0.0f) || o->srtradius > 1e6f || o->filtsize < 0 || o->filtsize > 1000))
        return dn_fail(DN_EINVAL, "circular taper: SRTRADIUS %g, FILTSIZE %d out of range", o->srtradius, o->filtsize);
    dn_model *m = s->m;
    DevState *ds;
    int st = dev_state(m->device, &ds);
    if (st) return st;
    CU(cudaSetDevice(m->device));
    const int nx = s->p.nx, ny = s->p.ny;
    const long long n = (long long)nx * ny;
    int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 16);
    char *buf = nullptr;
    float *We = nullptr;
    unsigned *maxbits = nullptr;
    ShotTaperArgs tp = {};
    std::vector<char> hbuf;     // box values, then the zeroed cells
    size_t tap_mb = 0;
    size_t we_bytes = precond ? carve_size(n, 4) + 256 : 0, tap_off = we_bytes;
    if (taper) {
        dnp_shot_taper_t t;
        if (dnp_shot_taper(nx, ny, s->p.dh, o->srtshape, o->srtradius, o->src_x, o->src_z, &t))
            return dn_fail(DN_ENOMEM, "circular taper set-up");
        int ci, cj, *cells = nullptr, ncells = 0;
        dnp_source_cell(o->src_x, o->src_z, s->p.dh, &ci, &cj);
        if (dnp_zero_cells(nx, ny, 1, &ci, &cj, o->filtsize, 1, &cells, &ncells)) {
            free(t.m);
            return dn_fail(DN_ENOMEM, "circular taper set-up");
        }
        tap_mb = carve_size((size_t)t.G * t.G, 4);
        hbuf.assign(tap_mb + carve_size((size_t)ncells + 1, 4), 0);
        memcpy(hbuf.data(), t.m, sizeof(float) * t.G * t.G);
        memcpy(hbuf.data() + tap_mb, cells, sizeof(int) * ncells);
        tp.on = 1;
        tp.G = t.G;
        tp.x0 = t.x0;
        tp.z0 = t.z0;
        tp.minm = t.minm;
        tp.maxm = t.maxm;
        tp.nz = ncells;
        tp.zr0 = ny + 1;
        tp.zr1 = 0;
        for (int k = 0; k < ncells; k++) {
            tp.zr0 = std::min(tp.zr0, cells[k] / nx + 1);
            tp.zr1 = std::max(tp.zr1, cells[k] / nx + 1);
        }
        free(t.m);
        free(cells);
    }
    const size_t total = tap_off + hbuf.size();
    if (total) CU(dn_malloc(&buf, total));
    if (precond) {
        We = (float *)buf;
        maxbits = (unsigned *)(buf + carve_size(n, 4));
        CU(cudaMemsetAsync(maxbits, 0, 4, ds->stream));
        k_energy_weight<<<blocks, 256, 0, ds->stream>>>(nx, ny, ep, s->p.dh, (const float *)acc_ptr(s, 3),
                                                        (const float *)acc_ptr(s, 4), We, maxbits);
    }
    if (taper) {
        CU(cudaMemcpyAsync(buf + tap_off, hbuf.data(), hbuf.size(), cudaMemcpyHostToDevice, ds->stream));
        tp.m = (const float *)(buf + tap_off);
        tp.zc = (const int *)(buf + tap_off + tap_mb);
    }
    const float cvp = precond ? o->c_vp : 0.0f, cvs = precond ? o->c_vs : 0.0f, crho = precond ? o->c_rho : 0.0f;
    k_ass_grad<<<blocks, 256, 0, ds->stream>>>(nx, ny, m->lay.pitch, m->field(MF_RHO), m->field(MF_VP),
                                               m->field(MF_VS), m->field(MF_GMUSS), m->field(MF_GLAMSS), acc_ptr(s, 0),
                                               acc_ptr(s, 1), acc_ptr(s, 2), s->acc64, s->p.dt, m->dgrad, m->grad64,
                                               We, maxbits, cvp, cvs, crho, tp);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ds->stream);
    dn_free(buf);
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "gradient assembly: %s", cudaGetErrorString(e));
    return DN_OK;
}

extern "C" int dn_shot_accumulate_gradient(dn_shot *s) { return accumulate(s, nullptr); }

extern "C" int dn_shot_accumulate_gradient_precond(dn_shot *s, float c_vp, float c_vs, float c_rho)
{
    dn_accum_opts o = {};
    o.energy = 1;
    o.c_vp = c_vp;
    o.c_vs = c_vs;
    o.c_rho = c_rho;
    return accumulate(s, &o);
}

extern "C" int dn_shot_accumulate_gradient_ex(dn_shot *s, const dn_accum_opts *o)
{
    if (!o) return dn_fail(DN_EINVAL, "dn_shot_accumulate_gradient_ex: null options");
    return accumulate(s, o);
}

extern "C" int dn_model_get_gradient(const dn_model *m, float *g_vp, float *g_vs, float *g_rho)
{
    if (!m) return dn_fail(DN_EINVAL, "null model");
    const int nx = m->p.nx, ny = m->p.ny;
    const size_t n = (size_t)nx * ny;
    std::vector<char> h(3 * n * (m->grad64 ? 8 : 4));
    CU(cudaSetDevice(m->device));
    CU(cudaMemcpy(h.data(), m->dgrad, h.size(), cudaMemcpyDeviceToHost));
    float *outs[3] = {g_vp, g_vs, g_rho};
    for (int c = 0; c < 3; c++) {
        if (!outs[c]) continue;
        for (int j = 1; j <= ny; j++)
            for (int i = 1; i <= nx; i++) {
                size_t w = c * n + (size_t)(j - 1) * nx + (i - 1);
                outs[c][(size_t)(i - 1) * ny + (j - 1)] = m->grad64 ? (float)((double *)h.data())[w] : ((float *)h.data())[w];
            }
    }
    return DN_OK;
}

extern "C" int dn_model_zero_gradient(dn_model *m)
{
    if (!m) return dn_fail(DN_EINVAL, "null model");
    CU(cudaSetDevice(m->device));
    CU(cudaMemset(m->dgrad, 0, 3 * (size_t)m->p.nx * m->p.ny * (m->grad64 ? 8 : 4)));
    return DN_OK;
}

extern "C" int dn_model_set_gradient(dn_model *m, const float *g_vp, const float *g_vs, const float *g_rho)
{
    if (!m) return dn_fail(DN_EINVAL, "null model");
    const int nx = m->p.nx, ny = m->p.ny;
    const size_t n = (size_t)nx * ny, eb = m->grad64 ? 8 : 4;
    const float *ins[3] = {g_vp, g_vs, g_rho};
    std::vector<char> h(n * eb);
    CU(cudaSetDevice(m->device));
    for (int c = 0; c < 3; c++) {
        if (!ins[c]) continue;
        for (int i = 1; i <= nx; i++)
            for (int j = 1; j <= ny; j++) {
                const float v = ins[c][(size_t)(i - 1) * ny + (j - 1)];
                const size_t w = (size_t)(j - 1) * nx + (i - 1);
                if (m->grad64)
                    ((double *)h.data())[w] = v;
                else
                    ((float *)h.data())[w] = v;
            }
        CU(cudaMemcpy((char *)m->dgrad + c * n * eb, h.data(), n * eb, cudaMemcpyHostToDevice));
    }
    return DN_OK;
}

// the stacked gradient as doubles on the device (for a collective sum over ranks) and back
static __global__ void k_grad_export(const void *__restrict__ g, int g64, double *__restrict__ out, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride)
        out[e] = g64 ? ((const double *)g)[e] : (double)((const float *)g)[e];
}
static __global__ void k_grad_import(void *__restrict__ g, int g64, const double *__restrict__ in, long long n)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        if (g64)
            ((double *)g)[e] = in[e];
        else
            ((float *)g)[e] = __double2float_rn(in[e]);
    }
}

extern "C" int dn_model_gradient_to_device(const dn_model *m, double *d_out)
{
    if (!m || !d_out) return dn_fail(DN_EINVAL, "dn_model_gradient_to_device: null argument");
    CU(cudaSetDevice(m->device));
    CU(cudaDeviceSynchronize());
    k_grad_export<<<148 * 4, 256>>>(m->dgrad, m->grad64, d_out, 3LL * m->p.nx * m->p.ny);
    CU(cudaGetLastError());
    CU(cudaDeviceSynchronize());
    return DN_OK;
}

extern "C" int dn_model_gradient_from_device(dn_model *m, const double *d_in)
{
    if (!m || !d_in) return dn_fail(DN_EINVAL, "dn_model_gradient_from_device: null argument");
    CU(cudaSetDevice(m->device));
    CU(cudaDeviceSynchronize());
    k_grad_import<<<148 * 4, 256>>>(m->dgrad, m->grad64, d_in, 3LL * m->p.nx * m->p.ny);
    CU(cudaGetLastError());
    CU(cudaDeviceSynchronize());
    return DN_OK;
}

extern "C" int dn_model_view_get(dn_model *m, dn_model_view *v)
{
    if (!m || !v) return dn_fail(DN_EINVAL, "null argument");
    v->nx = m->p.nx;
    v->ny = m->p.ny;
    v->pitch = m->lay.pitch;
    v->device = m->device;
    v->grad64 = m->grad64;
    v->dgrad = m->dgrad;
    v->vs = m->field(MF_VS);
    v->vp = m->field(MF_VP);
    v->rho = m->field(MF_RHO);
    return DN_OK;
}

// ---------------------------------------------------------------------------
// per-kernel timing of the batched step (direct launches, CUDA events on the
// engine stream between the kernels); ms_out[8]: average ms per launch of
// v, inject_v, s, inject_s, surface, seismo, snap_store, correlate
// ---------------------------------------------------------------------------
extern "C" int dn_profile_steps(dn_shot *const *shots, int n, int mode, int nsteps, double *ms_out)
{
    LaunchCfg c;
    int st = check_batch(shots, n, mode, c);
    if (st) return st;
    if (nsteps < 1 || !ms_out) return dn_fail(DN_EINVAL, "dn_profile_steps: bad arguments");
    const int device = shots[0]->m->device;
    DevState *ds;
    st = dev_state(device, &ds);
    if (st) return st;
    CU(cudaSetDevice(device));
    st = prepare_launch(c);
    if (st) return st;
    std::vector<Inst> h;
    int maxnt = 0;
    for (int k = 0; k < n; k++) {
        h.push_back(make_inst(shots[k], mode, &c));
        maxnt = std::max(maxnt, shots[k]->p.nt);
    }
    nsteps = std::min(nsteps, maxnt);
    Inst *d = nullptr;
    CU(dn_malloc(&d, sizeof(Inst) * n));
    CU(cudaMemcpyAsync(d, h.data(), sizeof(Inst) * n, cudaMemcpyHostToDevice, ds->stream));
    for (int k = 0; k < n; k++) {
        st = zero_for_run(shots[k], mode, ds->stream);
        if (st) {
            dn_free(d);
            return st;
        }
    }
    cudaEvent_t ev[9];
    for (int k = 0; k < 9; k++) cudaEventCreate(&ev[k]);
    double acc[8] = {0};
    long long nl = 0;
    for (int t = 1; t <= nsteps; t++) {
        launch_step(c, ds->stream, d, ds->d_zero, t, nl, ev);
        cudaEventSynchronize(ev[8]);
        for (int k = 0; k < 8; k++) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
            acc[k] += ms;
        }
    }
    for (int k = 0; k < 8; k++) ms_out[k] = acc[k] / nsteps;
    for (int k = 0; k < 9; k++) cudaEventDestroy(ev[k]);
    cudaError_t e = cudaGetLastError();
    cudaStreamSynchronize(ds->stream);
    dn_free(d);
    for (int k = 0; k < n; k++) {
        if (mode == 0) shots[k]->stored = 0;
        if (mode == 1) shots[k]->correlated = 0;
    }
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "dn_profile_steps: %s", cudaGetErrorString(e));
    return DN_OK;
}

// ---------------------------------------------------------------------------
// data residual of a forward-run shot into its adjoint sources (calc_res_PSV +
// calc_res, LNORM 2): obs [ntr][nt] host, comp DN_SEC_VX / VY / P
// ---------------------------------------------------------------------------
extern "C" int dn_residual_run_ex(const float *syn_tm, const float *obs, float *res, int ntr, int nt, float dt,
                                  float dh, const int *rec_i, const int *rec_j, const dn_residual_opts *o,
                                  double *misfit, cudaStream_t st);

// calc_res of one recorded component against host observed data; the residual
// becomes the shot's adjoint source of that component
static int shot_source(dn_shot *s, int comp, const float *obs, double *l2, const dn_residual_opts *o)
{
    DnRange range("adjoint source");
    if (!s || !obs || !o) return dn_fail(DN_EINVAL, "dn_shot_residual: null argument");
    if (comp != DN_SEC_VX && comp != DN_SEC_VY && comp != DN_SEC_P)
        return dn_fail(DN_EINVAL, "dn_shot_residual: component must be vx, vy or p");
    if (s->ntr < 1) return dn_fail(DN_EINVAL, "dn_shot_residual: shot has no receivers");
    DevState *ds;
    int st = dev_state(s->m->device, &ds);
    if (st) return st;
    CU(cudaSetDevice(s->m->device));
    const int nt = s->p.nt, ntr = s->ntr;
    const size_t n = (size_t)ntr * nt;
    float *dobs = nullptr;
    if (dn_malloc(&dobs, n * 4) != cudaSuccess) {
        cudaGetLastError();
        return dn_fail(DN_ENOMEM, "dn_shot_residual: device allocation failed");
    }
    const int k = comp == DN_SEC_VX ? 0 : (comp == DN_SEC_VY ? 1 : 2);
    const size_t rs = (size_t)std::max(s->ntr, 1) * nt;
    double h = 0.0;
    cudaError_t e = cudaMemcpyAsync(dobs, obs, n * 4, cudaMemcpyHostToDevice, ds->stream);
    if (e == cudaSuccess)
        st = dn_residual_run_ex(s->d_sec + (size_t)comp * nt * ntr, dobs, s->d_res + k * rs, ntr, nt, s->p.dt, s->p.dh,
                                s->rec_i.data(), s->rec_j.data(), o, &h, ds->stream);
    else
        st = dn_fail(DN_EDEVICE, "dn_shot_residual: %s", cudaGetErrorString(e));
    dn_free(dobs);
    if (st) return st;
    s->has_res[k] = 1;
    if (l2) *l2 = h;
    return DN_OK;
}

static dn_residual_opts l2_opts(const dn_shot *s, int rtm)
{
    dn_residual_opts o = {};
    o.lnorm = 2;
    o.grad_form = s ? s->p.grad_form : 1;
    o.mode = rtm ? 2 : 1;
    return o;
}

extern "C" int dn_shot_residual(dn_shot *s, int comp, const float *obs, double *l2)
{
    const dn_residual_opts o = l2_opts(s, 0);
    return shot_source(s, comp, obs, l2, &o);
}

extern "C" int dn_shot_rtm_source(dn_shot *s, int comp, const float *obs)
{
    const dn_residual_opts o = l2_opts(s, 1);
    return shot_source(s, comp, obs, nullptr, &o);
}

extern "C" int dn_shot_residual_ex(dn_shot *s, int comp, const float *obs, const dn_residual_opts *o, double *misfit)
{
    return shot_source(s, comp, obs, misfit, o);
}
