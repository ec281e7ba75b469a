// Per-kernel drop-ins with the exact signatures of the reference's
// update_v_PML_PSV (include/fd.h:324), update_s_elastic_PML_PSV (:309) and
// update_s_visc_PML_PSV (:316), built as their own library
// (libdenise_b200_fd.so).  A reference build links it in place of those files
// of src/PSV/ to swap one kernel at a time and compare;
// the library reads the reference's globals (NX, NY, FDORDER, FW, DT, DH,
// FREE_SURF, BOUNDARY, NPROCX, NPROCY, POS, GRAD_FORM, INVMAT1, QUELLTYPB, NT)
// and reports failures through the reference's err(), as its own functions do.
//
// Each call copies the NR-style arrays it reads (one MPI-free domain, the
// halos of nd = FDORDER/2 + 1 cells that alloc_PSV gives the fields) into the
// engine's padded device planes, runs the engine's kernel for that one step
// (k_update_v2 with its force sources or k_inject_v's adjoint forces;
// k_update_s_el2; k_update_s_vi reading the prepared fipjp, f, g, d, e, dip
// it is handed) and copies back what the reference function writes: the
// interior of the updated fields, vxp1 / vyp1 and the CPML memory.  The kernels
// are the ones dn_run uses, so the results are bit-identical to the
// reference's; the copies make a call cost milliseconds, so this boundary is a
// parity tool, not the fast path (that is dn_run, which keeps the state in HBM).
//
// Supported: the whole single-rank domain (nx1 = 1, nx2 = NX, ny1 = 1,
// ny2 = NY, NPROCX = NPROCY = 1), BOUNDARY 0, GRAD_FORM 1, INVMAT1 1 or 3; the
// CPML memory arrays as alloc_PSV allocates them (x frame NY x 2 FW, z frame
// 2 FW x NX, one block each), srcpos_loc, signals and signals1 as matrix()
// blocks.  Anything else ends in err().
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "dn_kernels.cuh"

extern "C" {
// the reference's globals (include/globvar.h) and error exit (src/util.c:7)
extern int NX, NY, NT, FDORDER, FW, FREE_SURF, BOUNDARY, NPROCX, NPROCY, GRAD_FORM, INVMAT1, QUELLTYP, QUELLTYPB, L;
extern int POS[3];
extern float DT, DH;
void err(char err_text[]);
}

namespace {

using dn::Inst;

// planes of the shim's device state
enum { P_VX, P_VY, P_SXX, P_SYY, P_SXY, P_VXP1, P_VYP1, P_RIP, P_RJP, P_UIPJP, P_MU, P_LAM, P_COUNT };

struct ShimState {
    int nx = 0, ny = 0, fw = -1, device = -1;
    int pitch = 0, rows = 0;
    long long plane = 0, origin = 0;
    float *planes = nullptr;          // P_COUNT padded planes
    float *psi = nullptr;             // two x-frame blocks (ny x 2fw), then two z-frame blocks (2fw x nx)
    float *pml = nullptr;             // 12 CPML vectors of 2fw
    int *d_zero = nullptr;            // step base 0 (the kernels' step is *ntb + off)
    Inst *d_inst = nullptr;
    std::vector<float> stage;         // one plane on the host
    float *visc = nullptr;            // viscoelastic planes: r, p, q, d, e, dip (L each), fipjp, f, g
    int visc_L = 0;
};
ShimState g;

void fail(const char *msg)
{
    char buf[512];
    snprintf(buf, sizeof(buf), "denise_b200 fd shim: %s", msg);
    err(buf);
}

void cu(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) {
        char buf[400];
        snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
        fail(buf);
    }
}

// the domain the reference functions may be called on here
void check_domain(int nx1, int nx2, int ny1, int ny2)
{
    if (nx1 != 1 || nx2 != NX || ny1 != 1 || ny2 != NY)
        fail("only the whole domain (1..NX, 1..NY) is supported");
    if (NPROCX != 1 || NPROCY != 1 || POS[1] != 0 || POS[2] != 0)
        fail("only one MPI rank (NPROCX = NPROCY = 1) is supported");
    if (BOUNDARY != 0) fail("BOUNDARY (periodic edges) is not supported");
    if (GRAD_FORM != 1) fail("only GRAD_FORM 1 is supported");
    if (FDORDER < 2 || FDORDER > 12 || (FDORDER & 1)) fail("FDORDER must be 2, 4, ..., 12");
}

float *plane(int k) { return g.planes + (long long)k * g.plane + g.origin; }

void ensure_state()
{
    const int fw = std::max(FW, 1);
    int dev = 0;
    cu(cudaGetDevice(&dev), "cudaGetDevice");
    if (g.planes && g.nx == NX && g.ny == NY && g.fw == fw && g.device == dev) return;
    if (g.visc) cudaFree(g.visc);
    g.visc = nullptr;
    g.visc_L = 0;
    if (g.planes) {
        cudaFree(g.planes);
        cudaFree(g.psi);
        cudaFree(g.pml);
        cudaFree(g.d_zero);
        cudaFree(g.d_inst);
    }
    g.nx = NX;
    g.ny = NY;
    g.fw = fw;
    g.device = dev;
    // the engine's padded layout: DN_HX / DN_HZ halo columns / rows (more than the
    // reference's nd = FDORDER/2 + 1 <= 7), pitch a multiple of 32 floats
    g.pitch = ((NX + 2 * DN_HX) + 31) / 32 * 32;
    g.rows = NY + 2 * DN_HZ;
    g.plane = (long long)g.pitch * g.rows;
    g.origin = (long long)(DN_HZ - 1) * g.pitch + (DN_HX - 1);
    const size_t xf = (size_t)NY * 2 * fw, zf = (size_t)2 * fw * NX;
    cu(cudaMalloc(&g.planes, (size_t)P_COUNT * g.plane * 4), "cudaMalloc planes");
    cu(cudaMemset(g.planes, 0, (size_t)P_COUNT * g.plane * 4), "cudaMemset planes");
    cu(cudaMalloc(&g.psi, (2 * xf + 2 * zf) * 4), "cudaMalloc CPML memory");
    cu(cudaMalloc(&g.pml, (size_t)12 * 2 * fw * 4), "cudaMalloc CPML vectors");
    cu(cudaMalloc(&g.d_zero, sizeof(int)), "cudaMalloc step base");
    cu(cudaMemset(g.d_zero, 0, sizeof(int)), "cudaMemset step base");
    cu(cudaMalloc(&g.d_inst, sizeof(Inst)), "cudaMalloc descriptor");
    g.stage.assign((size_t)g.plane, 0.0f);
}

// an NR field m[-nd+1..NY+nd][-nd+1..NX+nd] (halos included) into plane k
void field_in(int k, float **m)
{
    const int nd = FDORDER / 2 + 1;
    float *s = g.stage.data() + g.origin;
    for (int j = -nd + 1; j <= NY + nd; j++)
        memcpy(s + (long long)j * g.pitch - nd + 1, &m[j][-nd + 1], (size_t)(NX + 2 * nd) * 4);
    cu(cudaMemcpy(g.planes + (long long)k * g.plane, g.stage.data(), g.plane * 4, cudaMemcpyHostToDevice),
       "copy of a field");
}

// the interior m[1..NY][1..NX] into plane k (the kernels read no halo of it)
void interior_in(int k, float **m)
{
    std::fill(g.stage.begin(), g.stage.end(), 0.0f);
    float *s = g.stage.data() + g.origin;
    for (int j = 1; j <= NY; j++) memcpy(s + (long long)j * g.pitch + 1, &m[j][1], (size_t)NX * 4);
    cu(cudaMemcpy(g.planes + (long long)k * g.plane, g.stage.data(), g.plane * 4, cudaMemcpyHostToDevice),
       "copy of a material");
}

// the interior of plane k back into m[1..NY][1..NX]
void interior_out(int k, float **m)
{
    cu(cudaMemcpy(g.stage.data(), g.planes + (long long)k * g.plane, g.plane * 4, cudaMemcpyDeviceToHost),
       "copy back of a field");
    const float *s = g.stage.data() + g.origin;
    for (int j = 1; j <= NY; j++) memcpy(&m[j][1], s + (long long)j * g.pitch + 1, (size_t)NX * 4);
}

// CPML memory blocks: slot 0, 1 x frame (matrix(1,NY,1,2FW)), slot 2, 3 z frame (matrix(1,2FW,1,NX))
float *psi_slot(int k)
{
    const size_t xf = (size_t)NY * 2 * g.fw, zf = (size_t)2 * g.fw * NX;
    return k < 2 ? g.psi + k * xf : g.psi + 2 * xf + (k - 2) * zf;
}
size_t psi_count(int k) { return k < 2 ? (size_t)NY * 2 * g.fw : (size_t)2 * g.fw * NX; }
void psi_in(int k, float **m)
{
    if (FW > 0) cu(cudaMemcpy(psi_slot(k), &m[1][1], psi_count(k) * 4, cudaMemcpyHostToDevice), "copy of CPML memory");
}
void psi_out(int k, float **m)
{
    if (FW > 0)
        cu(cudaMemcpy(&m[1][1], psi_slot(k), psi_count(k) * 4, cudaMemcpyDeviceToHost), "copy back of CPML memory");
}

// descriptor fields shared by both updates
Inst base_inst(const float *hc, float *const v12[12])
{
    Inst I;
    memset(&I, 0, sizeof(I));
    I.nx = NX;
    I.ny = NY;
    I.nt = NT;
    I.pitch = g.pitch;
    I.fw = FW;
    I.free_surf = FREE_SURF;
    I.zch = 8;
    I.tiles_x = (NX + 127) / 128;
    I.tiles = I.tiles_x * ((NY + 7) / 8);
    I.dtinv = 1;
    I.DT = DT;
    I.DH = DH;
    I.rdh = 1.0f / DH;
    I.fastdiv = 0;   // the IEEE division by DH
    I.dhi_el = DT / DH;
    for (int m = 1; m <= FDORDER / 2; m++) I.hc[m] = hc[m];
    I.vx = plane(P_VX);
    I.vy = plane(P_VY);
    I.sxx = plane(P_SXX);
    I.syy = plane(P_SYY);
    I.sxy = plane(P_SXY);
    I.vxp1 = plane(P_VXP1);
    I.vyp1 = plane(P_VYP1);
    I.rip = plane(P_RIP);
    I.rjp = plane(P_RJP);
    I.uipjp = plane(P_UIPJP);
    I.mu = plane(P_MU);
    I.lam = plane(P_LAM);
    // CPML vectors, the reference's [1..2FW] at index h - 1
    const size_t w = 2 * (size_t)g.fw;
    if (FW > 0)
        for (int k = 0; k < 12; k++)
            cu(cudaMemcpy(g.pml + k * w, &v12[k][1], w * 4, cudaMemcpyHostToDevice), "copy of CPML vectors");
    I.K_x = g.pml + 0 * w;
    I.a_x = g.pml + 1 * w;
    I.b_x = g.pml + 2 * w;
    I.K_xh = g.pml + 3 * w;
    I.a_xh = g.pml + 4 * w;
    I.b_xh = g.pml + 5 * w;
    I.K_y = g.pml + 6 * w;
    I.a_y = g.pml + 7 * w;
    I.b_y = g.pml + 8 * w;
    I.K_yh = g.pml + 9 * w;
    I.a_yh = g.pml + 10 * w;
    I.b_yh = g.pml + 11 * w;
    return I;
}

template <int R, bool SRC>
void launch_v(const Inst *d, int nt, dim3 grid)
{
    dn::k_update_v2<R, true, SRC><<<grid, 64>>>(d, g.d_zero, nt);
}
template <bool SRC>
void launch_v_any(const Inst *d, int nt, dim3 grid)
{
    switch (FDORDER / 2) {
    case 1: launch_v<1, SRC>(d, nt, grid); break;
    case 2: launch_v<2, SRC>(d, nt, grid); break;
    case 3: launch_v<3, SRC>(d, nt, grid); break;
    case 4: launch_v<4, SRC>(d, nt, grid); break;
    case 5: launch_v<5, SRC>(d, nt, grid); break;
    default: launch_v<6, SRC>(d, nt, grid); break;
    }
}
void launch_s_any(const Inst *d, int nt, dim3 grid)
{
    switch (FDORDER / 2) {
    case 1: dn::k_update_s_el2<1, true><<<grid, 64>>>(d, g.d_zero, nt); break;
    case 2: dn::k_update_s_el2<2, true><<<grid, 64>>>(d, g.d_zero, nt); break;
    case 3: dn::k_update_s_el2<3, true><<<grid, 64>>>(d, g.d_zero, nt); break;
    case 4: dn::k_update_s_el2<4, true><<<grid, 64>>>(d, g.d_zero, nt); break;
    case 5: dn::k_update_s_el2<5, true><<<grid, 64>>>(d, g.d_zero, nt); break;
    default: dn::k_update_s_el2<6, true><<<grid, 64>>>(d, g.d_zero, nt); break;
    }
}

// small device buffers of one call, freed when the call returns
struct CallBufs {
    std::vector<void *> p;
    template <typename T> T *up(const std::vector<T> &h)
    {
        void *d = nullptr;
        cu(cudaMalloc(&d, std::max(h.size(), (size_t)1) * sizeof(T)), "cudaMalloc source tables");
        if (!h.empty()) cu(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), "copy of source tables");
        p.push_back(d);
        return (T *)d;
    }
    ~CallBufs()
    {
        for (void *d : p) cudaFree(d);
    }
};

}   // namespace

extern "C" void update_v_PML_PSV(int nx1, int nx2, int ny1, int ny2, int nt, float **vx, float **vxp1, float **vxm1,
                                 float **vy, float **vyp1, float **vym1, float **uttx, float **utty, float **sxx,
                                 float **syy, float **sxy, float **rip, float **rjp, float **srcpos_loc,
                                 float **signals, float **signals1, int nsrc, float **absorb_coeff, float *hc,
                                 int infoout, int sw, float *K_x, float *a_x, float *b_x, float *K_x_half,
                                 float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y, float *K_y_half,
                                 float *a_y_half, float *b_y_half, float **psi_sxx_x, float **psi_syy_y,
                                 float **psi_sxy_y, float **psi_sxy_x)
{
    (void)vxm1, (void)vym1, (void)uttx, (void)utty, (void)absorb_coeff, (void)infoout;
    check_domain(nx1, nx2, ny1, ny2);
    if (sw != 0 && sw != 1) fail("update_v_PML_PSV: sw must be 0 or 1");
    ensure_state();
    field_in(P_SXX, sxx);
    field_in(P_SYY, syy);
    field_in(P_SXY, sxy);
    field_in(P_VX, vx);
    field_in(P_VY, vy);
    if (sw == 1) {
        interior_in(P_VXP1, vxp1);
        interior_in(P_VYP1, vyp1);
    }
    interior_in(P_RIP, rip);
    interior_in(P_RJP, rjp);
    psi_in(0, psi_sxx_x);
    psi_in(1, psi_sxy_x);
    psi_in(2, psi_syy_y);
    psi_in(3, psi_sxy_y);
    float *v12[12] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half};
    Inst I = base_inst(hc, v12);
    I.psi_sxx_x = psi_slot(0);
    I.psi_sxy_x = psi_slot(1);
    I.psi_syy_y = psi_slot(2);
    I.psi_sxy_y = psi_slot(3);
    CallBufs cb;
    if (sw == 0) {
        // mode 0 with a snapshot every step: vxp1 = rip (sxx_x + sxy_y) / DH on every call, as
        // update_v_PML_PSV.c:451-453 writes it; force sources in the kernel, list order per cell
        I.mode = 0;
        I.store = 1;
        std::vector<int> perm(nsrc), ci, cj, cs, cc, ty(nsrc);
        std::vector<double> nsin(nsrc), cosv(nsrc);
        for (int l = 0; l < nsrc; l++) {
            perm[l] = l;
            ty[l] = (int)srcpos_loc[8][l + 1];
            const float azi_rad = srcpos_loc[7][l + 1] * 3.141592653589793 / 180;
            nsin[l] = -sin((double)azi_rad);
            cosv[l] = cos((double)azi_rad);
        }
        auto si = [&](int l) { return (int)srcpos_loc[1][l + 1]; };
        auto sj = [&](int l) { return (int)srcpos_loc[2][l + 1]; };
        std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) {
            return sj(a) != sj(b) ? sj(a) < sj(b) : si(a) < si(b);
        });
        for (int k = 0; k < nsrc; k++) {
            const int l = perm[k];
            if (ci.empty() || ci.back() != si(l) || cj.back() != sj(l)) {
                ci.push_back(si(l));
                cj.push_back(sj(l));
                cs.push_back(k);
                cc.push_back(0);
            }
            cc.back()++;
        }
        I.nsrc_cells = (int)ci.size();
        I.nsrc = nsrc;
        I.src_cell_i = cb.up(ci);
        I.src_cell_j = cb.up(cj);
        I.src_cell_start = cb.up(cs);
        I.src_cell_count = cb.up(cc);
        I.src_perm = cb.up(perm);
        I.src_type = cb.up(ty);
        I.src_nsin = cb.up(nsin);
        I.src_cos = cb.up(cosv);
        std::vector<float> sig(nsrc > 0 ? (size_t)nsrc * NT : 0);
        if (nsrc > 0) memcpy(sig.data(), &signals1[1][1], sig.size() * 4);   // matrix(1,nsrc,1,NT): one block
        I.signals = cb.up(sig);
        I.fsrc_v = nsrc > 0;
        if (nsrc > 0) QUELLTYP = ty[nsrc - 1];   // update_v_PML_PSV.c:745 leaves the last source's type
    } else {
        // mode 1: vxp1 += DT vx with the old velocity, then the residual forces of
        // :755-768 at the receivers (k_inject_v, QUELLTYPB)
        I.mode = 1;
        std::vector<int> ri(nsrc), rj(nsrc);
        for (int l = 0; l < nsrc; l++) {
            ri[l] = (int)srcpos_loc[1][l + 1];
            rj[l] = (int)srcpos_loc[2][l + 1];
        }
        I.ntr = nsrc;
        for (int a = 0; a < nsrc && !I.rec_dup; a++)
            for (int b = a + 1; b < nsrc; b++)
                if (ri[a] == ri[b] && rj[a] == rj[b]) I.rec_dup = 1;
        I.rec_i = cb.up(ri);
        I.rec_j = cb.up(rj);
        std::vector<float> rx(nsrc > 0 ? (size_t)nsrc * NT : 0), ry(rx.size());
        if (nsrc > 0) {
            memcpy(rx.data(), &signals[1][1], rx.size() * 4);
            memcpy(ry.data(), &signals1[1][1], ry.size() * 4);
        }
        I.res_vx = cb.up(rx);
        I.res_vy = cb.up(ry);
        I.quelltypb = QUELLTYPB;
    }
    cu(cudaMemcpy(g.d_inst, &I, sizeof(Inst), cudaMemcpyHostToDevice), "copy of the descriptor");
    const dim3 grid(I.tiles, 1);
    if (I.fsrc_v) launch_v_any<true>(g.d_inst, nt, grid);
    else launch_v_any<false>(g.d_inst, nt, grid);
    if (sw == 1 && nsrc > 0) dn::k_inject_v<<<dim3((nsrc + 127) / 128, 1), 128>>>(g.d_inst, g.d_zero, nt);
    cu(cudaGetLastError(), "update_v_PML_PSV launch");
    cu(cudaDeviceSynchronize(), "update_v_PML_PSV");
    interior_out(P_VX, vx);
    interior_out(P_VY, vy);
    interior_out(P_VXP1, vxp1);
    interior_out(P_VYP1, vyp1);
    psi_out(0, psi_sxx_x);
    psi_out(1, psi_sxy_x);
    psi_out(2, psi_syy_y);
    psi_out(3, psi_sxy_y);
}

extern "C" void update_s_elastic_PML_PSV(int nx1, int nx2, int ny1, int ny2, float **vx, float **vy, float **ux,
                                         float **uy, float **uxy, float **uyx, float **sxx, float **syy, float **sxy,
                                         float **pi, float **u, float **uipjp, float **absorb_coeff, float **rho,
                                         float *hc, int infoout, float *K_x, float *a_x, float *b_x, float *K_x_half,
                                         float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y,
                                         float *K_y_half, float *a_y_half, float *b_y_half, float **psi_vxx,
                                         float **psi_vyy, float **psi_vxy, float **psi_vyx, int mode)
{
    (void)ux, (void)uy, (void)uxy, (void)uyx, (void)absorb_coeff, (void)infoout, (void)mode;
    check_domain(nx1, nx2, ny1, ny2);
    if (INVMAT1 != 1 && INVMAT1 != 3) fail("update_s_elastic_PML_PSV: INVMAT1 must be 1 or 3");
    ensure_state();
    field_in(P_VX, vx);
    field_in(P_VY, vy);
    interior_in(P_SXX, sxx);
    interior_in(P_SYY, syy);
    interior_in(P_SXY, sxy);
    interior_in(P_UIPJP, uipjp);
    // f and g of update_s_elastic_PML_PSV.c:442-449: the moduli themselves (INVMAT1 3) or
    // rho u u and rho (pi pi - 2 u u) in float (INVMAT1 1)
    {
        std::vector<float *> fm(NY + 1), gm(NY + 1);
        std::vector<float> f((size_t)NY * NX), gg((size_t)NY * NX);
        for (int j = 1; j <= NY; j++) {
            fm[j] = f.data() + (size_t)(j - 1) * NX - 1;
            gm[j] = gg.data() + (size_t)(j - 1) * NX - 1;
            for (int i = 1; i <= NX; i++) {
                if (INVMAT1 == 3) {
                    fm[j][i] = u[j][i];
                    gm[j][i] = pi[j][i];
                } else {
                    fm[j][i] = rho[j][i] * u[j][i] * u[j][i];
                    gm[j][i] = rho[j][i] * ((pi[j][i] * pi[j][i]) - 2 * u[j][i] * u[j][i]);
                }
            }
        }
        interior_in(P_MU, fm.data());
        interior_in(P_LAM, gm.data());
    }
    psi_in(0, psi_vxx);
    psi_in(1, psi_vyx);
    psi_in(2, psi_vyy);
    psi_in(3, psi_vxy);
    float *v12[12] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half};
    Inst I = base_inst(hc, v12);
    I.mode = 0;
    I.psi_vxx = psi_slot(0);
    I.psi_vyx = psi_slot(1);
    I.psi_vyy = psi_slot(2);
    I.psi_vxy = psi_slot(3);
    cu(cudaMemcpy(g.d_inst, &I, sizeof(Inst), cudaMemcpyHostToDevice), "copy of the descriptor");
    // the stress kernels take their step from the descriptor only to skip steps outside 1..NT
    launch_s_any(g.d_inst, 1, dim3(I.tiles, 1));
    cu(cudaGetLastError(), "update_s_elastic_PML_PSV launch");
    cu(cudaDeviceSynchronize(), "update_s_elastic_PML_PSV");
    interior_out(P_SXX, sxx);
    interior_out(P_SYY, syy);
    interior_out(P_SXY, sxy);
    psi_out(0, psi_vxx);
    psi_out(1, psi_vyx);
    psi_out(2, psi_vyy);
    psi_out(3, psi_vxy);
}

namespace {

// plane k of the viscoelastic buffer (origin pointer)
float *vplane(int k) { return g.visc + (long long)k * g.plane + g.origin; }

// an f3tensor t[j][i][1..L] (interior) into the L planes from vplane(k0), or back
void tensor_in(int k0, float ***t)
{
    for (int l = 1; l <= L; l++) {
        std::fill(g.stage.begin(), g.stage.end(), 0.0f);
        float *s = g.stage.data() + g.origin;
        for (int j = 1; j <= NY; j++)
            for (int i = 1; i <= NX; i++) s[(long long)j * g.pitch + i] = t[j][i][l];
        cu(cudaMemcpy(g.visc + (long long)(k0 + l - 1) * g.plane, g.stage.data(), g.plane * 4, cudaMemcpyHostToDevice),
           "copy of a viscoelastic tensor");
    }
}
void tensor_out(int k0, float ***t)
{
    for (int l = 1; l <= L; l++) {
        cu(cudaMemcpy(g.stage.data(), g.visc + (long long)(k0 + l - 1) * g.plane, g.plane * 4, cudaMemcpyDeviceToHost),
           "copy back of a viscoelastic tensor");
        const float *s = g.stage.data() + g.origin;
        for (int j = 1; j <= NY; j++)
            for (int i = 1; i <= NX; i++) t[j][i][l] = s[(long long)j * g.pitch + i];
    }
}
void vinterior_in(int k, float **m)
{
    std::fill(g.stage.begin(), g.stage.end(), 0.0f);
    float *s = g.stage.data() + g.origin;
    for (int j = 1; j <= NY; j++) memcpy(s + (long long)j * g.pitch + 1, &m[j][1], (size_t)NX * 4);
    cu(cudaMemcpy(g.visc + (long long)k * g.plane, g.stage.data(), g.plane * 4, cudaMemcpyHostToDevice),
       "copy of a prepared coefficient");
}

template <int LL>
void launch_vi(const Inst *d, dim3 grid)
{
    switch (FDORDER / 2) {
    case 1: dn::k_update_s_vi<1, LL, true, false, true><<<grid, 128>>>(d, g.d_zero, 1); break;
    case 2: dn::k_update_s_vi<2, LL, true, false, true><<<grid, 128>>>(d, g.d_zero, 1); break;
    case 3: dn::k_update_s_vi<3, LL, true, false, true><<<grid, 128>>>(d, g.d_zero, 1); break;
    case 4: dn::k_update_s_vi<4, LL, true, false, true><<<grid, 128>>>(d, g.d_zero, 1); break;
    case 5: dn::k_update_s_vi<5, LL, true, false, true><<<grid, 128>>>(d, g.d_zero, 1); break;
    default: dn::k_update_s_vi<6, LL, true, false, true><<<grid, 128>>>(d, g.d_zero, 1); break;
    }
}

}   // namespace

extern "C" void update_s_visc_PML_PSV(int nx1, int nx2, int ny1, int ny2, float **vx, float **vy, float **ux,
                                      float **uy, float **uxy, float **uyx, float **sxx, float **syy, float **sxy,
                                      float **pi, float **u, float **uipjp, float **rho, float *hc, int infoout,
                                      float ***r, float ***p, float ***q, float **fipjp, float **f, float **gg,
                                      float *bip, float *bjm, float *cip, float *cjm, float ***d, float ***e,
                                      float ***dip, float *K_x, float *a_x, float *b_x, float *K_x_half,
                                      float *a_x_half, float *b_x_half, float *K_y, float *a_y, float *b_y,
                                      float *K_y_half, float *a_y_half, float *b_y_half, float **psi_vxx,
                                      float **psi_vyy, float **psi_vxy, float **psi_vyx, int mode)
{
    (void)ux, (void)uy, (void)uxy, (void)uyx, (void)pi, (void)u, (void)uipjp, (void)rho, (void)infoout, (void)mode;
    check_domain(nx1, nx2, ny1, ny2);
    if (L < 1 || L > DN_MAX_L) fail("update_s_visc_PML_PSV: L must be 1..5");
    // the engine applies one pair (bip, cip) to r, p and q; prepare_update_s_visc_PSV gives bjm = bip, cjm = cip
    for (int l = 1; l <= L; l++)
        if (memcmp(&bip[l], &bjm[l], 4) || memcmp(&cip[l], &cjm[l], 4))
            fail("update_s_visc_PML_PSV: bjm / cjm differ from bip / cip");
    ensure_state();
    if (!g.visc || g.visc_L != L) {
        if (g.visc) cudaFree(g.visc);
        cu(cudaMalloc(&g.visc, (size_t)(6 * L + 3) * g.plane * 4), "cudaMalloc viscoelastic planes");
        g.visc_L = L;
    }
    field_in(P_VX, vx);
    field_in(P_VY, vy);
    interior_in(P_SXX, sxx);
    interior_in(P_SYY, syy);
    interior_in(P_SXY, sxy);
    tensor_in(0 * L, r);
    tensor_in(1 * L, p);
    tensor_in(2 * L, q);
    tensor_in(3 * L, d);
    tensor_in(4 * L, e);
    tensor_in(5 * L, dip);
    vinterior_in(6 * L + 0, fipjp);
    vinterior_in(6 * L + 1, f);
    vinterior_in(6 * L + 2, gg);
    psi_in(0, psi_vxx);
    psi_in(1, psi_vyx);
    psi_in(2, psi_vyy);
    psi_in(3, psi_vxy);
    float *v12[12] = {K_x, a_x, b_x, K_x_half, a_x_half, b_x_half, K_y, a_y, b_y, K_y_half, a_y_half, b_y_half};
    Inst I = base_inst(hc, v12);
    I.mode = 0;
    I.L = L;
    I.plane = g.plane;
    I.dhi_vi = 1.0 / DH;       // update_s_visc_PML_PSV.c: dhi = 1.0/DH, dthalbe = DT/2.0
    I.dthalbe = DT / 2.0;
    for (int l = 0; l < L; l++) {
        I.bip[l] = bip[l + 1];
        I.cip[l] = cip[l + 1];
    }
    I.r = vplane(0 * L);
    I.p = vplane(1 * L);
    I.q = vplane(2 * L);
    I.pre_d = vplane(3 * L);
    I.pre_e = vplane(4 * L);
    I.pre_dip = vplane(5 * L);
    I.pre_fipjp = vplane(6 * L + 0);
    I.pre_f = vplane(6 * L + 1);
    I.pre_g = vplane(6 * L + 2);
    I.psi_vxx = psi_slot(0);
    I.psi_vyx = psi_slot(1);
    I.psi_vyy = psi_slot(2);
    I.psi_vxy = psi_slot(3);
    // one-column tiles of 128 x 8 cells
    I.tiles_x = (NX + 127) / 128;
    I.tiles = I.tiles_x * ((NY + 7) / 8);
    cu(cudaMemcpy(g.d_inst, &I, sizeof(Inst), cudaMemcpyHostToDevice), "copy of the descriptor");
    const dim3 grid(I.tiles, 1);
    switch (L) {
    case 1: launch_vi<1>(g.d_inst, grid); break;
    case 2: launch_vi<2>(g.d_inst, grid); break;
    case 3: launch_vi<3>(g.d_inst, grid); break;
    case 4: launch_vi<4>(g.d_inst, grid); break;
    default: launch_vi<5>(g.d_inst, grid); break;
    }
    cu(cudaGetLastError(), "update_s_visc_PML_PSV launch");
    cu(cudaDeviceSynchronize(), "update_s_visc_PML_PSV");
    interior_out(P_SXX, sxx);
    interior_out(P_SYY, syy);
    interior_out(P_SXY, sxy);
    tensor_out(0 * L, r);
    tensor_out(1 * L, p);
    tensor_out(2 * L, q);
    psi_out(0, psi_vxx);
    psi_out(1, psi_vyx);
    psi_out(2, psi_vyy);
    psi_out(3, psi_vxy);
}
