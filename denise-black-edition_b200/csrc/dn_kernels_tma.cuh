// Stencil kernels fed by the bulk-copy row pipeline (dn_pipe.cuh).
//
// Same arithmetic as the register-streaming kernels of dn_kernels.cuh (and so
// bit-identical to the reference in EXACT mode); only the data movement
// differs: each row item of a CTA is a set of row segments copied into shared
// memory Q-1 rows ahead, x-neighbours are read from shared memory and the
// vertical stencil is kept in a register window.
//
// Shared-memory row segments start 16-byte aligned: a W-wide segment starts at
// column i0 (padded offset i0-1+8, a multiple of 8 floats), a halo segment of
// W+16 floats at column i0-8 (padded offset i0-1, a multiple of W).  Edge
// tiles copy only up to the padded row end (pitch is a multiple of 32 and at
// least nx+16, so every column a thread with i <= nx reads is copied).
#pragma once

#include "dn_kernels.cuh"
#include "dn_pipe.cuh"

namespace dn {

constexpr int TMA_W = 128;           // columns per CTA (= threads)
constexpr int TMA_WH = TMA_W + 16;   // halo segment width
constexpr int QV = 6;                // pipeline slots of the velocity kernel
constexpr int QS_EL = 5;             // elastic stress kernel
constexpr int QS_VI = 4;             // viscoelastic stress kernel

__host__ __device__ constexpr int slot_floats_v() { return 6 * TMA_W + 2 * TMA_WH; }
__host__ __device__ constexpr int slot_floats_s_el() { return 8 * TMA_W + 2 * TMA_WH; }
__host__ __device__ constexpr int slot_floats_s_vi(int L) { return (11 + 3 * L) * TMA_W + 2 * TMA_WH; }
template <int Q> __host__ __device__ constexpr size_t pipe_smem_bytes(int slot_floats)
{
    return (size_t)Q * slot_floats * 4 + (size_t)Q * 8;
}

struct StripGeom {
    int i0, j0, j1, nrows, wW, wH;
    bool active;
};

__device__ __forceinline__ bool strip_of(const Inst &I, StripGeom &g)
{
    const int b = blockIdx.x;
    if (b >= I.tiles) return false;
    const int tx = b % I.tiles_x, tz = b / I.tiles_x;
    g.i0 = tx * TMA_W + 1;
    g.j0 = tz * I.zch + 1;
    g.j1 = min(g.j0 + I.zch - 1, I.ny);
    g.nrows = g.j1 - g.j0 + 1;
    g.wW = min(TMA_W, I.pitch - (g.i0 - 1 + DN_HX));
    g.wH = min(TMA_WH, I.pitch - (g.i0 - 1));
    g.active = g.i0 + (int)threadIdx.x <= I.nx;
    return true;
}

// ===========================================================================
// velocity update (same operations as k_update_v)
// slot: [0,W) syy row j+R | [W,2W) sxy row j+R-1 | sxx row j (W+16) | sxy row j (W+16)
//       | rip | rjp | vx | vy (W each)
// ===========================================================================
template <int R, bool X>
__global__ void __launch_bounds__(TMA_W) k_update_v_tma(const Inst *__restrict__ insts, const int *__restrict__ ntb,
                                                        int off)
{
    extern __shared__ __align__(128) float smem[];
    const Inst &I = insts[blockIdx.y];
    if (I.pp) return;   // the fused step handles this instance
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt) return;
    StripGeom g;
    if (!strip_of(I, g)) return;
    constexpr int W = TMA_W, WH = TMA_WH;
    const long long P = I.pitch;
    const int lane = threadIdx.x;
    const int i = g.i0 + lane;
    Pipe<QV> pipe;
    pipe.init(smem, slot_floats_v());

    const unsigned total = (unsigned)(6 * g.wW + 2 * g.wH) * 4;
    auto copy_of = [&](int item) {
        const long long j = g.j0 + item;
        RowCopy c;
        c.src = nullptr;
        c.dst = 0;
        c.bytes = 0;
        switch (lane) {
        case 0: c.src = I.syy + (j + R) * P + g.i0; c.dst = 0; c.bytes = g.wW * 4; break;
        case 1: c.src = I.sxy + (j + R - 1) * P + g.i0; c.dst = W; c.bytes = g.wW * 4; break;
        case 2: c.src = I.sxx + j * P + g.i0 - 8; c.dst = 2 * W; c.bytes = g.wH * 4; break;
        case 3: c.src = I.sxy + j * P + g.i0 - 8; c.dst = 2 * W + WH; c.bytes = g.wH * 4; break;
        case 4: c.src = I.rip + j * P + g.i0; c.dst = 2 * W + 2 * WH; c.bytes = g.wW * 4; break;
        case 5: c.src = I.rjp + j * P + g.i0; c.dst = 3 * W + 2 * WH; c.bytes = g.wW * 4; break;
        case 6: c.src = I.vx + j * P + g.i0; c.dst = 4 * W + 2 * WH; c.bytes = g.wW * 4; break;
        case 7: c.src = I.vy + j * P + g.i0; c.dst = 5 * W + 2 * WH; c.bytes = g.wW * 4; break;
        default: break;
        }
        return c;
    };
    if (threadIdx.x < 32)
        for (int it = 0; it < min(QV, g.nrows); it++) pipe.issue(it, copy_of(it), 8, total);

    float hc[R + 1];
#pragma unroll
    for (int m = 1; m <= R; m++) hc[m] = I.hc[m];
    const float DT = I.DT, DH = I.DH;
    const int mode = I.mode;
    const bool snapstep = (mode == 0) && I.store && ((nt - 1) % I.dtinv == 0);
    const int fw = I.fw, nx = I.nx, ny = I.ny, free_surf = I.free_surf;
    const bool xframe = fw > 0 && (i <= fw || i >= nx - fw + 1);
    float *__restrict__ vx = I.vx + i;
    float *__restrict__ vy = I.vy + i;
    float *__restrict__ vxp1 = I.vxp1 + i;
    float *__restrict__ vyp1 = I.vyp1 + i;

    float wyy[2 * R], wxy[2 * R];
#pragma unroll
    for (int k = 0; k < 2 * R - 1; k++) {
        wyy[k] = g.active ? __ldg(I.syy + i + (long long)(g.j0 - R + 1 + k) * P) : 0.0f;
        wxy[k] = g.active ? __ldg(I.sxy + i + (long long)(g.j0 - R + k) * P) : 0.0f;
    }
    for (int it = 0; it < g.nrows; it++) {
        if (!pipe.wait(it)) {
            if (threadIdx.x == 0) atomicOr(I.flag, 2);
            pipe.drain(it, min(it + QV, g.nrows) - 1);
            return;
        }
        // every thread has finished row it-1: its slot takes item it-1+QV
        if (threadIdx.x < 32 && it >= 1 && it - 1 + QV < g.nrows) pipe.issue(it - 1 + QV, copy_of(it - 1 + QV), 8, total);
        const int j = g.j0 + it;
        const float *s = pipe.slot(it);
        if (g.active) {
            const float *a_sxx = s + 2 * W + 8 + lane;
            const float *a_sxy = s + 2 * W + WH + 8 + lane;
            wyy[2 * R - 1] = s[lane];
            wxy[2 * R - 1] = s[W + lane];
            float sxx_x = MUL<X>(hc[1], SUB<X>(a_sxx[1], a_sxx[0]));
            float sxy_x = MUL<X>(hc[1], SUB<X>(a_sxy[0], a_sxy[-1]));
            float sxy_y = MUL<X>(hc[1], SUB<X>(wxy[R], wxy[R - 1]));
            float syy_y = MUL<X>(hc[1], SUB<X>(wyy[R], wyy[R - 1]));
#pragma unroll
            for (int m = 2; m <= R; m++) {
                sxx_x = ADD<X>(sxx_x, MUL<X>(hc[m], SUB<X>(a_sxx[m], a_sxx[1 - m])));
                sxy_x = ADD<X>(sxy_x, MUL<X>(hc[m], SUB<X>(a_sxy[m - 1], a_sxy[-m])));
                sxy_y = ADD<X>(sxy_y, MUL<X>(hc[m], SUB<X>(wxy[R + m - 1], wxy[R - m])));
                syy_y = ADD<X>(syy_y, MUL<X>(hc[m], SUB<X>(wyy[R - 1 + m], wyy[R - m])));
            }
            if (xframe) {
                for (int side = 0; side < 2; side++) {
                    if (side == 0 ? (i > fw) : (i < nx - fw + 1)) continue;
                    const int h = side == 0 ? i - 1 : i - nx + 2 * fw - 1;
                    float *ps = I.psi_sxx_x + (long long)(j - 1) * 2 * fw + h;
                    float v = ADD<X>(MUL<X>(I.b_xh[h], *ps), MUL<X>(I.a_xh[h], sxx_x));
                    *ps = v;
                    sxx_x = ADD<X>(DIV<X>(sxx_x, I.K_xh[h]), v);
                    float *pq = I.psi_sxy_x + (long long)(j - 1) * 2 * fw + h;
                    float w = ADD<X>(MUL<X>(I.b_x[h], *pq), MUL<X>(I.a_x[h], sxy_x));
                    *pq = w;
                    sxy_x = ADD<X>(DIV<X>(sxy_x, I.K_x[h]), w);
                }
            }
            if (fw > 0 && ((!free_surf && j <= fw) || j >= ny - fw + 1)) {
                for (int side = 0; side < 2; side++) {
                    if (side == 0 ? (free_surf || j > fw) : (j < ny - fw + 1)) continue;
                    const int h = side == 0 ? j - 1 : j - ny + 2 * fw - 1;
                    float *ps = I.psi_syy_y + (long long)h * nx + (i - 1);
                    float v = ADD<X>(MUL<X>(I.b_yh[h], *ps), MUL<X>(I.a_yh[h], syy_y));
                    *ps = v;
                    syy_y = ADD<X>(DIV<X>(syy_y, I.K_yh[h]), v);
                    float *pq = I.psi_sxy_y + (long long)h * nx + (i - 1);
                    float w = ADD<X>(MUL<X>(I.b_y[h], *pq), MUL<X>(I.a_y[h], sxy_y));
                    *pq = w;
                    sxy_y = ADD<X>(DIV<X>(sxy_y, I.K_y[h]), w);
                }
            }
            const float *rowv = s + 2 * W + 2 * WH + lane;
            const float ripv = rowv[0], rjpv = rowv[W], vxo = rowv[2 * W], vyo = rowv[3 * W];
            const long long o = (long long)j * P;
            const float s1 = ADD<X>(sxx_x, sxy_y);
            const float s2 = ADD<X>(sxy_x, syy_y);
            if (snapstep) {
                vxp1[o] = DIV<X>(MUL<X>(ripv, s1), DH);
                vyp1[o] = DIV<X>(MUL<X>(rjpv, s2), DH);
            } else if (mode == 1) {
                vxp1[o] = ADD<X>(vxp1[o], MUL<X>(DT, vxo));
                vyp1[o] = ADD<X>(vyp1[o], MUL<X>(DT, vyo));
            }
            vx[o] = ADD<X>(vxo, DIV<X>(MUL<X>(MUL<X>(DT, ripv), s1), DH));
            vy[o] = ADD<X>(vyo, DIV<X>(MUL<X>(MUL<X>(DT, rjpv), s2), DH));
#pragma unroll
            for (int k = 0; k < 2 * R - 1; k++) {
                wyy[k] = wyy[k + 1];
                wxy[k] = wxy[k + 1];
            }
        }
    }
}

// velocity derivatives of row j (update_s_*_PML_PSV.c :366-438) from the
// shared-memory row segments cxr (vx row j, centred on column i) and dyr
// (vy row j) and the register windows wx (vx rows j-R+1..j+R), wy (vy rows j-R..j+R-1)
template <int R, bool X>
__device__ __forceinline__ void vderiv_rows(const Inst &I, const float *hc, int i, int j, float dhi, const float *cxr,
                                            const float *dyr, const float *wx, const float *wy, float &vxx,
                                            float &vyx, float &vxy, float &vyy)
{
    float a = MUL<X>(hc[1], SUB<X>(cxr[0], cxr[-1]));
    float b = MUL<X>(hc[1], SUB<X>(dyr[1], dyr[0]));
    float c = MUL<X>(hc[1], SUB<X>(wx[R], wx[R - 1]));
    float d = MUL<X>(hc[1], SUB<X>(wy[R], wy[R - 1]));
#pragma unroll
    for (int m = 2; m <= R; m++) {
        a = ADD<X>(a, MUL<X>(hc[m], SUB<X>(cxr[m - 1], cxr[-m])));
        b = ADD<X>(b, MUL<X>(hc[m], SUB<X>(dyr[m], dyr[1 - m])));
        c = ADD<X>(c, MUL<X>(hc[m], SUB<X>(wx[R - 1 + m], wx[R - m])));
        d = ADD<X>(d, MUL<X>(hc[m], SUB<X>(wy[R + m - 1], wy[R - m])));
    }
    vxx = MUL<X>(a, dhi);
    vyx = MUL<X>(b, dhi);
    vxy = MUL<X>(c, dhi);
    vyy = MUL<X>(d, dhi);
    const int fw = I.fw, nx = I.nx, ny = I.ny;
    if (fw > 0 && (i <= fw || i >= nx - fw + 1)) {
        for (int side = 0; side < 2; side++) {
            if (side == 0 ? (i > fw) : (i < nx - fw + 1)) continue;
            const int h = side == 0 ? i - 1 : i - nx + 2 * fw - 1;
            float *p1 = I.psi_vxx + (long long)(j - 1) * 2 * fw + h;
            float v = ADD<X>(MUL<X>(I.b_x[h], *p1), MUL<X>(I.a_x[h], vxx));
            *p1 = v;
            vxx = ADD<X>(DIV<X>(vxx, I.K_x[h]), v);
            float *p2 = I.psi_vyx + (long long)(j - 1) * 2 * fw + h;
            float w = ADD<X>(MUL<X>(I.b_xh[h], *p2), MUL<X>(I.a_xh[h], vyx));
            *p2 = w;
            vyx = ADD<X>(DIV<X>(vyx, I.K_xh[h]), w);
        }
    }
    if (fw > 0 && ((!I.free_surf && j <= fw) || j >= ny - fw + 1)) {
        for (int side = 0; side < 2; side++) {
            if (side == 0 ? (I.free_surf || j > fw) : (j < ny - fw + 1)) continue;
            const int h = side == 0 ? j - 1 : j - ny + 2 * fw - 1;
            float *p1 = I.psi_vyy + (long long)h * nx + (i - 1);
            float *p2 = I.psi_vxy + (long long)h * nx + (i - 1);
            float v = ADD<X>(MUL<X>(I.b_y[h], *p1), MUL<X>(I.a_y[h], vyy));
            float w = ADD<X>(MUL<X>(I.b_yh[h], *p2), MUL<X>(I.a_yh[h], vxy));
            *p1 = v;
            *p2 = w;
            vyy = ADD<X>(DIV<X>(vyy, I.K_y[h]), v);
            vxy = ADD<X>(DIV<X>(vxy, I.K_yh[h]), w);
        }
    }
}

// copy `lane` of a stress-kernel item: 0 vx row j+R, 1 vy row j+R-1, 2 vx row j (halo),
// 3 vy row j (halo), 4.. the W-wide per-row fields listed in `rowf`
__device__ __forceinline__ RowCopy stress_copy(const Inst &I, const StripGeom &g, int item, int lane, int R,
                                               const float *const *rowf, int nrowf, const long long *rowoff)
{
    constexpr int W = TMA_W, WH = TMA_WH;
    const long long P = I.pitch;
    const long long j = g.j0 + item;
    RowCopy c;
    c.src = nullptr;
    c.dst = 0;
    c.bytes = 0;
    if (lane == 0) { c.src = I.vx + (j + R) * P + g.i0; c.dst = 0; c.bytes = g.wW * 4; }
    else if (lane == 1) { c.src = I.vy + (j + R - 1) * P + g.i0; c.dst = W; c.bytes = g.wW * 4; }
    else if (lane == 2) { c.src = I.vx + j * P + g.i0 - 8; c.dst = 2 * W; c.bytes = g.wH * 4; }
    else if (lane == 3) { c.src = I.vy + j * P + g.i0 - 8; c.dst = 2 * W + WH; c.bytes = g.wH * 4; }
    else if (lane < 4 + nrowf) {
        const int f = lane - 4;
        c.src = rowf[f] + rowoff[f] + j * P + g.i0;
        c.dst = 2 * W + 2 * WH + f * W;
        c.bytes = g.wW * 4;
    }
    return c;
}

// ===========================================================================
// elastic stress update (same operations as k_update_s_el)
// slot: vx row j+R | vy row j+R-1 | vx row j (W+16) | vy row j (W+16) | uipjp | mu | lam | sxx | syy | sxy
// ===========================================================================
template <int R, bool X>
__global__ void __launch_bounds__(TMA_W) k_update_s_el_tma(const Inst *__restrict__ insts,
                                                           const int *__restrict__ ntb, int off)
{
    extern __shared__ __align__(128) float smem[];
    const Inst &I = insts[blockIdx.y];
    if (I.pp) return;   // the fused step handles this instance
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt) return;
    StripGeom g;
    if (!strip_of(I, g)) return;
    constexpr int W = TMA_W, WH = TMA_WH;
    const long long P = I.pitch;
    const int lane = threadIdx.x;
    const int i = g.i0 + lane;
    Pipe<QS_EL> pipe;
    pipe.init(smem, slot_floats_s_el());
    const float *rowf[6] = {I.uipjp, I.mu, I.lam, I.sxx, I.syy, I.sxy};
    const long long rowoff[6] = {0, 0, 0, 0, 0, 0};
    const unsigned total = (unsigned)(8 * g.wW + 2 * g.wH) * 4;
    if (threadIdx.x < 32)
        for (int it = 0; it < min(QS_EL, g.nrows); it++)
            pipe.issue(it, stress_copy(I, g, it, lane, R, rowf, 6, rowoff), 10, total);

    float hc[R + 1];
#pragma unroll
    for (int m = 1; m <= R; m++) hc[m] = I.hc[m];
    const float dhi = I.dhi_el;
    float wx[2 * R], wy[2 * R];
#pragma unroll
    for (int k = 0; k < 2 * R - 1; k++) {
        wx[k] = g.active ? __ldg(I.vx + i + (long long)(g.j0 - R + 1 + k) * P) : 0.0f;
        wy[k] = g.active ? __ldg(I.vy + i + (long long)(g.j0 - R + k) * P) : 0.0f;
    }
    for (int it = 0; it < g.nrows; it++) {
        if (!pipe.wait(it)) {
            if (threadIdx.x == 0) atomicOr(I.flag, 2);
            pipe.drain(it, min(it + QS_EL, g.nrows) - 1);
            return;
        }
        if (threadIdx.x < 32 && it >= 1 && it - 1 + QS_EL < g.nrows)
            pipe.issue(it - 1 + QS_EL, stress_copy(I, g, it - 1 + QS_EL, lane, R, rowf, 6, rowoff), 10, total);
        const int j = g.j0 + it;
        const float *s = pipe.slot(it);
        if (g.active) {
            wx[2 * R - 1] = s[lane];
            wy[2 * R - 1] = s[W + lane];
            float vxx, vyx, vxy, vyy;
            vderiv_rows<R, X>(I, hc, i, j, dhi, s + 2 * W + 8 + lane, s + 2 * W + WH + 8 + lane, wx, wy, vxx, vyx,
                              vxy, vyy);
            const float *rv = s + 2 * W + 2 * WH + lane;
            const float fipjp = rv[0], f = rv[W], gl = rv[2 * W];
            const float s_xx = rv[3 * W], s_yy = rv[4 * W], s_xy = rv[5 * W];
            const long long o = (long long)j * P + i;
            const float div = ADD<X>(vxx, vyy);
            const float gdiv = MUL<X>(gl, div);
            const double f2 = 2.0 * (double)f;
            I.sxy[o] = ADD<X>(s_xy, MUL<X>(fipjp, ADD<X>(vyx, vxy)));
            I.sxx[o] = F(DADD((double)s_xx, DADD((double)gdiv, DMUL(f2, (double)vxx))));
            I.syy[o] = F(DADD((double)s_yy, DADD((double)gdiv, DMUL(f2, (double)vyy))));
#pragma unroll
            for (int k = 0; k < 2 * R - 1; k++) {
                wx[k] = wx[k + 1];
                wy[k] = wy[k + 1];
            }
        }
    }
}

// ===========================================================================
// viscoelastic stress update (same operations as k_update_s_vi)
// slot: vx/vy window rows | vx/vy row j (halo) | muipjp tausipjp mu taus pi taup | sxx syy sxy | r[L] p[L] q[L]
// ===========================================================================
template <int R, int L, bool X>
__global__ void __launch_bounds__(TMA_W) k_update_s_vi_tma(const Inst *__restrict__ insts,
                                                           const int *__restrict__ ntb, int off)
{
    extern __shared__ __align__(128) float smem[];
    const Inst &I = insts[blockIdx.y];
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt) return;
    StripGeom g;
    if (!strip_of(I, g)) return;
    constexpr int W = TMA_W, WH = TMA_WH;
    constexpr int NF = 9 + 3 * L;
    const long long P = I.pitch;
    const long long PL = I.plane;
    const int lane = threadIdx.x;
    const int i = g.i0 + lane;
    Pipe<QS_VI> pipe;
    pipe.init(smem, slot_floats_s_vi(L));
    const float *rowf[NF];
    long long rowoff[NF];
    {
        const float *base[9] = {I.c_muipjp, I.c_tausipjp, I.c_mu, I.c_taus, I.c_pi, I.c_taup, I.sxx, I.syy, I.sxy};
#pragma unroll
        for (int f = 0; f < 9; f++) {
            rowf[f] = base[f];
            rowoff[f] = 0;
        }
#pragma unroll
        for (int l = 0; l < L; l++) {
            rowf[9 + l] = I.r;
            rowoff[9 + l] = l * PL;
            rowf[9 + L + l] = I.p;
            rowoff[9 + L + l] = l * PL;
            rowf[9 + 2 * L + l] = I.q;
            rowoff[9 + 2 * L + l] = l * PL;
        }
    }
    const unsigned total = (unsigned)((4 + NF - 2) * g.wW + 2 * g.wH) * 4;
    if (threadIdx.x < 32)
        for (int it = 0; it < min(QS_VI, g.nrows); it++)
            pipe.issue(it, stress_copy(I, g, it, lane, R, rowf, NF, rowoff), 4 + NF, total);

    float hc[R + 1];
#pragma unroll
    for (int m = 1; m <= R; m++) hc[m] = I.hc[m];
    const float dhi = I.dhi_vi, DT = I.DT, dthalbe = I.dthalbe;
    const float fL = (float)L;
    float eta[L], bip[L], cip[L];
#pragma unroll
    for (int l = 0; l < L; l++) {
        eta[l] = I.eta[l];
        bip[l] = I.bip[l];
        cip[l] = I.cip[l];
    }
    float wx[2 * R], wy[2 * R];
#pragma unroll
    for (int k = 0; k < 2 * R - 1; k++) {
        wx[k] = g.active ? __ldg(I.vx + i + (long long)(g.j0 - R + 1 + k) * P) : 0.0f;
        wy[k] = g.active ? __ldg(I.vy + i + (long long)(g.j0 - R + k) * P) : 0.0f;
    }
    for (int it = 0; it < g.nrows; it++) {
        if (!pipe.wait(it)) {
            if (threadIdx.x == 0) atomicOr(I.flag, 2);
            pipe.drain(it, min(it + QS_VI, g.nrows) - 1);
            return;
        }
        if (threadIdx.x < 32 && it >= 1 && it - 1 + QS_VI < g.nrows)
            pipe.issue(it - 1 + QS_VI, stress_copy(I, g, it - 1 + QS_VI, lane, R, rowf, NF, rowoff), 4 + NF, total);
        const int j = g.j0 + it;
        const float *s = pipe.slot(it);
        if (g.active) {
            wx[2 * R - 1] = s[lane];
            wy[2 * R - 1] = s[W + lane];
            float vxx, vyx, vxy, vyy;
            vderiv_rows<R, X>(I, hc, i, j, dhi, s + 2 * W + 8 + lane, s + 2 * W + WH + 8 + lane, wx, wy, vxx, vyx,
                              vxy, vyy);
            const float *rv = s + 2 * W + 2 * WH + lane;
            const float muipjp = rv[0], tsij = rv[W], mu = rv[2 * W], taus = rv[3 * W], pi = rv[4 * W],
                        taup = rv[5 * W];
            const float s_xx = rv[6 * W], s_yy = rv[7 * W], s_xy = rv[8 * W];
            const long long o = (long long)j * P + i;
            const float fipjp = F(DMUL((double)__fmul_rn(muipjp, DT), DADD(1.0, (double)__fmul_rn(fL, tsij))));
            const float f = F(DMUL((double)__fmul_rn(mu, DT), DADD(1.0, (double)__fmul_rn(fL, taus))));
            const float gl = F(DMUL((double)__fmul_rn(pi, DT), DADD(1.0, (double)__fmul_rn(fL, taup))));
            float rr[L], pp[L], qq[L];
            float sumr = 0.0f, sump = 0.0f, sumq = 0.0f;
#pragma unroll
            for (int l = 0; l < L; l++) {
                rr[l] = rv[(9 + l) * W];
                pp[l] = rv[(9 + L + l) * W];
                qq[l] = rv[(9 + 2 * L + l) * W];
                sumr = ADD<X>(sumr, rr[l]);
                sump = ADD<X>(sump, pp[l]);
                sumq = ADD<X>(sumq, qq[l]);
            }
            const float sh = ADD<X>(vxy, vyx);
            const float dv = ADD<X>(vxx, vyy);
            const float gdv = MUL<X>(gl, dv);
            const double f2 = 2.0 * (double)f;
            float sxy = ADD<X>(s_xy, ADD<X>(MUL<X>(fipjp, sh), MUL<X>(dthalbe, sumr)));
            float sxx = F(DADD((double)s_xx, DADD(DSUB((double)gdv, DMUL(f2, (double)vyy)), (double)MUL<X>(dthalbe, sump))));
            float syy = F(DADD((double)s_yy, DADD(DSUB((double)gdv, DMUL(f2, (double)vxx)), (double)MUL<X>(dthalbe, sumq))));
            sumr = sump = sumq = 0.0f;
#pragma unroll
            for (int l = 0; l < L; l++) {
                const float dip = MUL<X>(MUL<X>(muipjp, eta[l]), tsij);
                const float dd = MUL<X>(MUL<X>(mu, eta[l]), taus);
                const float ee = MUL<X>(MUL<X>(pi, eta[l]), taup);
                const float r = MUL<X>(bip[l], SUB<X>(MUL<X>(rr[l], cip[l]), MUL<X>(dip, sh)));
                const double d2 = 2.0 * (double)dd;
                const float pv = F(DMUL((double)bip[l], DADD((double)SUB<X>(MUL<X>(pp[l], cip[l]), MUL<X>(ee, dv)), DMUL(d2, (double)vyy))));
                const float qv = F(DMUL((double)bip[l], DADD((double)SUB<X>(MUL<X>(qq[l], cip[l]), MUL<X>(ee, dv)), DMUL(d2, (double)vxx))));
                I.r[o + l * PL] = r;
                I.p[o + l * PL] = pv;
                I.q[o + l * PL] = qv;
                sumr = ADD<X>(sumr, r);
                sump = ADD<X>(sump, pv);
                sumq = ADD<X>(sumq, qv);
            }
            I.sxy[o] = ADD<X>(sxy, MUL<X>(dthalbe, sumr));
            I.sxx[o] = ADD<X>(sxx, MUL<X>(dthalbe, sump));
            I.syy[o] = ADD<X>(syy, MUL<X>(dthalbe, sumq));
#pragma unroll
            for (int k = 0; k < 2 * R - 1; k++) {
                wx[k] = wx[k + 1];
                wy[k] = wy[k + 1];
            }
        }
    }
}

}   // namespace dn
