// Fused elastic time step for forward runs without snapshots (modes 0 and 2).
//
// One kernel does what k_update_v2, k_inject_v, k_update_s_el2, k_inject_s
// and k_surface_el do in sequence: the velocity update with its CPML terms
// (update_v_PML_PSV.c case 2..12 and :386-438), the force sources
// (update_v_PML_PSV.c:738-752), the elastic stress update
// (update_s_elastic_PML_PSV.c), the explosive source (psource.c:23-39) and the
// free surface (surface_elastic_PML_PSV.c:29-103).  Every cell goes through the
// same IEEE operations in the same order as in those kernels, so the state is
// bit-identical to theirs.
//
// Data flow.  The fields and the velocity update's CPML memory alternate
// between two buffers: step nt reads the set written by step nt-1 and writes
// the other one (the primary set when NT - nt is even, so the last step leaves
// the state there).  A CTA owns W = 2 FZ_NP - 2H columns (H = R rounded up to
// even) by f_zc rows.  Its FZ_NP threads each take one column pair of the
// velocity extent, the owned columns plus H on either side, and march down the
// rows: at row k a thread computes the new velocities of its pair into a
// shared-memory ring of 2R+2 rows (and, for owned cells, into the field
// buffer), then, after one barrier, the new stresses of row k - R of its pair
// from the ring.  The halo velocities are recomputed by both neighbouring CTAs
// from the same old values, so they agree bit for bit; the CPML memory they
// read is the old buffer, which nobody writes during the step.  The stress
// update's CPML memory and the free-surface one are touched by their owners
// only and stay in place.
//
// DRAM traffic per cell and step: the old stresses, velocities, rip, rjp,
// uipjp, mu and lambda (40 B) and the new stresses and velocities (20 B):
// 60 B against the 80 B of the separate velocity and stress kernels.
#pragma once

#include "dn_kernels.cuh"

namespace dn {

#ifndef DN_FZ_NP
#define DN_FZ_NP 64
#endif
#ifndef DN_FZ_MINB
#define DN_FZ_MINB (1024 / DN_FZ_NP)
#endif
#ifndef DN_FZ_HOIST
#define DN_FZ_HOIST 1
#endif
constexpr int FZ_NP = DN_FZ_NP;   // threads per CTA, one velocity column pair each
constexpr int FZ_MAXSRC = 32;     // source cells of a shot that runs the fused step

__host__ __device__ constexpr int fz_halo(int R) { return (R + 1) & ~1; }
// shared memory of the velocity ring: 2R+2 rows x (vx, vy) x 2 FZ_NP columns
__host__ __device__ constexpr int fz_ring_bytes(int R) { return (2 * R + 2) * 2 * (2 * FZ_NP) * 4; }
// owned columns of a tile
__host__ __device__ constexpr int fz_width(int R) { return 2 * FZ_NP - 2 * fz_halo(R); }

// read (step nt-1) and write (step nt) sets of a fused instance
struct FzBufs {
    const float *vx, *vy, *sxx, *syy, *sxy;
    const float *psxx_x, *psxy_x, *psyy_y, *psxy_y;
    float *wvx, *wvy, *wsxx, *wsyy, *wsxy;
    float *wpsxx_x, *wpsxy_x, *wpsyy_y, *wpsxy_y;
};

__device__ __forceinline__ FzBufs fz_bufs(const Inst &I, int nt)
{
    const bool wb = ((I.nt - nt) & 1) != 0;   // step nt writes the second set
    FzBufs b;
    b.vx = wb ? I.vx : I.vx_b;
    b.vy = wb ? I.vy : I.vy_b;
    b.sxx = wb ? I.sxx : I.sxx_b;
    b.syy = wb ? I.syy : I.syy_b;
    b.sxy = wb ? I.sxy : I.sxy_b;
    b.psxx_x = wb ? I.psi_sxx_x : I.psi_sxx_x_b;
    b.psxy_x = wb ? I.psi_sxy_x : I.psi_sxy_x_b;
    b.psyy_y = wb ? I.psi_syy_y : I.psi_syy_y_b;
    b.psxy_y = wb ? I.psi_sxy_y : I.psi_sxy_y_b;
    b.wvx = wb ? I.vx_b : I.vx;
    b.wvy = wb ? I.vy_b : I.vy;
    b.wsxx = wb ? I.sxx_b : I.sxx;
    b.wsyy = wb ? I.syy_b : I.syy;
    b.wsxy = wb ? I.sxy_b : I.sxy;
    b.wpsxx_x = wb ? I.psi_sxx_x_b : I.psi_sxx_x;
    b.wpsxy_x = wb ? I.psi_sxy_x_b : I.psi_sxy_x;
    b.wpsyy_y = wb ? I.psi_syy_y_b : I.psi_syy_y;
    b.wpsxy_y = wb ? I.psi_sxy_y_b : I.psi_sxy_y;
    return b;
}

// New velocities of the pair (i0, i0 + 1) at row j from the old buffers, as
// k_update_v2 computes them (mode 0 / 2 without snapshots); `own` cells also
// write their CPML memory.
template <int R, bool X>
__device__ __forceinline__ void fz_velocity(const Inst &I, const FzBufs &B, const float *hc, int i0, int j, bool own,
                                            float2 &nvx, float2 &nvy)
{
    const long long P = I.pitch;
    const long long o = (long long)j * P + i0;
    const float DT = I.DT, DH = I.DH, rdh = I.rdh;
    const bool fd = I.fastdiv;
    const int fw = I.fw, nx = I.nx, ny = I.ny, free_surf = I.free_surf;
    pf_l1(B.syy + o + (R + 1) * P);
    pf_l1(B.sxy + o + R * P);
    pf_l1(B.sxx + o + P);
    pf_l1(I.rip + o + P);
    pf_l1(I.rjp + o + P);
    pf_l1(B.vx + o + P);
    pf_l1(B.vy + o + P);
    float2 ax[2 * R];
    {
        const float *row = B.sxx + o - R + 1;
        constexpr int kb = (R % 2 == 0) ? -1 : 0;
        float2 L[R + 1];
#pragma unroll
        for (int q = 0; q <= R; q++) L[q] = ld2(row + kb + 2 * q);
#pragma unroll
        for (int k = 0; k < 2 * R; k++) {
            if (((k - kb) & 1) == 0) ax[k] = L[(k - kb) / 2];
            else ax[k] = make_float2(L[(k - 1 - kb) / 2].y, L[(k + 1 - kb) / 2].x);
        }
    }
    float2 bx[2 * R];
    {
        const float *row = B.sxy + o - R;
        constexpr int kb = (R % 2 == 0) ? 0 : -1;
        float2 L[R + 1];
#pragma unroll
        for (int q = 0; q <= R; q++) L[q] = ld2(row + kb + 2 * q);
#pragma unroll
        for (int k = 0; k < 2 * R; k++) {
            if (((k - kb) & 1) == 0) bx[k] = L[(k - kb) / 2];
            else bx[k] = make_float2(L[(k - 1 - kb) / 2].y, L[(k + 1 - kb) / 2].x);
        }
    }
    float2 sxx_x = MUL2<X>(bc2(hc[1]), SUB2<X>(ax[R], ax[R - 1]));
    float2 sxy_x = MUL2<X>(bc2(hc[1]), SUB2<X>(bx[R], bx[R - 1]));
    float2 sxy_y = MUL2<X>(bc2(hc[1]), SUB2<X>(ld2(B.sxy + o), ld2(B.sxy + o - P)));
    float2 syy_y = MUL2<X>(bc2(hc[1]), SUB2<X>(ld2(B.syy + o + P), ld2(B.syy + o)));
#pragma unroll
    for (int m = 2; m <= R; m++) {
        sxx_x = ADD2<X>(sxx_x, MUL2<X>(bc2(hc[m]), SUB2<X>(ax[R - 1 + m], ax[R - m])));
        sxy_x = ADD2<X>(sxy_x, MUL2<X>(bc2(hc[m]), SUB2<X>(bx[R + m - 1], bx[R - m])));
        sxy_y = ADD2<X>(sxy_y, MUL2<X>(bc2(hc[m]), SUB2<X>(ld2(B.sxy + o + (m - 1) * P), ld2(B.sxy + o - m * P))));
        syy_y = ADD2<X>(syy_y, MUL2<X>(bc2(hc[m]), SUB2<X>(ld2(B.syy + o + m * P), ld2(B.syy + o - (m - 1) * P))));
    }
    if (fw > 0 && (i0 <= fw || i0 + 1 >= nx - fw + 1)) {
        float *sx = &sxx_x.x, *sy = &sxy_x.x;
        for (int lane = 0; lane < 2; lane++) {
            const int i = i0 + lane;
            if (i > nx || !(i <= fw || i >= nx - fw + 1)) continue;
            for (int side = 0; side < 2; side++) {
                if (side == 0 ? (i > fw) : (i < nx - fw + 1)) continue;
                const int h = side == 0 ? i - 1 : i - nx + 2 * fw - 1;
                const long long e = (long long)(j - 1) * 2 * fw + h;
                float v = ADD<X>(MUL<X>(I.b_xh[h], B.psxx_x[e]), MUL<X>(I.a_xh[h], sx[lane]));
                if (own) B.wpsxx_x[e] = v;
                sx[lane] = ADD<X>(DIVK<X>(sx[lane], I.K_xh[h]), v);
                float w = ADD<X>(MUL<X>(I.b_x[h], B.psxy_x[e]), MUL<X>(I.a_x[h], sy[lane]));
                if (own) B.wpsxy_x[e] = w;
                sy[lane] = ADD<X>(DIVK<X>(sy[lane], I.K_x[h]), w);
            }
        }
    }
    if (fw > 0 && ((!free_surf && j <= fw) || j >= ny - fw + 1)) {
        float *sy = &syy_y.x, *sx = &sxy_y.x;
        for (int lane = 0; lane < 2; lane++) {
            const int i = i0 + lane;
            if (i > nx) continue;
            for (int side = 0; side < 2; side++) {
                if (side == 0 ? (free_surf || j > fw) : (j < ny - fw + 1)) continue;
                const int h = side == 0 ? j - 1 : j - ny + 2 * fw - 1;
                const long long e = (long long)h * nx + (i - 1);
                float v = ADD<X>(MUL<X>(I.b_yh[h], B.psyy_y[e]), MUL<X>(I.a_yh[h], sy[lane]));
                if (own) B.wpsyy_y[e] = v;
                sy[lane] = ADD<X>(DIVK<X>(sy[lane], I.K_yh[h]), v);
                float w = ADD<X>(MUL<X>(I.b_y[h], B.psxy_y[e]), MUL<X>(I.a_y[h], sx[lane]));
                if (own) B.wpsxy_y[e] = w;
                sx[lane] = ADD<X>(DIVK<X>(sx[lane], I.K_y[h]), w);
            }
        }
    }
    const float2 ripv = ld2(I.rip + o), rjpv = ld2(I.rjp + o);
    const float2 vxo = ld2(B.vx + o), vyo = ld2(B.vy + o);
    const float2 s1 = ADD2<X>(sxx_x, sxy_y);
    const float2 s2 = ADD2<X>(sxy_x, syy_y);
    nvx = ADD2<X>(vxo, DIVH2<X>(MUL2<X>(MUL2<X>(bc2(DT), ripv), s1), fd, DH, rdh));
    nvy = ADD2<X>(vyo, DIVH2<X>(MUL2<X>(MUL2<X>(bc2(DT), rjpv), s2), fd, DH, rdh));
}

template <int R, bool X>
__global__ void __launch_bounds__(FZ_NP, DN_FZ_MINB) k_step_el_fused(const Inst *__restrict__ insts, const int *__restrict__ ntb,
                                                             int off)
{
    extern __shared__ float2 fz_ring2[];   // [2R+2][vx, vy][FZ_NP] column pairs
    __shared__ int s_ci[FZ_MAXSRC], s_cj[FZ_MAXSRC], s_cs[FZ_MAXSRC], s_cc[FZ_MAXSRC];
    __shared__ int s_n;
    const Inst &I = insts[blockIdx.y];
    if (!I.pp) return;
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt) return;
    const int b = blockIdx.x;
    if (b >= I.f_tiles) return;
    constexpr int H = fz_halo(R);
    constexpr int SV = 2 * R + 2;
    const int tx = b % I.f_tiles_x, tz = b / I.f_tiles_x;
    const int c0 = tx * I.f_w + 1;                 // first owned column (odd)
    const int j0 = tz * I.f_zc + 1, j1 = min(j0 + I.f_zc - 1, I.ny);
    const int t = threadIdx.x;
    const int i0 = c0 - H + 2 * t;                 // this thread's column pair (i0, i0 + 1), i0 odd
    const int nx = I.nx, ny = I.ny;
    const bool own_col = t >= H / 2 && t < FZ_NP - H / 2 && i0 <= nx;
    const bool two = i0 + 1 <= nx;
    const long long P = I.pitch;
    float hc[R + 1];
#pragma unroll
    for (int m = 1; m <= R; m++) hc[m] = I.hc[m];
    const FzBufs B = fz_bufs(I, nt);
    if (t == 0) {
        int n = 0;
        for (int c = 0; c < I.nsrc_cells && n < FZ_MAXSRC; c++) {
            const int ci = I.src_cell_i[c], cj = I.src_cell_j[c];
            if (cj >= j0 - R && cj <= j1 + R && ci >= c0 - H && ci < c0 - H + 2 * FZ_NP) {
                s_ci[n] = ci;
                s_cj[n] = cj;
                s_cs[n] = I.src_cell_start[c];
                s_cc[n] = I.src_cell_count[c];
                n++;
            }
        }
        s_n = n;
    }
    __syncthreads();
    const int nloc = s_n;
    const bool explosive = I.quelltyp_last == 1;
    const float dhi = I.dhi_el;
    const int kbeg = j0 - R;
    // ring slot of row r (r >= kbeg)
    auto slot = [&](int r) { return (r - kbeg) % SV; };
    for (int k = kbeg; k <= j1 + R; k++) {
        const int j = k - R;   // the stress row of this iteration
        const bool srow = own_col && j >= j0;
        const long long o = (long long)j * P + i0;
#if DN_FZ_HOIST
        // the stress row's own operands are requested before the velocity row is computed
        float2 fipjp, f, g, s_xx, s_yy, s_xy;
        if (srow) {
            fipjp = ld2(I.uipjp + o), f = ld2(I.mu + o), g = ld2(I.lam + o);
            s_xx = ld2(B.sxx + o), s_yy = ld2(B.syy + o), s_xy = ld2(B.sxy + o);
        }
#endif
        // ---- new velocities of row k (zero outside the grid: the halo the reference never updates)
        float2 nvx = make_float2(0.0f, 0.0f), nvy = nvx;
        if (k >= 1 && k <= ny && i0 >= 1 && i0 <= nx) {
            const bool own = own_col && k >= j0 && k <= j1;
            fz_velocity<R, X>(I, B, hc, i0, k, own, nvx, nvy);
            if (!two) nvx.y = nvy.y = 0.0f;
            for (int c = 0; c < nloc; c++) {
                if (s_cj[c] != k || (s_ci[c] != i0 && s_ci[c] != i0 + 1)) continue;
                const bool l1 = s_ci[c] != i0;
                float vx = l1 ? nvx.y : nvx.x, vy = l1 ? nvy.y : nvy.x;
                fz_force(I, s_cs[c], s_cc[c], nt, vx, vy);
                if (l1) nvx.y = vx, nvy.y = vy;
                else nvx.x = vx, nvy.x = vy;
            }
            if (own) {
                const long long o = (long long)k * P + i0;
                st2(B.wvx + o, nvx, two);
                st2(B.wvy + o, nvy, two);
            }
        }
        float2 *ring = fz_ring2 + slot(k) * 2 * FZ_NP;
        ring[t] = nvx;
        ring[FZ_NP + t] = nvy;
        __syncthreads();
        // ---- new stresses of row j = k - R from the ring (rows j - R .. j + R)
        if (!srow) continue;
        const float *rx = reinterpret_cast<const float *>(fz_ring2 + slot(j) * 2 * FZ_NP);
        const float *ry = rx + 2 * FZ_NP;
        // vx x stencil: columns i0-R .. i0+R (ring index of column c: c - c0 + H)
        const int e0 = 2 * t - R;
        float ex[2 * R + 1], ey[2 * R + 1];
#pragma unroll
        for (int m = 0; m <= 2 * R; m++) {
            ex[m] = rx[e0 + m];
            ey[m] = ry[e0 + 1 + m];
        }
        auto VX = [&](int r) { return fz_ring2[slot(r) * 2 * FZ_NP + t]; };
        auto VY = [&](int r) { return fz_ring2[slot(r) * 2 * FZ_NP + FZ_NP + t]; };
        float2 a = MUL2<X>(bc2(hc[1]), SUB2<X>(make_float2(ex[R], ex[R + 1]), make_float2(ex[R - 1], ex[R])));
        float2 bb = MUL2<X>(bc2(hc[1]), SUB2<X>(make_float2(ey[R], ey[R + 1]), make_float2(ey[R - 1], ey[R])));
        float2 c = MUL2<X>(bc2(hc[1]), SUB2<X>(VX(j + 1), VX(j)));
        float2 d = MUL2<X>(bc2(hc[1]), SUB2<X>(VY(j), VY(j - 1)));
#pragma unroll
        for (int m = 2; m <= R; m++) {
            a = ADD2<X>(a, MUL2<X>(bc2(hc[m]), SUB2<X>(make_float2(ex[R + m - 1], ex[R + m]),
                                                       make_float2(ex[R - m], ex[R - m + 1]))));
            bb = ADD2<X>(bb, MUL2<X>(bc2(hc[m]), SUB2<X>(make_float2(ey[R - 1 + m], ey[R + m]),
                                                         make_float2(ey[R - m], ey[R - m + 1]))));
            c = ADD2<X>(c, MUL2<X>(bc2(hc[m]), SUB2<X>(VX(j + m), VX(j - m + 1))));
            d = ADD2<X>(d, MUL2<X>(bc2(hc[m]), SUB2<X>(VY(j + m - 1), VY(j - m))));
        }
        float2 vxx = MUL2<X>(a, bc2(dhi));
        float2 vyx = MUL2<X>(bb, bc2(dhi));
        float2 vxy = MUL2<X>(c, bc2(dhi));
        float2 vyy = MUL2<X>(d, bc2(dhi));
        const int fw = I.fw;
        if (fw > 0 && (i0 <= fw || i0 + 1 >= nx - fw + 1)) {
            float *px = &vxx.x, *py = &vyx.x;
            for (int lane = 0; lane < 2; lane++) {
                const int i = i0 + lane;
                if (i > nx || !(i <= fw || i >= nx - fw + 1)) continue;
                for (int side = 0; side < 2; side++) {
                    if (side == 0 ? (i > fw) : (i < nx - fw + 1)) continue;
                    const int h = side == 0 ? i - 1 : i - nx + 2 * fw - 1;
                    float *p1 = I.psi_vxx + (long long)(j - 1) * 2 * fw + h;
                    float v = ADD<X>(MUL<X>(I.b_x[h], *p1), MUL<X>(I.a_x[h], px[lane]));
                    *p1 = v;
                    px[lane] = ADD<X>(DIVK<X>(px[lane], I.K_x[h]), v);
                    float *p2 = I.psi_vyx + (long long)(j - 1) * 2 * fw + h;
                    float w = ADD<X>(MUL<X>(I.b_xh[h], *p2), MUL<X>(I.a_xh[h], py[lane]));
                    *p2 = w;
                    py[lane] = ADD<X>(DIVK<X>(py[lane], I.K_xh[h]), w);
                }
            }
        }
        if (fw > 0 && ((!I.free_surf && j <= fw) || j >= ny - fw + 1)) {
            float *pyy = &vyy.x, *pxy = &vxy.x;
            for (int lane = 0; lane < 2; lane++) {
                const int i = i0 + lane;
                if (i > nx) continue;
                for (int side = 0; side < 2; side++) {
                    if (side == 0 ? (I.free_surf || j > fw) : (j < ny - fw + 1)) continue;
                    const int h = side == 0 ? j - 1 : j - ny + 2 * fw - 1;
                    float *p1 = I.psi_vyy + (long long)h * nx + (i - 1);
                    float *p2 = I.psi_vxy + (long long)h * nx + (i - 1);
                    float v = ADD<X>(MUL<X>(I.b_y[h], *p1), MUL<X>(I.a_y[h], pyy[lane]));
                    float w = ADD<X>(MUL<X>(I.b_yh[h], *p2), MUL<X>(I.a_yh[h], pxy[lane]));
                    *p1 = v;
                    *p2 = w;
                    pyy[lane] = ADD<X>(DIVK<X>(pyy[lane], I.K_y[h]), v);
                    pxy[lane] = ADD<X>(DIVK<X>(pxy[lane], I.K_yh[h]), w);
                }
            }
        }
#if !DN_FZ_HOIST
        const float2 fipjp = ld2(I.uipjp + o), f = ld2(I.mu + o), g = ld2(I.lam + o);
        const float2 s_xx = ld2(B.sxx + o), s_yy = ld2(B.syy + o), s_xy = ld2(B.sxy + o);
#endif
        const float2 div = ADD2<X>(vxx, vyy);
        const float2 gdiv = MUL2<X>(g, div);
        const float2 nsxy = ADD2<X>(s_xy, MUL2<X>(fipjp, ADD2<X>(vyx, vxy)));
        float2 nsxx, nsyy;
        {
            const double f2x = 2.0 * (double)f.x, f2y = 2.0 * (double)f.y;
            nsxx.x = F(DADD((double)s_xx.x, DADD((double)gdiv.x, DMUL(f2x, (double)vxx.x))));
            nsxx.y = F(DADD((double)s_xx.y, DADD((double)gdiv.y, DMUL(f2y, (double)vxx.y))));
            nsyy.x = F(DADD((double)s_yy.x, DADD((double)gdiv.x, DMUL(f2x, (double)vyy.x))));
            nsyy.y = F(DADD((double)s_yy.y, DADD((double)gdiv.y, DMUL(f2y, (double)vyy.y))));
        }
        if (explosive)
            for (int cc = 0; cc < nloc; cc++) {
                if (s_cj[cc] != j || (s_ci[cc] != i0 && s_ci[cc] != i0 + 1)) continue;
                if (s_ci[cc] == i0) fz_explosive(I, s_cs[cc], s_cc[cc], nt, nsxx.x, nsyy.x);
                else fz_explosive(I, s_cs[cc], s_cc[cc], nt, nsxx.y, nsyy.y);
            }
        st2(B.wsxy + o, nsxy, two);
        st2(B.wsxx + o, nsxx, two);
        st2(B.wsyy + o, nsyy, two);
        // ---- free surface (image method) once rows 1 .. R+1 of these columns are final
        if (I.free_surf && j0 == 1 && j == min(R + 1, j1)) {
            for (int lane = 0; lane < 2; lane++) {
                const int i = i0 + lane;
                if (i > nx) continue;
                const long long os = P + i;   // row 1
                B.wsyy[os] = 0.0f;
                float sxv = 0.0f, syv = 0.0f;
                const float *r1x = reinterpret_cast<const float *>(fz_ring2 + slot(1) * 2 * FZ_NP);
                const int ci = i - c0 + H;   // ring index of column i
#pragma unroll
                for (int m = 1; m <= R; m++) {
                    B.wsyy[os - m * P] = -B.wsyy[os + m * P];
                    B.wsxy[os - m * P] = -B.wsxy[os + (m - 1) * P];
                    sxv = ADD<X>(sxv, MUL<X>(hc[m], SUB<X>(r1x[ci + m - 1], r1x[ci - m])));
                    const float yu = reinterpret_cast<const float *>(fz_ring2 + slot(m) * 2 * FZ_NP + FZ_NP)[ci];
                    const float yd = 1 - m >= 1
                                         ? reinterpret_cast<const float *>(fz_ring2 + slot(1 - m) * 2 * FZ_NP + FZ_NP)[ci]
                                         : 0.0f;
                    syv = ADD<X>(syv, MUL<X>(hc[m], SUB<X>(yu, yd)));
                }
                sxv = MUL<X>(sxv, I.dh1);
                syv = MUL<X>(syv, I.dh1);
                if (fw > 0) {
                    if (i <= fw) {
                        const int h = i - 1;
                        float *ps = I.psi_vxxs + h;
                        float v = ADD<X>(MUL<X>(I.b_x[h], *ps), MUL<X>(I.a_x[h], sxv));
                        *ps = v;
                        sxv = ADD<X>(DIVK<X>(sxv, I.K_x[h]), v);
                    }
                    if (i >= nx - fw + 1) {
                        const int h = i - nx + 2 * fw - 1;
                        float *ps = I.psi_vxxs + h;
                        float v = ADD<X>(MUL<X>(I.b_x[h], *ps), MUL<X>(I.a_x[h], sxv));
                        *ps = v;
                        sxv = ADD<X>(DIVK<X>(sxv, I.K_x[h]), v);
                    }
                }
                const float gs = I.lam[os];
                const float fjm = MUL<X>(I.mu[os], 2.0f);
                const float t1 = MUL<X>(DIV<X>(MUL<X>(gs, gs), ADD<X>(gs, fjm)), sxv);
                const float t2 = MUL<X>(gs, syv);
                B.wsxx[os] = ADD<X>(B.wsxx[os], MUL<X>(-I.DT, ADD<X>(t1, t2)));
            }
        }
    }
}

}   // namespace dn
