// Device kernels of the P-SV propagator (sm_100a).
//
// Every kernel works on a batch of shot instances: blockIdx.y selects the
// instance, blockIdx.x a tile of it.  A tile is `bx` columns wide and `zch`
// rows tall.  In the one-column kernels each of bx threads owns one column and
// streams down the rows, keeping the vertical stencil of the fields it
// differentiates in z in a register window (one new load per row per field);
// horizontal neighbours come from L1 (the warp reads 32 consecutive floats,
// shifted by m).  The paired-column kernels (k_update_v2, k_update_s_el2, the
// default for the velocity and elastic stress updates) give each of bx / 2
// threads two adjacent columns computed with packed FP32x2 instructions, read
// their z neighbours from L1 and prefetch the next row's first lines.
//
// Arithmetic: with EXACT = true every float operation is issued with an
// explicit round-to-nearest intrinsic (__fmul_rn, __fadd_rn, ...), which the
// compiler may neither contract into FMA nor reorder, and every term the
// reference's C promotes to double (a float meeting a double literal such as
// 2.0*f*vxx) is evaluated in double.  The result is the IEEE float sequence
// the reference's C source spells out, so the GPU state is bit-identical to
// the reference's CPU state step by step.  EXACT = false allows FMA.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "denise_b200.h"
#include "dn_internal.h"

namespace dn {

// ---------------------------------------------------------------------------
// Per-instance descriptor (one shot in one mode).  Field pointers are
// "origin" pointers: element (j, i) (1-based, the reference's indices) is
// p[j * pitch + i].
// ---------------------------------------------------------------------------
struct Inst {
    int nx, ny, nt, pitch;
    int fw, free_surf, L, mode;       // mode: 0 forward, 1 adjoint, 2 objective
    int zch, tiles_x, tiles;          // rows per tile, tiles across, total tiles
    int store;                        // mode 0: store snapshots
    int dtinv, nsnap, snap_prec, acc64, eprecond;
    int seismo;                       // SEISMO
    float DT, DH, dhi_el, dhi_vi, dh1, dthalbe;
    float hc[7];
    // wavefield state
    float *vx, *vy, *sxx, *syy, *sxy, *vxp1, *vyp1;
    float *r, *p, *q;                 // visco memory variables, plane l at + l * plane
    long long plane;
    // materials (origin pointers)
    const float *rip, *rjp, *uipjp, *mu, *lam;
    const float *rho, *vp, *vs;                       // raw model (gradient terms)
    const float *c_muipjp, *c_tausipjp, *c_mu, *c_taus, *c_pi, *c_taup;   // visco
    const float *gmuss, *glamss;                      // muss, lamss of psv.c:333-334
    float eta[DN_MAX_L], bip[DN_MAX_L], cip[DN_MAX_L];
    // visco free-surface constants per column i (index i-1)
    const float *s_mu, *s_pi, *s_taus, *s_taup;
    float s_bjm[DN_MAX_L];
    // CPML profile vectors (index h-1)
    const float *K_x, *a_x, *b_x, *K_xh, *a_xh, *b_xh, *K_y, *a_y, *b_y, *K_yh, *a_yh, *b_yh;
    // CPML memory: x frame [ny][2fw], z frame [2fw][nx]
    float *psi_sxx_x, *psi_sxy_x, *psi_syy_y, *psi_sxy_y;
    float *psi_vxx, *psi_vyx, *psi_vyy, *psi_vxy, *psi_vxxs;
    // sources (forward) / adjoint sources
    int nsrc_cells;                   // unique source cells
    const int *src_cell_i, *src_cell_j, *src_cell_start, *src_cell_count, *src_perm;
    const int *src_type;              // per source
    const double *src_nsin, *src_cos; // -sin(azimuth), cos(azimuth) (QUELLTYP 4)
    const float *signals;             // [nsrc][nt]
    int quelltyp_last;                // QUELLTYP after update_v's overwrite (last source)
    int nsrc;
    int quelltypb;
    const float *res_vx, *res_vy, *res_p;   // [ntr][nt] adjoint sources (receivers)
    // receivers
    int ntr;
    const int *rec_i, *rec_j;
    float *sec;                       // [ncomp][nt][ntr]
    // snapshots
    void *snap;                       // [nsnap][5][tiles][tile cells] in snap_prec
    float *snap_scale;                // [nsnap][5][tiles]
    // per-shot correlation accumulators (float or double, origin pointers)
    void *wc, *wcu, *wcrho;
    float *Ws, *Wr;
    // status
    int *flag;                        // bit 0: NaN seen at the psv.c:99 probe
    float rdh;                        // RN(1 / DH)
    int fastdiv;                      // division by DH through div_markstein (verified for this DH)
    int t0;                           // step base when the instance joined: its step is *ntb + off - t0
    int snap_base;                    // snapshot k lives in slot k - snap_base (checkpointed segments)
    // fused elastic step (k_step_el_fused): the fields and the velocity update's CPML memory
    // alternate between the buffers above and these; step nt writes the second set when
    // (nt_total - nt) is odd, so the last step leaves the state in the first
    int pp;                           // this instance runs the fused step
    // forward sources applied inside the paired velocity kernel (force, QUELLTYP 2-4) and the
    // stress kernels (explosive, QUELLTYP 1) instead of k_inject_v / k_inject_s
    int fsrc_v, fsrc_s;
    int rec_dup;                      // two receivers share a cell: adjoint sources added in list order
    // prepared viscoelastic coefficients (the per-kernel drop-in of update_s_visc_PML_PSV,
    // which receives them): fipjp, f, g planes and d, e, dip planes per mechanism at + l * plane
    const float *pre_fipjp, *pre_f, *pre_g, *pre_d, *pre_e, *pre_dip;
    int f_w, f_tiles_x, f_zc, f_tiles;   // its tiles: f_w columns x f_zc rows
    float *vx_b, *vy_b, *sxx_b, *syy_b, *sxy_b;
    float *psi_sxx_x_b, *psi_sxy_x_b, *psi_syy_y_b, *psi_sxy_y_b;
};

// ---------------------------------------------------------------------------
// arithmetic helpers
// ---------------------------------------------------------------------------
template <bool X> __device__ __forceinline__ float MUL(float a, float b) { return X ? __fmul_rn(a, b) : a * b; }
template <bool X> __device__ __forceinline__ float ADD(float a, float b) { return X ? __fadd_rn(a, b) : a + b; }
template <bool X> __device__ __forceinline__ float SUB(float a, float b) { return X ? __fsub_rn(a, b) : a - b; }
template <bool X> __device__ __forceinline__ float DIV(float a, float b) { return X ? __fdiv_rn(a, b) : a / b; }
__device__ __forceinline__ double DMUL(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double DADD(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double DSUB(double a, double b) { return __dadd_rn(a, -b); }
__device__ __forceinline__ double DDIV(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float F(double a) { return __double2float_rn(a); }

// ---------------------------------------------------------------------------
// Division by the grid spacing DH without the general division routine.
// Markstein's correction step (P. W. Markstein, "Computation of elementary
// functions on the IBM RISC System/6000 processor", IBM J. Res. Develop.
// 34(1), 1990): with y = RN(1/d), q = RN(a y) and the exact residual
// r = fma(-q, d, a), RN(q + r y) is the correctly rounded a / d while no
// intermediate leaves the normal range.  Dividends outside [2^-100, 2^100]
// (zeros, subnormals, huge values, inf, NaN) take __fdiv_rn; a zero dividend
// returns q = a y, which carries the sign of a.  The host enables this path
// for a DH only after comparing it with __fdiv_rn on all 2^32 dividends
// (k_fastdiv_check), so the result is bit-identical to a / DH.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float div_markstein(float a, float d, float y)
{
    const float q = __fmul_rn(a, y);
    const float r = __fmaf_rn(-q, d, a);
    const float q1 = __fmaf_rn(r, y, q);
    const float aa = fabsf(a);
    if (aa >= 0x1p-100f && aa <= 0x1p100f) return q1;
    if (a == 0.0f) return q;
    return __fdiv_rn(a, d);
}
template <bool X>
__device__ __forceinline__ float DIVH(float a, const Inst &I)
{
    if (!X) return a * I.rdh;
    return I.fastdiv ? div_markstein(a, I.DH, I.rdh) : __fdiv_rn(a, I.DH);
}
// Division by a CPML K coefficient: K = 1 (k_max_PML = 1) divides exactly,
// a / 1 = a in IEEE arithmetic, so only K != 1 needs the division.
template <bool X>
__device__ __forceinline__ float DIVK(float a, float k)
{
    return k == 1.0f ? a : DIV<X>(a, k);
}

// ---------------------------------------------------------------------------
// tile location
// ---------------------------------------------------------------------------
struct TileLoc {
    int i, j0, j1;
};
__device__ __forceinline__ bool tile_of(const Inst &I, TileLoc &t)
{
    int b = blockIdx.x;
    if (b >= I.tiles) return false;
    int tx = b % I.tiles_x, tz = b / I.tiles_x;
    t.i = tx * blockDim.x + threadIdx.x + 1;
    t.j0 = tz * I.zch + 1;
    t.j1 = min(t.j0 + I.zch - 1, I.ny);
    return t.i <= I.nx;
}

// ===========================================================================
// Velocity update: update_v_PML_PSV.c:53-715 (FDORDER 2..12) + CPML on the
// stress derivatives; mode 0/2: vxp1 = rip (sxx_x + sxy_y) / DH (:451-453),
// mode 1: vxp1 += DT * vx with the old vx (:455-457).
// Each thread streams down its column; the loads of row j+1 are issued before
// row j is computed so two rows of DRAM traffic are in flight per thread.
// The register caps of the stencil kernels (velocity 40, elastic stress 64,
// viscoelastic stress 80 registers at FDORDER 8) were measured fastest of the
// caps tried (velocity 40/48/56/74, stresses 48-96): the kernels are bound by
// the loads in flight per SM, so resident warps count more than registers per
// thread (the velocity kernel spills 48 bytes at 40 and is still 4% faster).
// ===========================================================================
template <int R, bool X>
__global__ void __maxnreg__(40) k_update_v(const Inst *__restrict__ insts, const int *__restrict__ ntb, int off)
{
    const Inst &I = insts[blockIdx.y];
    if (I.pp) return;   // the fused step handles this instance
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt) return;
    TileLoc t;
    if (!tile_of(I, t)) return;
    const long long P = I.pitch;
    const int i = t.i;
    const float *__restrict__ sxx = I.sxx + i;
    const float *__restrict__ syy = I.syy + i;
    const float *__restrict__ sxy = I.sxy + i;
    const float *__restrict__ rip = I.rip + i;
    const float *__restrict__ rjp = I.rjp + i;
    float *__restrict__ vx = I.vx + i;
    float *__restrict__ vy = I.vy + i;
    float *__restrict__ vxp1 = I.vxp1 + i;
    float *__restrict__ vyp1 = I.vyp1 + i;
    float hc[R + 1];
#pragma unroll
    for (int m = 1; m <= R; m++) hc[m] = I.hc[m];
    const float DT = I.DT;
    const int mode = I.mode;
    const bool snapstep = (mode == 0) && I.store && ((nt - 1) % I.dtinv == 0);
    const int fw = I.fw, nx = I.nx, ny = I.ny, free_surf = I.free_surf;
    const bool xframe = fw > 0 && (i <= fw || i >= nx - fw + 1);

    // z windows: wyy[k] = syy[j-R+1+k], wxy[k] = sxy[j-R+k]
    float wyy[2 * R], wxy[2 * R];
#pragma unroll
    for (int k = 0; k < 2 * R - 1; k++) {
        wyy[k] = __ldg(syy + (long long)(t.j0 - R + 1 + k) * P);
        wxy[k] = __ldg(sxy + (long long)(t.j0 - R + k) * P);
    }
    // own-column operands of row j+1 are fetched before row j is computed
    // (this also brings the cache lines the x-neighbour loads of the row will hit
    // into L1); the own sxy of row j is the window's wxy[R]
    struct Ops {
        float yy, xy, sx, rip, rjp, vx, vy;
    };
    auto fetch = [&](int j) {
        const long long o = (long long)j * P;
        Ops n;
        n.yy = __ldg(syy + o + R * P);
        n.xy = __ldg(sxy + o + (R - 1) * P);
        n.sx = __ldg(sxx + o);
        n.rip = __ldg(rip + o);
        n.rjp = __ldg(rjp + o);
        n.vx = vx[o];
        n.vy = vy[o];
        return n;
    };
    Ops n1 = fetch(t.j0);
    for (int j = t.j0; j <= t.j1; j++) {
        wyy[2 * R - 1] = n1.yy;
        wxy[2 * R - 1] = n1.xy;
        const float ripv = n1.rip, rjpv = n1.rjp, vxo = n1.vx, vyo = n1.vy, csx = n1.sx, csy = wxy[R];
        if (j < t.j1) n1 = fetch(j + 1);
        // ax[k] = sxx[j][i-R+1+k], bx[k] = sxy[j][i-R+k]; the own-column entries come from the prefetch
        const float *rs = sxx + (long long)j * P;
        const float *rx = sxy + (long long)j * P;
        float ax[2 * R], bx[2 * R];
#pragma unroll
        for (int k = 0; k < 2 * R; k++) {
            ax[k] = k == R - 1 ? csx : __ldg(rs + (k - R + 1));
            bx[k] = k == R ? csy : __ldg(rx + (k - R));
        }

        float sxx_x = MUL<X>(hc[1], SUB<X>(ax[R], ax[R - 1]));
        float sxy_x = MUL<X>(hc[1], SUB<X>(bx[R], bx[R - 1]));
        float sxy_y = MUL<X>(hc[1], SUB<X>(wxy[R], wxy[R - 1]));
        float syy_y = MUL<X>(hc[1], SUB<X>(wyy[R], wyy[R - 1]));
#pragma unroll
        for (int m = 2; m <= R; m++) {
            sxx_x = ADD<X>(sxx_x, MUL<X>(hc[m], SUB<X>(ax[R - 1 + m], ax[R - m])));
            sxy_x = ADD<X>(sxy_x, MUL<X>(hc[m], SUB<X>(bx[R + m - 1], bx[R - m])));
            sxy_y = ADD<X>(sxy_y, MUL<X>(hc[m], SUB<X>(wxy[R + m - 1], wxy[R - m])));
            syy_y = ADD<X>(syy_y, MUL<X>(hc[m], SUB<X>(wyy[R - 1 + m], wyy[R - m])));
        }
        if (xframe) {
            // left frame h = i, right frame h1 = i - nx + 2 fw (BOUNDARY == 0); both apply when they overlap
            for (int side = 0; side < 2; side++) {
                if (side == 0 ? (i > fw) : (i < nx - fw + 1)) continue;
                const int h = side == 0 ? i - 1 : i - nx + 2 * fw - 1;
                float *ps = I.psi_sxx_x + (long long)(j - 1) * 2 * fw + h;
                float v = ADD<X>(MUL<X>(I.b_xh[h], *ps), MUL<X>(I.a_xh[h], sxx_x));
                *ps = v;
                sxx_x = ADD<X>(DIVK<X>(sxx_x, I.K_xh[h]), v);
                float *pq = I.psi_sxy_x + (long long)(j - 1) * 2 * fw + h;
                float w = ADD<X>(MUL<X>(I.b_x[h], *pq), MUL<X>(I.a_x[h], sxy_x));
                *pq = w;
                sxy_x = ADD<X>(DIVK<X>(sxy_x, I.K_x[h]), w);
            }
        }
        if (fw > 0 && ((!free_surf && j <= fw) || j >= ny - fw + 1)) {
            for (int side = 0; side < 2; side++) {
                if (side == 0 ? (free_surf || j > fw) : (j < ny - fw + 1)) continue;
                const int h = side == 0 ? j - 1 : j - ny + 2 * fw - 1;
                float *ps = I.psi_syy_y + (long long)h * nx + (i - 1);
                float v = ADD<X>(MUL<X>(I.b_yh[h], *ps), MUL<X>(I.a_yh[h], syy_y));
                *ps = v;
                syy_y = ADD<X>(DIVK<X>(syy_y, I.K_yh[h]), v);
                float *pq = I.psi_sxy_y + (long long)h * nx + (i - 1);
                float w = ADD<X>(MUL<X>(I.b_y[h], *pq), MUL<X>(I.a_y[h], sxy_y));
                *pq = w;
                sxy_y = ADD<X>(DIVK<X>(sxy_y, I.K_y[h]), w);
            }
        }
        const long long o = (long long)j * P;
        const float s1 = ADD<X>(sxx_x, sxy_y);
        const float s2 = ADD<X>(sxy_x, syy_y);
        if (snapstep) {
            vxp1[o] = DIVH<X>(MUL<X>(ripv, s1), I);
            vyp1[o] = DIVH<X>(MUL<X>(rjpv, s2), I);
        } else if (mode == 1) {
            vxp1[o] = ADD<X>(vxp1[o], MUL<X>(DT, vxo));
            vyp1[o] = ADD<X>(vyp1[o], MUL<X>(DT, vyo));
        }
        vx[o] = ADD<X>(vxo, DIVH<X>(MUL<X>(MUL<X>(DT, ripv), s1), I));
        vy[o] = ADD<X>(vyo, DIVH<X>(MUL<X>(MUL<X>(DT, rjpv), s2), I));
#pragma unroll
        for (int k = 0; k < 2 * R - 1; k++) {
            wyy[k] = wyy[k + 1];
            wxy[k] = wxy[k + 1];
        }
    }
}

// ===========================================================================
// Paired-column kernels: each thread owns two adjacent columns (i0, i0 + 1),
// i0 odd, and computes both with the packed FP32x2 instructions of sm_100
// (__fadd2_rn, __fmul2_rn, __ffma2_rn: per lane the same IEEE operation as
// the scalar intrinsic, so results stay bit-identical).  Fields are read as
// float2 (column i0 of the padded layout sits at an even element, so the pair
// is 8-byte aligned); an x stencil needs one pair per offset, half of which
// straddle two loaded pairs and are assembled from them.  z neighbours are
// read from L1 row by row (no register window), which keeps the kernels at
// 64 registers or fewer.  Per cell this issues roughly a third of the
// instructions of the one-column kernels above, which were bound by
// instruction issue, not by DRAM.
// ===========================================================================
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }
// The compiler contracts a packed product feeding a packed sum into one fused
// multiply-add (one rounding instead of two) although both are _rn intrinsics
// (measured on sm_100a: 1-ulp differences in the stencil sums; the scalar
// _rn intrinsics are never contracted).  An empty asm statement that takes the
// product as a 64-bit register hides it from that rewrite.
__device__ __forceinline__ float2 opaque2(float2 a)
{
    unsigned long long u = ((unsigned long long)__float_as_uint(a.y) << 32) | __float_as_uint(a.x);
    asm volatile("" : "+l"(u));
    return make_float2(__uint_as_float((unsigned)u), __uint_as_float((unsigned)(u >> 32)));
}
template <bool X> __device__ __forceinline__ float2 MUL2(float2 a, float2 b) { return opaque2(__fmul2_rn(a, b)); }
template <bool X> __device__ __forceinline__ float2 ADD2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b as a + (-b): IEEE defines subtraction as addition of the negation (same bits, signed zeros included)
template <bool X> __device__ __forceinline__ float2 SUB2(float2 a, float2 b) { return __fadd2_rn(a, neg2(b)); }
__device__ __forceinline__ float2 ld2(const float *p) { return __ldg(reinterpret_cast<const float2 *>(p)); }
__device__ __forceinline__ float2 ldw2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ void pf_l1(const float *p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }
// resident CTAs of 128 threads per SM the paired kernels are compiled for (8: 64 registers)
#ifndef DN_V2_MINB
#define DN_V2_MINB 8
#endif
#ifndef DN_S2_MINB
#define DN_S2_MINB 8
#endif
#ifndef DN_PF_ROWS
#define DN_PF_ROWS 1
#endif


// float2 store of a lane pair, or lane 0 alone for the last column of an odd nx
__device__ __forceinline__ void st2(float *p, float2 v, bool two)
{
    if (two) *reinterpret_cast<float2 *>(p) = v;
    else *p = v.x;
}

// force sources of one cell (k_inject_v, forward modes), list order
__device__ __forceinline__ void fz_force(const Inst &I, int s0, int ns, int nt, float &vx, float &vy)
{
    for (int k = 0; k < ns; k++) {
        const int l = I.src_perm[s0 + k];
        const int ty = I.src_type[l];
        const float s = I.signals[(long long)l * I.nt + (nt - 1)];
        if (ty == 2) vx = __fadd_rn(vx, s);
        if (ty == 3) vy = __fadd_rn(vy, s);
        if (ty == 4) {
            vx = F(DADD((double)vx, DMUL(I.src_nsin[l], (double)s)));
            vy = F(DADD((double)vy, DMUL(I.src_cos[l], (double)s)));
        }
    }
}

// explosive sources of one cell (k_inject_s, QUELLTYP 1), list order
__device__ __forceinline__ void fz_explosive(const Inst &I, int s0, int ns, int nt, float &sxx, float &syy)
{
    const int NT = I.nt;
    const float DT = I.DT;
    for (int k = 0; k < ns; k++) {
        const float *sg = I.signals + (long long)I.src_perm[s0 + k] * NT;
        float amp = 0.0f;
        if (nt == 1) amp = __fdiv_rn(sg[1], DT);
        if (nt > 1 && nt < NT) amp = __fdiv_rn(__fsub_rn(sg[nt], sg[nt - 2]), DT);
        if (nt == NT) amp = __fdiv_rn(-sg[nt - 2], DT);
        sxx = __fadd_rn(sxx, amp);
        syy = __fadd_rn(syy, amp);
    }
}

// whether a source cell lies in columns (i0, i0 + two) of rows j0..j1
__device__ __forceinline__ bool src_in_columns(const Inst &I, int i0, bool two, int j0, int j1)
{
    for (int c = 0; c < I.nsrc_cells; c++) {
        const int ci = I.src_cell_i[c], cj = I.src_cell_j[c];
        if (cj >= j0 && cj <= j1 && (ci == i0 || (two && ci == i0 + 1))) return true;
    }
    return false;
}

// forward sources of the source cells at row j in columns (i0, i0 + two) (fsrc_v / fsrc_s)
__device__ __forceinline__ void src_force_pair(const Inst &I, int i0, bool two, int j, int nt, float2 &vx, float2 &vy)
{
    for (int c = 0; c < I.nsrc_cells; c++) {
        const int cj = I.src_cell_j[c], ci = I.src_cell_i[c];
        if (cj != j || (ci != i0 && !(two && ci == i0 + 1))) continue;
        if (ci == i0) fz_force(I, I.src_cell_start[c], I.src_cell_count[c], nt, vx.x, vy.x);
        else fz_force(I, I.src_cell_start[c], I.src_cell_count[c], nt, vx.y, vy.y);
    }
}
__device__ __forceinline__ void src_explosive_pair(const Inst &I, int i0, bool two, int j, int nt, float2 &sxx,
                                                   float2 &syy)
{
    for (int c = 0; c < I.nsrc_cells; c++) {
        const int cj = I.src_cell_j[c], ci = I.src_cell_i[c];
        if (cj != j || (ci != i0 && !(two && ci == i0 + 1))) continue;
        if (ci == i0) fz_explosive(I, I.src_cell_start[c], I.src_cell_count[c], nt, sxx.x, syy.x);
        else fz_explosive(I, I.src_cell_start[c], I.src_cell_count[c], nt, sxx.y, syy.y);
    }
}

// division by DH of both lanes, as DIVH per lane
template <bool X>
__device__ __forceinline__ float2 DIVH2(float2 a, bool fd, float DH, float rdh)
{
    if (!X) return __fmul2_rn(a, bc2(rdh));
    if (!fd) return make_float2(__fdiv_rn(a.x, DH), __fdiv_rn(a.y, DH));
    const float2 q = __fmul2_rn(a, bc2(rdh));
    const float2 r = __ffma2_rn(neg2(q), bc2(DH), a);
    float2 q1 = __ffma2_rn(r, bc2(rdh), q);
    const float ax = fabsf(a.x), ay = fabsf(a.y);
    if (!(ax >= 0x1p-100f && ax <= 0x1p100f)) q1.x = a.x == 0.0f ? q.x : __fdiv_rn(a.x, DH);
    if (!(ay >= 0x1p-100f && ay <= 0x1p100f)) q1.y = a.y == 0.0f ? q.y : __fdiv_rn(a.y, DH);
    return q1;
}

// SRC: the variant that applies the forward sources of its cells (Inst::fsrc_v)
template <int R, bool X, bool SRC = false>
__global__ void __launch_bounds__(128, DN_V2_MINB) k_update_v2(const Inst *__restrict__ insts, const int *__restrict__ ntb, int off)
{
    const Inst &I = insts[blockIdx.y];
    if (I.pp) return;   // the fused step handles this instance
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt) return;
    const int b = blockIdx.x;
    if (b >= I.tiles) return;
    const int bxw = 2 * blockDim.x;
    const int tx = b % I.tiles_x, tz = b / I.tiles_x;
    const int i0 = tx * bxw + 2 * threadIdx.x + 1;
    if (i0 > I.nx) return;
    const int j0 = tz * I.zch + 1, j1 = min(j0 + I.zch - 1, I.ny);
    const bool two = i0 + 1 <= I.nx;
    const long long P = I.pitch;
    float hc[R + 1];
#pragma unroll
    for (int m = 1; m <= R; m++) hc[m] = I.hc[m];
    const float DT = I.DT, DH = I.DH, rdh = I.rdh;
    const bool fd = I.fastdiv;
    const int mode = I.mode;
    const bool snapstep = (mode == 0) && I.store && ((nt - 1) % I.dtinv == 0);
    const int fw = I.fw, nx = I.nx, ny = I.ny, free_surf = I.free_surf;
    const bool xframe = fw > 0 && (i0 <= fw || i0 + 1 >= nx - fw + 1);
    const bool srcs = SRC && I.fsrc_v && src_in_columns(I, i0, two, j0, j1);   // a source cell in this thread's rows
    for (int j = j0; j <= j1; j++) {
        const long long o = (long long)j * P + i0;
        // the lines row j + 1 reads first (its new z-stencil rows and its own-row operands) are
        // requested into L1 now; every address stays inside the padded planes (rows up to ny + R + 1)
        {
            constexpr int D = DN_PF_ROWS;   // rows ahead; D <= HZ - R keeps the addresses inside the planes
            pf_l1(I.syy + o + (R + D) * P);
            pf_l1(I.sxy + o + (R - 1 + D) * P);
            pf_l1(I.sxx + o + D * P);
            pf_l1(I.rip + o + D * P);
            pf_l1(I.rjp + o + D * P);
            pf_l1(I.vx + o + D * P);
            pf_l1(I.vy + o + D * P);
        }
        // sxx x stencil of lane 0: columns i0-R+1 .. i0+R (A[k], k = 0..2R); pairs (A[k], A[k+1]);
        // column i0-R+1+k is odd when k - R is odd
        float2 ax[2 * R];
        {
            const float *row = I.sxx + o - R + 1;   // A[0]
            constexpr int kb = (R % 2 == 0) ? -1 : 0;   // first aligned k
            float2 L[R + 1];
#pragma unroll
            for (int q = 0; q <= R; q++) L[q] = ld2(row + kb + 2 * q);
#pragma unroll
            for (int k = 0; k < 2 * R; k++) {
                if (((k - kb) & 1) == 0) ax[k] = L[(k - kb) / 2];
                else ax[k] = make_float2(L[(k - 1 - kb) / 2].y, L[(k + 1 - kb) / 2].x);
            }
        }
        // sxy x stencil of lane 0: columns i0-R .. i0+R-1 (B[k], k = 0..2R); column i0-R+k odd when k - R even
        float2 bx[2 * R];
        {
            const float *row = I.sxy + o - R;       // B[0]
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
        // derivatives, in the reference's term order (update_v_PML_PSV.c case 8 :366-480)
        float2 sxx_x = MUL2<X>(bc2(hc[1]), SUB2<X>(ax[R], ax[R - 1]));
        float2 sxy_x = MUL2<X>(bc2(hc[1]), SUB2<X>(bx[R], bx[R - 1]));
        float2 sxy_y = MUL2<X>(bc2(hc[1]), SUB2<X>(ld2(I.sxy + o), ld2(I.sxy + o - P)));
        float2 syy_y = MUL2<X>(bc2(hc[1]), SUB2<X>(ld2(I.syy + o + P), ld2(I.syy + o)));
#pragma unroll
        for (int m = 2; m <= R; m++) {
            sxx_x = ADD2<X>(sxx_x, MUL2<X>(bc2(hc[m]), SUB2<X>(ax[R - 1 + m], ax[R - m])));
            sxy_x = ADD2<X>(sxy_x, MUL2<X>(bc2(hc[m]), SUB2<X>(bx[R + m - 1], bx[R - m])));
            sxy_y = ADD2<X>(sxy_y, MUL2<X>(bc2(hc[m]), SUB2<X>(ld2(I.sxy + o + (m - 1) * P), ld2(I.sxy + o - m * P))));
            syy_y = ADD2<X>(syy_y, MUL2<X>(bc2(hc[m]), SUB2<X>(ld2(I.syy + o + m * P), ld2(I.syy + o - (m - 1) * P))));
        }

        if (xframe) {
            // per lane: left frame h = i, right frame h1 = i - nx + 2 fw (both when they overlap)
            float *sx = &sxx_x.x, *sy = &sxy_x.x;
            for (int lane = 0; lane < 2; lane++) {
                const int i = i0 + lane;
                if (i > nx || !(i <= fw || i >= nx - fw + 1)) continue;
                for (int side = 0; side < 2; side++) {
                    if (side == 0 ? (i > fw) : (i < nx - fw + 1)) continue;
                    const int h = side == 0 ? i - 1 : i - nx + 2 * fw - 1;
                    float *ps = I.psi_sxx_x + (long long)(j - 1) * 2 * fw + h;
                    float v = ADD<X>(MUL<X>(I.b_xh[h], *ps), MUL<X>(I.a_xh[h], sx[lane]));
                    *ps = v;
                    sx[lane] = ADD<X>(DIVK<X>(sx[lane], I.K_xh[h]), v);
                    float *pq = I.psi_sxy_x + (long long)(j - 1) * 2 * fw + h;
                    float w = ADD<X>(MUL<X>(I.b_x[h], *pq), MUL<X>(I.a_x[h], sy[lane]));
                    *pq = w;
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
                    float *ps = I.psi_syy_y + (long long)h * nx + (i - 1);
                    float v = ADD<X>(MUL<X>(I.b_yh[h], *ps), MUL<X>(I.a_yh[h], sy[lane]));
                    *ps = v;
                    sy[lane] = ADD<X>(DIVK<X>(sy[lane], I.K_yh[h]), v);
                    float *pq = I.psi_sxy_y + (long long)h * nx + (i - 1);
                    float w = ADD<X>(MUL<X>(I.b_y[h], *pq), MUL<X>(I.a_y[h], sx[lane]));
                    *pq = w;
                    sx[lane] = ADD<X>(DIVK<X>(sx[lane], I.K_y[h]), w);
                }
            }
        }
        const float2 ripv = ld2(I.rip + o), rjpv = ld2(I.rjp + o);
        const float2 vxo = ldw2(I.vx + o), vyo = ldw2(I.vy + o);
        const float2 s1 = ADD2<X>(sxx_x, sxy_y);
        const float2 s2 = ADD2<X>(sxy_x, syy_y);
        float2 nvx = ADD2<X>(vxo, DIVH2<X>(MUL2<X>(MUL2<X>(bc2(DT), ripv), s1), fd, DH, rdh));
        float2 nvy = ADD2<X>(vyo, DIVH2<X>(MUL2<X>(MUL2<X>(bc2(DT), rjpv), s2), fd, DH, rdh));
        if (srcs) src_force_pair(I, i0, two, j, nt, nvx, nvy);
        float2 p1x, p1y;
        const bool wp = snapstep || mode == 1;
        if (snapstep) {
            p1x = DIVH2<X>(MUL2<X>(ripv, s1), fd, DH, rdh);
            p1y = DIVH2<X>(MUL2<X>(rjpv, s2), fd, DH, rdh);
        } else if (mode == 1) {
            p1x = ADD2<X>(ldw2(I.vxp1 + o), MUL2<X>(bc2(DT), vxo));
            p1y = ADD2<X>(ldw2(I.vyp1 + o), MUL2<X>(bc2(DT), vyo));
        }
        if (two) {
            *reinterpret_cast<float2 *>(I.vx + o) = nvx;
            *reinterpret_cast<float2 *>(I.vy + o) = nvy;
            if (wp) {
                *reinterpret_cast<float2 *>(I.vxp1 + o) = p1x;
                *reinterpret_cast<float2 *>(I.vyp1 + o) = p1y;
            }
        } else {   // the last column of an odd nx: column nx + 1 is halo and stays zero
            I.vx[o] = nvx.x;
            I.vy[o] = nvy.x;
            if (wp) {
                I.vxp1[o] = p1x.x;
                I.vyp1[o] = p1y.x;
            }
        }
    }
}

// ===========================================================================
// Force sources (update_v_PML_PSV.c:738-752) and adjoint residual forces
// (:755-768).  One thread per unique source cell; sources sharing a cell are
// added in their list order, as the reference's sequential loop does.
// ===========================================================================
static __global__ void k_inject_v(const Inst *__restrict__ insts, const int *__restrict__ ntb, int off)
{
    const Inst &I = insts[blockIdx.y];
    if (I.pp) return;   // the fused step handles this instance
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt) return;
    const long long P = I.pitch;
    if (I.mode == 1) {
        const int q = I.quelltypb;
        // receivers that share a cell add their forces one after the other in list order, as
        // the reference's loop does (update_v_PML_PSV.c:755-768): one thread for them all
        const int l0 = I.rec_dup ? (blockIdx.x == 0 && threadIdx.x == 0 ? 0 : I.ntr) : blockIdx.x * blockDim.x + threadIdx.x;
        const int dl = I.rec_dup ? 1 : gridDim.x * blockDim.x;
        for (int l = l0; l < I.ntr; l += dl) {
            const long long o = (long long)I.rec_j[l] * P + I.rec_i[l];
            const long long s = (long long)l * I.nt + (nt - 1);
            if (q == 1) {
                I.vx[o] = __fadd_rn(I.vx[o], I.res_vx[s]);
                I.vy[o] = __fadd_rn(I.vy[o], I.res_vy[s]);
            }
            if (q == 2 || q == 6 || q == 7) I.vy[o] = __fadd_rn(I.vy[o], I.res_vy[s]);
            if (q == 3 || q == 5 || q == 7) I.vx[o] = __fadd_rn(I.vx[o], I.res_vx[s]);
        }
        return;
    }
    if (I.fsrc_v) return;   // applied by the velocity kernel
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < I.nsrc_cells; c += gridDim.x * blockDim.x) {
        const long long o = (long long)I.src_cell_j[c] * P + I.src_cell_i[c];
        float vx = I.vx[o], vy = I.vy[o];
        const int s0 = I.src_cell_start[c], ns = I.src_cell_count[c];
        for (int k = 0; k < ns; k++) {
            const int l = I.src_perm[s0 + k];
            const int ty = I.src_type[l];
            const float s = I.signals[(long long)l * I.nt + (nt - 1)];
            if (ty == 2) vx = __fadd_rn(vx, s);
            if (ty == 3) vy = __fadd_rn(vy, s);
            if (ty == 4) {
                vx = F(DADD((double)vx, DMUL(I.src_nsin[l], (double)s)));
                vy = F(DADD((double)vy, DMUL(I.src_cos[l], (double)s)));
            }
        }
        I.vx[o] = vx;
        I.vy[o] = vy;
    }
}

// ===========================================================================
// Stress derivatives shared by the elastic and viscoelastic updates:
// vxx, vyx, vxy, vyy of update_s_*_PML_PSV.c (case 8 = :366-384 elastic),
// multiplied by dhi, followed by the CPML correction (:386-438).
// The operands of row j+1 are fetched before row j is computed.
// ===========================================================================
template <int R, bool X>
struct VDeriv {
    const float *__restrict__ vx;   // column i
    const float *__restrict__ vy;
    long long P;
    float wx[2 * R];                // vx rows j-R+1 .. j+R (vx[j] = wx[R-1])
    float wy[2 * R];                // vy rows j-R .. j+R-1 (vy[j] = wy[R])
    float cx[2 * R], dx[2 * R];     // cx[k] = vx[j][i-R+k], dx[k] = vy[j][i-R+1+k]
    float nwx, nwy;

    __device__ __forceinline__ void fetch(int j)
    {
        const long long o = (long long)j * P;
        nwx = __ldg(vx + o + R * P);
        nwy = __ldg(vy + o + (R - 1) * P);
    }
    __device__ __forceinline__ void prime(const Inst &I, int i, int j0)
    {
        vx = I.vx + i;
        vy = I.vy + i;
        P = I.pitch;
#pragma unroll
        for (int k = 0; k < 2 * R - 1; k++) {
            wx[k] = __ldg(vx + (long long)(j0 - R + 1 + k) * P);
            wy[k] = __ldg(vy + (long long)(j0 - R + k) * P);
        }
        fetch(j0);
    }
    // makes row j current: completes the windows and reads the row's x-neighbours (L1)
    __device__ __forceinline__ void advance(int j)
    {
        wx[2 * R - 1] = nwx;
        wy[2 * R - 1] = nwy;
        const long long o = (long long)j * P;
#pragma unroll
        for (int k = 0; k < 2 * R; k++) {
            cx[k] = k == R ? wx[R - 1] : __ldg(vx + o + (k - R));
            dx[k] = k == R - 1 ? wy[R] : __ldg(vy + o + (k - R + 1));
        }
    }
    __device__ __forceinline__ void shift()
    {
#pragma unroll
        for (int k = 0; k < 2 * R - 1; k++) {
            wx[k] = wx[k + 1];
            wy[k] = wy[k + 1];
        }
    }
    __device__ __forceinline__ void compute(const Inst &I, const float *hc, int i, int j, float dhi, float &vxx,
                                            float &vyx, float &vxy, float &vyy)
    {
        float a = MUL<X>(hc[1], SUB<X>(cx[R], cx[R - 1]));
        float b = MUL<X>(hc[1], SUB<X>(dx[R], dx[R - 1]));
        float c = MUL<X>(hc[1], SUB<X>(wx[R], wx[R - 1]));
        float d = MUL<X>(hc[1], SUB<X>(wy[R], wy[R - 1]));
#pragma unroll
        for (int m = 2; m <= R; m++) {
            a = ADD<X>(a, MUL<X>(hc[m], SUB<X>(cx[R + m - 1], cx[R - m])));
            b = ADD<X>(b, MUL<X>(hc[m], SUB<X>(dx[R - 1 + m], dx[R - m])));
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
                vxx = ADD<X>(DIVK<X>(vxx, I.K_x[h]), v);
                float *p2 = I.psi_vyx + (long long)(j - 1) * 2 * fw + h;
                float w = ADD<X>(MUL<X>(I.b_xh[h], *p2), MUL<X>(I.a_xh[h], vyx));
                *p2 = w;
                vyx = ADD<X>(DIVK<X>(vyx, I.K_xh[h]), w);
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
                vyy = ADD<X>(DIVK<X>(vyy, I.K_y[h]), v);
                vxy = ADD<X>(DIVK<X>(vxy, I.K_yh[h]), w);
            }
        }
    }
};

// ===========================================================================
// Elastic stress update: update_s_elastic_PML_PSV.c (case 8 = :335-476),
// with f = rho vs^2 and g = rho (vp^2 - 2 vs^2) precomputed per cell
// (:442-444) and the double-promoted 2.0*f*vxx terms (:454-456).
// ===========================================================================
template <int R, bool X>
__global__ void __launch_bounds__(256, 4) k_update_s_el(const Inst *__restrict__ insts, const int *__restrict__ ntb, int off)
{
    const Inst &I = insts[blockIdx.y];
    if (I.pp) return;   // the fused step handles this instance
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt) return;
    TileLoc t;
    if (!tile_of(I, t)) return;
    const long long P = I.pitch;
    const int i = t.i;
    float hc[R + 1];
#pragma unroll
    for (int m = 1; m <= R; m++) hc[m] = I.hc[m];
    const float dhi = I.dhi_el;
    const float *__restrict__ uipjp = I.uipjp + i;
    const float *__restrict__ mu = I.mu + i;
    const float *__restrict__ lam = I.lam + i;
    float *__restrict__ sxx = I.sxx + i;
    float *__restrict__ syy = I.syy + i;
    float *__restrict__ sxy = I.sxy + i;
    VDeriv<R, X> D;
    D.prime(I, i, t.j0);
    float nfip, nf, ng, nsxx, nsyy, nsxy;
    auto fetch = [&](int j) {
        const long long o = (long long)j * P;
        nfip = __ldg(uipjp + o);
        nf = __ldg(mu + o);
        ng = __ldg(lam + o);
        nsxx = sxx[o];
        nsyy = syy[o];
        nsxy = sxy[o];
    };
    fetch(t.j0);
    for (int j = t.j0; j <= t.j1; j++) {
        D.advance(j);
        const float fipjp = nfip, f = nf, g = ng, s_xx = nsxx, s_yy = nsyy, s_xy = nsxy;
        if (j < t.j1) {
            D.fetch(j + 1);
            fetch(j + 1);
        }
        float vxx, vyx, vxy, vyy;
        D.compute(I, hc, i, j, dhi, vxx, vyx, vxy, vyy);
        const long long o = (long long)j * P;
        const float div = ADD<X>(vxx, vyy);
        const float gdiv = MUL<X>(g, div);
        const double f2 = 2.0 * (double)f;
        sxy[o] = ADD<X>(s_xy, MUL<X>(fipjp, ADD<X>(vyx, vxy)));
        sxx[o] = F(DADD((double)s_xx, DADD((double)gdiv, DMUL(f2, (double)vxx))));
        syy[o] = F(DADD((double)s_yy, DADD((double)gdiv, DMUL(f2, (double)vyy))));
        D.shift();
    }
}

// ===========================================================================
// Paired-column stress derivatives: vxx, vyx, vxy, vyy of update_s_*_PML_PSV.c
// for columns (i0, i0 + 1), times dhi, then the CPML correction per lane
// (the scalar VDeriv::compute, two lanes at a time).
// ===========================================================================
template <int R, bool X>
__device__ __forceinline__ void vderiv2(const Inst &I, const float *hc, int i0, int j, long long o, long long P,
                                        float dhi, float2 &vxx, float2 &vyx, float2 &vxy, float2 &vyy)
{
    // vx x stencil of lane 0: columns i0-R .. i0+R-1 (C[k]); column i0-R+k odd when k - R is even
    float2 cx[2 * R], dx[2 * R];
    {
        const float *row = I.vx + o - R;
        constexpr int kb = (R % 2 == 0) ? 0 : -1;
        float2 L[R + 1];
#pragma unroll
        for (int q = 0; q <= R; q++) L[q] = ldw2(row + kb + 2 * q);
#pragma unroll
        for (int k = 0; k < 2 * R; k++) {
            if (((k - kb) & 1) == 0) cx[k] = L[(k - kb) / 2];
            else cx[k] = make_float2(L[(k - 1 - kb) / 2].y, L[(k + 1 - kb) / 2].x);
        }
    }
    // vy x stencil of lane 0: columns i0-R+1 .. i0+R (D[k]); column i0-R+1+k odd when k - R is odd
    {
        const float *row = I.vy + o - R + 1;
        constexpr int kb = (R % 2 == 0) ? -1 : 0;
        float2 L[R + 1];
#pragma unroll
        for (int q = 0; q <= R; q++) L[q] = ldw2(row + kb + 2 * q);
#pragma unroll
        for (int k = 0; k < 2 * R; k++) {
            if (((k - kb) & 1) == 0) dx[k] = L[(k - kb) / 2];
            else dx[k] = make_float2(L[(k - 1 - kb) / 2].y, L[(k + 1 - kb) / 2].x);
        }
    }
    float2 a = MUL2<X>(bc2(hc[1]), SUB2<X>(cx[R], cx[R - 1]));
    float2 b = MUL2<X>(bc2(hc[1]), SUB2<X>(dx[R], dx[R - 1]));
    float2 c = MUL2<X>(bc2(hc[1]), SUB2<X>(ldw2(I.vx + o + P), ldw2(I.vx + o)));
    float2 d = MUL2<X>(bc2(hc[1]), SUB2<X>(ldw2(I.vy + o), ldw2(I.vy + o - P)));
#pragma unroll
    for (int m = 2; m <= R; m++) {
        a = ADD2<X>(a, MUL2<X>(bc2(hc[m]), SUB2<X>(cx[R + m - 1], cx[R - m])));
        b = ADD2<X>(b, MUL2<X>(bc2(hc[m]), SUB2<X>(dx[R - 1 + m], dx[R - m])));
        c = ADD2<X>(c, MUL2<X>(bc2(hc[m]), SUB2<X>(ldw2(I.vx + o + m * P), ldw2(I.vx + o - (m - 1) * P))));
        d = ADD2<X>(d, MUL2<X>(bc2(hc[m]), SUB2<X>(ldw2(I.vy + o + (m - 1) * P), ldw2(I.vy + o - m * P))));
    }
    vxx = MUL2<X>(a, bc2(dhi));
    vyx = MUL2<X>(b, bc2(dhi));
    vxy = MUL2<X>(c, bc2(dhi));
    vyy = MUL2<X>(d, bc2(dhi));
    const int fw = I.fw, nx = I.nx, ny = I.ny;
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
}


// Paired-column elastic stress update (k_update_s_el for two columns per thread).
template <int R, bool X, bool SRC = false>
__global__ void __launch_bounds__(128, DN_S2_MINB) k_update_s_el2(const Inst *__restrict__ insts, const int *__restrict__ ntb, int off)
{
    const Inst &I = insts[blockIdx.y];
    if (I.pp) return;   // the fused step handles this instance
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt) return;
    const int b = blockIdx.x;
    if (b >= I.tiles) return;
    const int bxw = 2 * blockDim.x;
    const int tx = b % I.tiles_x, tz = b / I.tiles_x;
    const int i0 = tx * bxw + 2 * threadIdx.x + 1;
    if (i0 > I.nx) return;
    const int j0 = tz * I.zch + 1, j1 = min(j0 + I.zch - 1, I.ny);
    const bool two = i0 + 1 <= I.nx;
    const long long P = I.pitch;
    float hc[R + 1];
#pragma unroll
    for (int m = 1; m <= R; m++) hc[m] = I.hc[m];
    const float dhi = I.dhi_el;
    const bool srcs = SRC && I.fsrc_s && src_in_columns(I, i0, two, j0, j1);
    for (int j = j0; j <= j1; j++) {
        const long long o = (long long)j * P + i0;
        {
            constexpr int D = DN_PF_ROWS;
            pf_l1(I.vx + o + (R + D) * P);
            pf_l1(I.vy + o + (R - 1 + D) * P);
            pf_l1(I.uipjp + o + D * P);
            pf_l1(I.mu + o + D * P);
            pf_l1(I.lam + o + D * P);
            pf_l1(I.sxx + o + D * P);
            pf_l1(I.syy + o + D * P);
            pf_l1(I.sxy + o + D * P);
        }
        float2 vxx, vyx, vxy, vyy;
        vderiv2<R, X>(I, hc, i0, j, o, P, dhi, vxx, vyx, vxy, vyy);
        const float2 fipjp = ld2(I.uipjp + o), f = ld2(I.mu + o), g = ld2(I.lam + o);
        const float2 s_xx = ldw2(I.sxx + o), s_yy = ldw2(I.syy + o), s_xy = ldw2(I.sxy + o);
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
        if (srcs) src_explosive_pair(I, i0, two, j, nt, nsxx, nsyy);
        st2(I.sxy + o, nsxy, two);
        st2(I.sxx + o, nsxx, two);
        st2(I.syy + o, nsyy, two);
    }
}

// ===========================================================================
// Viscoelastic stress update: update_s_visc_PML_PSV.c (case 8 = :391-511).
// fipjp, f, g, dip, d, e are regenerated per cell from the six relaxed-modulus
// factors exactly as prepare_update_s_visc_PSV.c:52-62 forms them; the PRE
// variant reads them prepared (Inst::pre_*), as the reference function takes them.
// ===========================================================================
template <int R, int L, bool X, bool SRC = false, bool PRE = false>
__global__ void __launch_bounds__(256, 3) k_update_s_vi(const Inst *__restrict__ insts, const int *__restrict__ ntb, int off)
{
    const Inst &I = insts[blockIdx.y];
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt) return;
    TileLoc t;
    if (!tile_of(I, t)) return;
    const long long P = I.pitch;
    const long long PL = I.plane;
    const int i = t.i;
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
    const float *__restrict__ c_muipjp = I.c_muipjp + i;
    const float *__restrict__ c_tausipjp = I.c_tausipjp + i;
    const float *__restrict__ c_mu = I.c_mu + i;
    const float *__restrict__ c_taus = I.c_taus + i;
    const float *__restrict__ c_pi = I.c_pi + i;
    const float *__restrict__ c_taup = I.c_taup + i;
    float *__restrict__ sxxp = I.sxx + i;
    float *__restrict__ syyp = I.syy + i;
    float *__restrict__ sxyp = I.sxy + i;
    float *__restrict__ rp = I.r + i;
    float *__restrict__ pp_ = I.p + i;
    float *__restrict__ qp = I.q + i;
    VDeriv<R, X> D;
    D.prime(I, i, t.j0);
    float nm[6], ns[3], nr[L], np_[L], nq[L];
    float npre[PRE ? 3 * L : 1];
    auto fetch = [&](int j) {
        const long long o = (long long)j * P;
        if constexpr (PRE) {   // nm[0..2]: the prepared fipjp, f, g
            nm[3] = nm[4] = nm[5] = 0.0f;
            nm[0] = __ldg(I.pre_fipjp + i + o);
            nm[1] = __ldg(I.pre_f + i + o);
            nm[2] = __ldg(I.pre_g + i + o);
#pragma unroll
            for (int l = 0; l < L; l++) {
                npre[l] = __ldg(I.pre_dip + i + o + l * PL);
                npre[L + l] = __ldg(I.pre_d + i + o + l * PL);
                npre[2 * L + l] = __ldg(I.pre_e + i + o + l * PL);
            }
        } else {
            nm[0] = __ldg(c_muipjp + o);
            nm[1] = __ldg(c_tausipjp + o);
            nm[2] = __ldg(c_mu + o);
            nm[3] = __ldg(c_taus + o);
            nm[4] = __ldg(c_pi + o);
            nm[5] = __ldg(c_taup + o);
        }
        ns[0] = sxxp[o];
        ns[1] = syyp[o];
        ns[2] = sxyp[o];
#pragma unroll
        for (int l = 0; l < L; l++) {
            nr[l] = rp[o + l * PL];
            np_[l] = pp_[o + l * PL];
            nq[l] = qp[o + l * PL];
        }
    };
    const bool srcs = SRC && I.fsrc_s && src_in_columns(I, i, false, t.j0, t.j1);
    fetch(t.j0);
    for (int j = t.j0; j <= t.j1; j++) {
        D.advance(j);
        const float muipjp = nm[0], tsij = nm[1], mu = nm[2], taus = nm[3], pi = nm[4], taup = nm[5];
        const float s_xx = ns[0], s_yy = ns[1], s_xy = ns[2];
        float rr[L], pp[L], qq[L];
        float pre[PRE ? 3 * L : 1];
#pragma unroll
        for (int l = 0; l < L; l++) {
            rr[l] = nr[l];
            pp[l] = np_[l];
            qq[l] = nq[l];
        }
        if constexpr (PRE) {
#pragma unroll
            for (int k = 0; k < 3 * L; k++) pre[k] = npre[k];
        }
        if (j < t.j1) {
            D.fetch(j + 1);
            fetch(j + 1);
        }
        float vxx, vyx, vxy, vyy;
        D.compute(I, hc, i, j, dhi, vxx, vyx, vxy, vyy);
        const long long o = (long long)j * P;
        const float fipjp = PRE ? muipjp : F(DMUL((double)__fmul_rn(muipjp, DT), DADD(1.0, (double)__fmul_rn(fL, tsij))));
        const float f = PRE ? tsij : F(DMUL((double)__fmul_rn(mu, DT), DADD(1.0, (double)__fmul_rn(fL, taus))));
        const float g = PRE ? mu : F(DMUL((double)__fmul_rn(pi, DT), DADD(1.0, (double)__fmul_rn(fL, taup))));
        float sumr = 0.0f, sump = 0.0f, sumq = 0.0f;
#pragma unroll
        for (int l = 0; l < L; l++) {
            sumr = ADD<X>(sumr, rr[l]);
            sump = ADD<X>(sump, pp[l]);
            sumq = ADD<X>(sumq, qq[l]);
        }
        const float sh = ADD<X>(vxy, vyx);
        const float dv = ADD<X>(vxx, vyy);
        const float gdv = MUL<X>(g, dv);
        const double f2 = 2.0 * (double)f;
        float sxy = ADD<X>(s_xy, ADD<X>(MUL<X>(fipjp, sh), MUL<X>(dthalbe, sumr)));
        float sxx = F(DADD((double)s_xx, DADD(DSUB((double)gdv, DMUL(f2, (double)vyy)), (double)MUL<X>(dthalbe, sump))));
        float syy = F(DADD((double)s_yy, DADD(DSUB((double)gdv, DMUL(f2, (double)vxx)), (double)MUL<X>(dthalbe, sumq))));
        sumr = sump = sumq = 0.0f;
#pragma unroll
        for (int l = 0; l < L; l++) {
            const float dip = PRE ? pre[l] : MUL<X>(MUL<X>(muipjp, eta[l]), tsij);
            const float dd = PRE ? pre[L + l] : MUL<X>(MUL<X>(mu, eta[l]), taus);
            const float ee = PRE ? pre[2 * L + l] : MUL<X>(MUL<X>(pi, eta[l]), taup);
            const float r = MUL<X>(bip[l], SUB<X>(MUL<X>(rr[l], cip[l]), MUL<X>(dip, sh)));
            const double d2 = 2.0 * (double)dd;
            const float pv = F(DMUL((double)bip[l], DADD((double)SUB<X>(MUL<X>(pp[l], cip[l]), MUL<X>(ee, dv)), DMUL(d2, (double)vyy))));
            const float qv = F(DMUL((double)bip[l], DADD((double)SUB<X>(MUL<X>(qq[l], cip[l]), MUL<X>(ee, dv)), DMUL(d2, (double)vxx))));
            rp[o + l * PL] = r;
            pp_[o + l * PL] = pv;
            qp[o + l * PL] = qv;
            sumr = ADD<X>(sumr, r);
            sump = ADD<X>(sump, pv);
            sumq = ADD<X>(sumq, qv);
        }
        sxyp[o] = ADD<X>(sxy, MUL<X>(dthalbe, sumr));
        float fsxx = ADD<X>(sxx, MUL<X>(dthalbe, sump)), fsyy = ADD<X>(syy, MUL<X>(dthalbe, sumq));
        if (srcs)
            for (int c = 0; c < I.nsrc_cells; c++)
                if (I.src_cell_j[c] == j && I.src_cell_i[c] == i)
                    fz_explosive(I, I.src_cell_start[c], I.src_cell_count[c], nt, fsxx, fsyy);
        sxxp[o] = fsxx;
        syyp[o] = fsyy;
        D.shift();
    }
}

// ===========================================================================
// Explosive source psource.c:23-39 (mode 0/2 when QUELLTYP == 1), adjoint
// pressure source psource.c:41-53 (mode 1, QUELLTYPB >= 4) and the moment
// tensor source msource.c:27-41 (QUELLTYP == 5, forward modes).
// ===========================================================================
static __global__ void k_inject_s(const Inst *__restrict__ insts, const int *__restrict__ ntb, int off)
{
    const Inst &I = insts[blockIdx.y];
    if (I.pp) return;   // the fused step handles this instance
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt) return;
    const long long P = I.pitch;
    if (I.mode == 1) {
        if (I.quelltypb < 4) return;
        // receivers sharing a cell: one thread, list order (psource.c:41-53)
        const int l0 = I.rec_dup ? (blockIdx.x == 0 && threadIdx.x == 0 ? 0 : I.ntr) : blockIdx.x * blockDim.x + threadIdx.x;
        const int dl = I.rec_dup ? 1 : gridDim.x * blockDim.x;
        for (int l = l0; l < I.ntr; l += dl) {
            const long long o = (long long)I.rec_j[l] * P + I.rec_i[l];
            const float s = I.res_p[(long long)l * I.nt + (nt - 1)];
            I.sxx[o] = __fadd_rn(I.sxx[o], s);
            I.syy[o] = __fadd_rn(I.syy[o], s);
        }
        return;
    }
    const int NT = I.nt;
    const float DT = I.DT;
    if (I.quelltyp_last == 1 && !I.fsrc_s) {   // fsrc_s: applied by the stress kernel
        for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < I.nsrc_cells; c += gridDim.x * blockDim.x) {
            const long long o = (long long)I.src_cell_j[c] * P + I.src_cell_i[c];
            float sxx = I.sxx[o], syy = I.syy[o];
            const int s0 = I.src_cell_start[c], ns = I.src_cell_count[c];
            for (int k = 0; k < ns; k++) {
                const float *sg = I.signals + (long long)I.src_perm[s0 + k] * NT;   // sg[n-1] = signals[l][n]
                float amp = 0.0f;
                if (nt == 1) amp = __fdiv_rn(sg[1], DT);
                if (nt > 1 && nt < NT) amp = __fdiv_rn(__fsub_rn(sg[nt], sg[nt - 2]), DT);
                if (nt == NT) amp = __fdiv_rn(-sg[nt - 2], DT);
                sxx = __fadd_rn(sxx, amp);
                syy = __fadd_rn(syy, amp);
            }
            I.sxx[o] = sxx;
            I.syy[o] = syy;
        }
    } else if (I.quelltyp_last == 5) {
        // neighbouring moment-tensor sources touch overlapping cells: one thread, list order
        if (blockIdx.x != 0 || threadIdx.x != 0) return;
        for (int cidx = 0; cidx < I.nsrc_cells; cidx++) {
            const int s0 = I.src_cell_start[cidx], ns = I.src_cell_count[cidx];
            for (int k = 0; k < ns; k++) {
                const int l = I.src_perm[s0 + k];
                const int si = I.src_cell_i[cidx], sj = I.src_cell_j[cidx];
                const float *sg = I.signals + (long long)l * NT;
                float amp = 0.0f;
                if (nt == 1) amp = __fdiv_rn(sg[1], DT);
                if (nt > 1 && nt < NT) amp = __fdiv_rn(__fsub_rn(sg[nt], sg[nt - 2]), DT);
                if (nt == NT) amp = __fdiv_rn(-sg[nt - 2], DT);
                const long long o = (long long)sj * P + si;
                I.sxx[o] = __fadd_rn(I.sxx[o], __fmul_rn(amp, 0.0f));
                I.syy[o] = __fadd_rn(I.syy[o], __fmul_rn(amp, 0.0f));
                const double a4 = DMUL(DMUL(0.25, (double)amp), 1.0);
                const long long o2[4] = {o, o - 1, o - P, o - P - 1};
                for (int z = 0; z < 4; z++) I.sxy[o2[z]] = F(DADD((double)I.sxy[o2[z]], a4));
            }
        }
    }
}

// ===========================================================================
// Free surface at row j = 1 (image method), surface_elastic_PML_PSV.c:29-103.
// ===========================================================================
template <int R, bool X>
__global__ void k_surface_el(const Inst *__restrict__ insts, const int *__restrict__ ntb, int off)
{
    const Inst &I = insts[blockIdx.y];
    if (I.pp) return;   // the fused step handles this instance
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt || !I.free_surf) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (i > I.nx) return;
    const long long P = I.pitch;
    const int j = 1;
    const long long o = (long long)j * P + i;
    I.syy[o] = 0.0f;
    float vxx = 0.0f, vyy = 0.0f;
#pragma unroll
    for (int m = 1; m <= R; m++) {
        I.syy[o - m * P] = -I.syy[o + m * P];
        I.sxy[o - m * P] = -I.sxy[o + (m - 1) * P];
        vxx = ADD<X>(vxx, MUL<X>(I.hc[m], SUB<X>(I.vx[o + m - 1], I.vx[o - m])));
        vyy = ADD<X>(vyy, MUL<X>(I.hc[m], SUB<X>(I.vy[o + (m - 1) * P], I.vy[o - m * P])));
    }
    vxx = MUL<X>(vxx, I.dh1);
    vyy = MUL<X>(vyy, I.dh1);
    const int fw = I.fw, nx = I.nx;
    if (fw > 0) {
        if (i <= fw) {
            const int h = i - 1;
            float *ps = I.psi_vxxs + (long long)(j - 1) * 2 * fw + h;
            float v = ADD<X>(MUL<X>(I.b_x[h], *ps), MUL<X>(I.a_x[h], vxx));
            *ps = v;
            vxx = ADD<X>(DIVK<X>(vxx, I.K_x[h]), v);
        }
        if (i >= nx - fw + 1) {
            const int h = i - nx + 2 * fw - 1;
            float *ps = I.psi_vxxs + (long long)(j - 1) * 2 * fw + h;
            float v = ADD<X>(MUL<X>(I.b_x[h], *ps), MUL<X>(I.a_x[h], vxx));
            *ps = v;
            vxx = ADD<X>(DIVK<X>(vxx, I.K_x[h]), v);
        }
    }
    const float g = I.lam[o];
    const float fjm = MUL<X>(I.mu[o], 2.0f);   // rho*u*u*2.0 (exact doubling)
    const float t1 = MUL<X>(DIV<X>(MUL<X>(g, g), ADD<X>(g, fjm)), vxx);
    const float t2 = MUL<X>(g, vyy);
    I.sxx[o] = ADD<X>(I.sxx[o], MUL<X>(-I.DT, ADD<X>(t1, t2)));
}

// ===========================================================================
// Viscoelastic free surface, surface_visc_PML_PSV.c:60-170 (relaxed moduli
// from ws = 2 pi / TS, per-column constants precomputed on the host).
// ===========================================================================
template <int R, int L, bool X>
__global__ void k_surface_vi(const Inst *__restrict__ insts, const int *__restrict__ ntb, int off)
{
    const Inst &I = insts[blockIdx.y];
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt || !I.free_surf) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (i > I.nx) return;
    const long long P = I.pitch;
    const int j = 1;
    const long long o = (long long)j * P + i;
    I.syy[o] = 0.0f;
#pragma unroll
    for (int l = 0; l < L; l++) I.q[o + l * I.plane] = 0.0f;
    float vxx = 0.0f, vyy = 0.0f;
#pragma unroll
    for (int m = 1; m <= R; m++) {
        I.syy[o - m * P] = -I.syy[o + m * P];
        I.sxy[o - m * P] = -I.sxy[o + (m - 1) * P];
        vxx = ADD<X>(vxx, MUL<X>(I.hc[m], SUB<X>(I.vx[o + m - 1], I.vx[o - m])));
        vyy = ADD<X>(vyy, MUL<X>(I.hc[m], SUB<X>(I.vy[o + (m - 1) * P], I.vy[o - m * P])));
    }
    vxx = MUL<X>(vxx, I.dh1);
    vyy = MUL<X>(vyy, I.dh1);
    const int fw = I.fw, nx = I.nx;
    if (fw > 0) {
        if (i <= fw) {
            const int h = i - 1;
            float *ps = I.psi_vxxs + (long long)(j - 1) * 2 * fw + h;
            float v = ADD<X>(MUL<X>(I.b_x[h], *ps), MUL<X>(I.a_x[h], vxx));
            *ps = v;
            vxx = ADD<X>(DIVK<X>(vxx, I.K_x[h]), v);
        }
        if (i >= nx - fw + 1) {
            const int h = i - nx + 2 * fw - 1;
            float *ps = I.psi_vxxs + (long long)(j - 1) * 2 * fw + h;
            float v = ADD<X>(MUL<X>(I.b_x[h], *ps), MUL<X>(I.a_x[h], vxx));
            *ps = v;
            vxx = ADD<X>(DIVK<X>(vxx, I.K_x[h]), v);
        }
    }
    const float mu = I.s_mu[i - 1], pi = I.s_pi[i - 1], taus = I.s_taus[i - 1], taup = I.s_taup[i - 1];
    const float DT = I.DT, dthalbe = I.dthalbe;
    const float fL = (float)L;
    float sump = 0.0f;
#pragma unroll
    for (int l = 0; l < L; l++) sump = ADD<X>(sump, I.p[o + l * I.plane]);
    const float fjm = F(DMUL(DMUL((double)mu, 2.0), DADD(1.0, (double)MUL<X>(fL, taus))));
    const float g = F(DMUL((double)pi, DADD(1.0, (double)MUL<X>(fL, taup))));
    const float gf = SUB<X>(g, fjm);
    const float DTgf = MUL<X>(DT, gf);
    float a = -DIV<X>(MUL<X>(MUL<X>(DTgf, gf), vxx), g);
    a = SUB<X>(a, MUL<X>(DTgf, vyy));
    a = SUB<X>(a, MUL<X>(dthalbe, sump));
    float sxx = ADD<X>(I.sxx[o], a);
    sump = 0.0f;
    const float djm = F(DMUL(DMUL(2.0, (double)mu), (double)taus));
    const float e = MUL<X>(pi, taup);
    const float de = SUB<X>(djm, e);
    const double fg1 = DSUB((double)DIV<X>(fjm, g), 1.0);
#pragma unroll
    for (int l = 0; l < L; l++) {
        const float bjm = I.s_bjm[l];
        const double inner = DSUB(DMUL(DMUL((double)de, fg1), (double)vxx), (double)MUL<X>(de, vyy));
        const float pv = F(DADD((double)I.p[o + l * I.plane], DMUL((double)bjm, inner)));
        I.p[o + l * I.plane] = pv;
        sump = ADD<X>(sump, pv);
    }
    I.sxx[o] = ADD<X>(sxx, MUL<X>(dthalbe, sump));
}

// ===========================================================================
// Receivers, seismo_ssg.c:24-105 (SEISMO 1..4), sample nt of every trace,
// plus the psv.c:99 NaN probe on vy[NY/2][NX/2].
// sec layout: [comp][nt][ntr] (comp 0 vx, 1 vy, 2 p, 3 curl, 4 div).
// ===========================================================================
template <int R>
__global__ void k_seismo(const Inst *__restrict__ insts, const int *__restrict__ ntb, int off)
{
    const Inst &I = insts[blockIdx.y];
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt) return;
    const long long P = I.pitch;
    // the buffers holding step nt's result (the second set after odd-distance steps of a fused instance)
    const bool alt = I.pp && ((I.nt - nt) & 1) != 0;
    const float *vxc = alt ? I.vx_b : I.vx, *vyc = alt ? I.vy_b : I.vy;
    const float *sxxc = alt ? I.sxx_b : I.sxx, *syyc = alt ? I.syy_b : I.syy;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        float v = vyc[(long long)(I.ny / 2) * P + I.nx / 2];
        if (isnan(v)) atomicOr(I.flag, 1);
    }
    if (I.mode == 1 || !I.seismo) return;
    const long long slab = (long long)I.nt * I.ntr;
    for (int itr = blockIdx.x * blockDim.x + threadIdx.x; itr < I.ntr; itr += gridDim.x * blockDim.x) {
        const int i = I.rec_i[itr], j = I.rec_j[itr];
        const long long o = (long long)j * P + i;
        const long long s = (long long)(nt - 1) * I.ntr + itr;
        const int S = I.seismo;
        if (S == 1 || S == 4) {
            I.sec[0 * slab + s] = vxc[o];
            I.sec[1 * slab + s] = vyc[o];
        }
        if (S == 2 || S == 4) I.sec[2 * slab + s] = __fsub_rn(-sxxc[o], syyc[o]);
        if (S == 3 || S == 4) {
            float vxx = 0.0f, vyy = 0.0f, vyx = 0.0f, vxy = 0.0f;
            for (int m = 1; m <= R; m++) {
                const float h = I.hc[m];
                vxx = __fadd_rn(vxx, __fmul_rn(h, __fsub_rn(vxc[o + m - 1], vxc[o - m])));
                vyy = __fadd_rn(vyy, __fmul_rn(h, __fsub_rn(vyc[o + (m - 1) * P], vyc[o - m * P])));
                vyx = __fadd_rn(vyx, __fmul_rn(h, __fsub_rn(vyc[o + m], vyc[o - m + 1])));
                vxy = __fadd_rn(vxy, __fmul_rn(h, __fsub_rn(vxc[o + m * P], vxc[o - (m - 1) * P])));
            }
            const float dhi = I.dhi_el;
            vxx = __fmul_rn(vxx, dhi);
            vyy = __fmul_rn(vyy, dhi);
            vyx = __fmul_rn(vyx, dhi);
            vxy = __fmul_rn(vxy, dhi);
            const float u = I.vs[o], pi = I.vp[o], rho = I.rho[o];
            const float muss = __fmul_rn(__fmul_rn(u, u), rho);
            const float lamss = __fmul_rn(__fmul_rn(pi, pi), rho);
            I.sec[4 * slab + s] = F(DMUL((double)__fadd_rn(vxx, vyy), sqrt((double)lamss)));
            I.sec[3 * slab + s] = F(DMUL((double)__fsub_rn(vxy, vyx), sqrt((double)muss)));
        }
    }
}

// ===========================================================================
// Snapshot encoding.  Snapshot k holds the five fields of psv.c:246-298
// (vxp1, vyp1, sxx, syy, sxy) of forward step 1 + k*DTINV.  Each field of
// each tile (blockDim.x x zch cells) carries its own power-of-two scale so
// FP16 keeps ~11 significant bits over the whole dynamic range.
// ===========================================================================
__device__ __forceinline__ float warp_max(float v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float block_max(float v, float *red)
{
    v = warp_max(v);
    const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if ((threadIdx.x & 31) == 0) red[w] = v;
    __syncthreads();
    float m = 0.0f;
    for (int k = 0; k < nw; k++) m = fmaxf(m, red[k]);
    __syncthreads();
    return m;
}

// scale s = 2^e with e chosen so max|x| / s lies in [2^14, 2^15); e >= -126 keeps
// s normal and its inverse finite (a tile whose values are all below 2^-111 is
// stored with s = 2^-126 and keeps fewer bits, which FP16 could not hold anyway)
__device__ __forceinline__ float pow2_scale(float amax)
{
    if (!(amax > 0.0f) || isinf(amax)) return 1.0f;
    int e;
    frexpf(amax, &e);   // amax = f * 2^e, f in [0.5, 1)
    return ldexpf(1.0f, max(e - 15, -126));
}

// the scaled store of one field's tile column, values already in hand
template <int PREC>
__device__ __forceinline__ void snap_put(const Inst &I, long long base, int r, float x, float inv)
{
    const long long e = base + (long long)r * blockDim.x + threadIdx.x;
    if (PREC == DN_SNAP_F16)
        ((__half *)I.snap)[e] = __float2half_rn(x * inv);
    else
        ((__nv_bfloat16 *)I.snap)[e] = __float2bfloat16_rn(x * inv);
}

// Tiles of at most ZR rows (the default 8): each thread loads its column of all
// five fields once, the five block maxima share one reduction, and the scaled
// values are stored from registers.  Same maxima (fmaxf ignores NaN in any
// order) and the same conversions as the two-pass loop below.
template <int PREC, int ZR>
__device__ __forceinline__ void snap_store_regs(const Inst &I, int k, int b, int i, int j0, int nrow, bool in, float *red)
{
    const long long P = I.pitch;
    const long long tile_cells = (long long)blockDim.x * I.zch;
    const float *src[5] = {I.vxp1, I.vyp1, I.sxx, I.syy, I.sxy};
    float v[5][ZR], am[5];
#pragma unroll
    for (int f = 0; f < 5; f++) {
        am[f] = 0.0f;
#pragma unroll
        for (int r = 0; r < ZR; r++) {
            v[f][r] = (in && r < nrow) ? src[f][(long long)(j0 + r) * P + i] : 0.0f;
            am[f] = fmaxf(am[f], fabsf(v[f][r]));
        }
    }
    const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int f = 0; f < 5; f++) {
        const float m = warp_max(am[f]);
        if ((threadIdx.x & 31) == 0) red[f * 8 + w] = m;
    }
    __syncthreads();
#pragma unroll
    for (int f = 0; f < 5; f++) {
        float m = 0.0f;
        for (int q = 0; q < nw; q++) m = fmaxf(m, red[f * 8 + q]);
        const long long slot = ((long long)k * 5 + f) * I.tiles + b;
        const float sc = pow2_scale(m);
        const float inv = 1.0f / sc;   // exact: power of two
        if (threadIdx.x == 0) I.snap_scale[slot] = sc;
        if (in) {
#pragma unroll
            for (int r = 0; r < ZR; r++)
                if (r < nrow) snap_put<PREC>(I, slot * tile_cells, r, v[f][r], inv);
        }
    }
}

static __global__ void k_snap_store(const Inst *__restrict__ insts, const int *__restrict__ ntb, int off)
{
    const Inst &I = insts[blockIdx.y];
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt || I.mode != 0 || !I.store || ((nt - 1) % I.dtinv) != 0) return;
    const int k = (nt - 1) / I.dtinv - I.snap_base;
    if (k < 0 || k >= I.nsnap) return;
    const int b = blockIdx.x;
    if (b >= I.tiles) return;
    __shared__ float red[5 * 8];   // five maxima of up to 8 warps
    const int tx = b % I.tiles_x, tz = b / I.tiles_x;
    const int i = tx * blockDim.x + threadIdx.x + 1;
    const int j0 = tz * I.zch + 1;
    const int nrow = min(I.zch, I.ny - j0 + 1);
    const bool in = i <= I.nx;
    const long long P = I.pitch;
    const long long tile_cells = (long long)blockDim.x * I.zch;
    const float *src[5] = {I.vxp1, I.vyp1, I.sxx, I.syy, I.sxy};
    if (I.eprecond == 1 || I.eprecond == 3) {
        for (int r = 0; r < nrow && in; r++) {
            const long long o = (long long)(j0 + r) * P + i;
            const long long w = (long long)(j0 + r - 1) * I.nx + (i - 1);
            I.Ws[w] = __fadd_rn(I.Ws[w], __fadd_rn(__fmul_rn(I.vx[o], I.vx[o]), __fmul_rn(I.vy[o], I.vy[o])));
        }
    }
    if (I.snap_prec != DN_SNAP_F32 && I.zch <= 4) {   // the default tile height: 20 values in registers
        if (I.snap_prec == DN_SNAP_F16)
            snap_store_regs<DN_SNAP_F16, 4>(I, k, b, i, j0, nrow, in, red);
        else
            snap_store_regs<DN_SNAP_BF16, 4>(I, k, b, i, j0, nrow, in, red);
        return;
    }
    if (I.snap_prec != DN_SNAP_F32 && I.zch <= 8) {
        if (I.snap_prec == DN_SNAP_F16)
            snap_store_regs<DN_SNAP_F16, 8>(I, k, b, i, j0, nrow, in, red);
        else
            snap_store_regs<DN_SNAP_BF16, 8>(I, k, b, i, j0, nrow, in, red);
        return;
    }
    for (int f = 0; f < 5; f++) {
        const long long slot = ((long long)k * 5 + f) * I.tiles + b;
        const long long base = slot * tile_cells;
        if (I.snap_prec == DN_SNAP_F32) {
            float *dst = (float *)I.snap + base;
            for (int r = 0; r < nrow; r++)
                if (in) dst[(long long)r * blockDim.x + threadIdx.x] = src[f][(long long)(j0 + r) * P + i];
            continue;
        }
        float amax = 0.0f;
        for (int r = 0; r < nrow && in; r++) amax = fmaxf(amax, fabsf(src[f][(long long)(j0 + r) * P + i]));
        amax = block_max(amax, red);
        const float sc = pow2_scale(amax);
        const float inv = 1.0f / sc;   // exact: power of two
        if (threadIdx.x == 0) I.snap_scale[slot] = sc;
        for (int r = 0; r < nrow && in; r++) {
            const float x = src[f][(long long)(j0 + r) * P + i];
            if (I.snap_prec == DN_SNAP_F16)
                snap_put<DN_SNAP_F16>(I, base, r, x, inv);
            else
                snap_put<DN_SNAP_BF16>(I, base, r, x, inv);
        }
    }
}

// resident CTAs of 256 threads asked of the correlation kernel (40 registers at 6)
#ifndef DN_CORR_MINB
#define DN_CORR_MINB 6
#endif

// ---------------------------------------------------------------------------
// a / b from y = RN(1/b) without the general division routine.  q0 = RN(a y)
// is within 1.5 ulp of a / b; one correction q1 = RN(q0 + RN(a - b q0) y)
// leaves a relative error of about 2^-104 before its rounding, so q1 is within
// one ulp, and then by Markstein's theorem (P. W. Markstein, IBM J. Res.
// Develop. 34(1), 1990) the remainder r1 = a - b q1 is exact in an fma and
// RN(q1 + r1 y) is the correctly rounded quotient.  This holds while every
// intermediate stays in the normal range of double, which is the case for
// operands converted from float: |a| and |b| lie in [2^-151, 2^128], the
// quotient in [2^-279, 2^279] and the remainders are multiples of 2^-480.  A
// zero dividend, b = 0 (y = inf) and b = inf (y = 0) and non-finite
// dividends make the corrections NaN or lose the sign of zero; there q0 is
// the IEEE quotient (a * inf or a * 0 with the sign of a), so it is returned.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double ddiv_rcp(double a, double b, double y)
{
    const double q0 = __dmul_rn(a, y);
    const double q1 = __fma_rn(__fma_rn(-b, q0, a), y, q0);
    const double q2 = __fma_rn(__fma_rn(-b, q1, a), y, q1);
    return (isfinite(q2) && a != 0.0) ? q2 : q0;
}

// the snapshot value at element e of a tile slot with scale s
template <int PREC> __device__ __forceinline__ float snap_at(const void *base, long long e, float s);
template <> __device__ __forceinline__ float snap_at<DN_SNAP_F32>(const void *base, long long e, float)
{
    return ((const float *)base)[e];
}
template <> __device__ __forceinline__ float snap_at<DN_SNAP_F16>(const void *base, long long e, float s)
{
    return __half2float(((const __half *)base)[e]) * s;
}
template <> __device__ __forceinline__ float snap_at<DN_SNAP_BF16>(const void *base, long long e, float s)
{
    return __bfloat162float(((const __nv_bfloat16 *)base)[e]) * s;
}

// ===========================================================================
// Adjoint cross-correlation, psv.c:313-387 (GRAD_FORM 1, INVMAT1 1), at the
// adjoint steps whose mirrored forward step NT-nt+1 stored a snapshot.  Of the
// mu term's three double divisions, the two by muss^2 share one reciprocal:
// psv.c's first term multiplies by 1.0/(muss*muss) itself and the third
// quotient comes out of ddiv_rcp from the same reciprocal, bit-identical to
// the division it replaces.
// ===========================================================================
// accumulator update in the accumulator's precision: float sums as psv.c's
// float grad arrays, double sums for DN_ACC_F64
__device__ __forceinline__ float acc_add(float w, float t) { return __fadd_rn(w, t); }
__device__ __forceinline__ double acc_add(double w, float t) { return DADD(w, (double)t); }
__device__ __forceinline__ float acc_add_mu(float w, double t) { return F(DADD((double)w, t)); }
__device__ __forceinline__ double acc_add_mu(double w, double t) { return DADD(w, t); }

// One tile column of the correlation.  Each row first loads everything it
// reads, the three accumulators included, and only then stores: the stores
// may alias the loads as far as the compiler knows, so loads placed after a
// store would wait for it and serialise three memory round trips per row.
template <int PREC, typename A>
__device__ __forceinline__ void correlate_tile(const Inst &I, int k, int b, int i, int j0, int nrow)
{
    const long long P = I.pitch;
    const long long T = I.tiles;
    const long long tc = (long long)blockDim.x * I.zch;   // cells per tile slot
    const long long s0 = (long long)k * 5 * T + b;        // slot of the first of the five fields
    const size_t esz = PREC == DN_SNAP_F32 ? 4 : 2;
    const char *sp = (const char *)I.snap + (s0 * tc + threadIdx.x) * esz;
    const long long sstep = T * tc * esz;                 // bytes from one field's slot to the next
    float sc[5];
#pragma unroll
    for (int f = 0; f < 5; f++) sc[f] = PREC == DN_SNAP_F32 ? 1.0f : I.snap_scale[s0 + f * T];
    const long long o0 = (long long)j0 * P + i;
    const long long w0 = (long long)(j0 - 1) * I.nx + (i - 1);
    A *wc = (A *)I.wc + w0, *wcu = (A *)I.wcu + w0, *wcr = (A *)I.wcrho + w0;
    const bool wr = I.eprecond == 1;
#pragma unroll 1
    for (int r = 0; r < nrow; r++) {
        const long long o = o0 + r * P, w = r * (long long)I.nx;
        const char *se = sp + (long long)r * blockDim.x * esz;
        const float frx = snap_at<PREC>(se, 0, sc[0]);
        const float fry = snap_at<PREC>(se + sstep, 0, sc[1]);
        const float fx = snap_at<PREC>(se + 2 * sstep, 0, sc[2]);
        const float fy = snap_at<PREC>(se + 3 * sstep, 0, sc[3]);
        const float fu = snap_at<PREC>(se + 4 * sstep, 0, sc[4]);
        const float vxp1 = I.vxp1[o], vyp1 = I.vyp1[o];
        const float sxx = I.sxx[o], syy = I.syy[o], sxy = I.sxy[o];
        const float muss = I.gmuss[o], lamss = I.glamss[o];
        const A ar = wcr[w], al = wc[w], au = wcu[w];
        float vx = 0.0f, vy = 0.0f, wrv = 0.0f;
        if (wr) {
            vx = I.vx[o];
            vy = I.vy[o];
            wrv = I.Wr[w0 + w];
        }
        const float trho = __fadd_rn(__fmul_rn(vxp1, frx), __fmul_rn(vyp1, fry));
        const float tlam = __fmul_rn(__fadd_rn(fx, fy), __fadd_rn(sxx, syy));
        const bool mpos = muss > 0.0f;
        double tmu = 0.0;
        if (mpos) {
            const double mm = (double)__fmul_rn(muss, muss);
            const float lm = __fadd_rn(lamss, muss);
            const double y = DDIV(1.0, mm);
            const double t1 = DMUL(y, (double)__fmul_rn(fu, sxy));
            const double t2 = DDIV(DMUL(0.25, (double)tlam), (double)__fmul_rn(lm, lm));
            const double t3 = ddiv_rcp(DMUL(0.25, (double)__fmul_rn(__fsub_rn(fx, fy), __fsub_rn(sxx, syy))), mm, y);
            tmu = DADD(DADD(t1, t2), t3);
        }
        wcr[w] = acc_add(ar, trho);
        wc[w] = acc_add(al, tlam);
        if (mpos) wcu[w] = acc_add_mu(au, tmu);
        if (wr) I.Wr[w0 + w] = __fadd_rn(wrv, __fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)));
    }
}

template <int PREC>
__device__ __forceinline__ void correlate_prec(const Inst &I, int k, int b, int i, int j0, int nrow)
{
    if (I.acc64)
        correlate_tile<PREC, double>(I, k, b, i, j0, nrow);
    else
        correlate_tile<PREC, float>(I, k, b, i, j0, nrow);
}

// insts is not __restrict__ here: with it the compiler keeps a dozen instance
// pointers live across the row loop and spills at 40 registers; without it they
// are re-read from the (L1-resident) descriptor, which measured ~1 ms faster on the
// 4-shot 2000 x 600 FP16 adjoint
static __global__ void __launch_bounds__(256, DN_CORR_MINB) k_correlate(const Inst *insts, const int *__restrict__ ntb, int off)
{
    const Inst &I = insts[blockIdx.y];
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt || I.mode != 1) return;
    const int nf = I.nt - nt + 1;   // mirrored forward step
    if (((nf - 1) % I.dtinv) != 0) return;
    const int k = (nf - 1) / I.dtinv - I.snap_base;
    if (k < 0 || k >= I.nsnap) return;
    const int b = blockIdx.x;
    if (b >= I.tiles) return;
    const int tx = b % I.tiles_x, tz = b / I.tiles_x;
    const int i = tx * blockDim.x + threadIdx.x + 1;
    if (i > I.nx) return;
    const int j0 = tz * I.zch + 1;
    const int nrow = min(I.zch, I.ny - j0 + 1);
    if (I.snap_prec == DN_SNAP_F16)
        correlate_prec<DN_SNAP_F16>(I, k, b, i, j0, nrow);
    else if (I.snap_prec == DN_SNAP_BF16)
        correlate_prec<DN_SNAP_BF16>(I, k, b, i, j0, nrow);
    else
        correlate_prec<DN_SNAP_F32>(I, k, b, i, j0, nrow);
}

}   // namespace dn
