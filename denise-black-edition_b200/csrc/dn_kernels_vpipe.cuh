// Velocity update fed by a warp-specialised bulk-copy pipeline (sm_100a).
//
// Same operations as k_update_v2 (update_v_PML_PSV.c:53-715 with CPML and the
// mode-dependent vxp1/vyp1 terms; bit-identical with EXACT = true), different
// data movement.  A CTA owns a strip of VP_W = 256 columns and `sh` rows and
// streams down it.  One producer warp copies, row after row, the row segments
// the strip needs (sxx and sxy with an 8-column halo on each side, syy, rip,
// rjp, vx, vy) with 1-D bulk copies (cp.async.bulk global -> shared, completion
// counted on a per-slot mbarrier) into a ring of VP_S slots, VP_S - R - 1 rows
// ahead of the consumers.  128 consumer threads own two adjacent columns each
// (packed FP32x2 arithmetic as in k_update_v2): the z stencils of syy and sxy
// live in register windows that take one new row per step, the x stencils and
// the own-row operands are read from shared memory, and each consumer warp
// releases a slot (an arrive on its "empty" mbarrier) as soon as it is done
// with it.  The producer refills a slot after all four consumer warps released
// it.  Rows j0 - R .. j0 - 1 and j1 + 1 .. j1 + R are copied for the windows
// only (syy and sxy).
//
// Every wait is bounded: a wait that runs out sets bit 1 of the shot's status
// flag, and the CTA stops issuing copies, waits (bounded) for the copies it
// issued and exits; the host reports DN_ETIMEDOUT.  No cluster or multicast
// copy is used; every source address lies in this GPU's memory.
//
// Copy bounds: the padded planes hold rows 1 - HZ .. ny + HZ (HZ = 8 > R) and
// pitch >= nx + 16 floats per row, a multiple of 32.  A halo segment starts at
// column c0 - 8 (element c0 - 1 of the row, a multiple of 256 floats) and a
// W-wide segment at column c0 (element c0 + 7); both are cut at the row's end,
// so every copy stays inside its row, starts 16-byte aligned and has a size
// that is a multiple of 16 bytes.
#pragma once

#include "dn_kernels.cuh"
#include "dn_pipe.cuh"

namespace dn {

constexpr int VP_W = 256;                  // columns per CTA
constexpr int VP_CT = VP_W / 2;            // consumer threads (two columns each)
constexpr int VP_THREADS = VP_CT + 32;     // + one producer warp
constexpr int VP_HW = VP_W + 16;           // halo segment width
constexpr int VP_S = 8;                    // ring slots
constexpr int VP_SLOT = 2 * VP_HW + 5 * VP_W;   // floats per slot: sxx, sxy (halo) | syy, rip, rjp, vx, vy
constexpr size_t vpipe_smem_bytes() { return (size_t)VP_S * VP_SLOT * 4 + (size_t)2 * VP_S * 8; }

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <int R, bool X>
__global__ void __launch_bounds__(VP_THREADS, 3) k_update_v_pipe(const Inst *__restrict__ insts,
                                                                 const int *__restrict__ ntb, int off, int sh)
{
    extern __shared__ __align__(128) float smem[];
    const Inst &I = insts[blockIdx.y];
    if (I.pp) return;   // the fused step handles this instance
    const int nt = *ntb + off - I.t0;   // the instance's own time step
    if (nt < 1 || nt > I.nt) return;
    const int tiles_x = (I.nx + VP_W - 1) / VP_W;
    const int b = blockIdx.x;
    if (b >= tiles_x * ((I.ny + sh - 1) / sh)) return;
    const int tx = b % tiles_x, tz = b / tiles_x;
    const int c0 = tx * VP_W + 1;
    const int j0 = tz * sh + 1, j1 = min(j0 + sh - 1, I.ny);
    const long long P = I.pitch;
    // items: rows j0 - R .. j1 + R
    const int nitems = j1 - j0 + 1 + 2 * R;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + (size_t)VP_S * VP_SLOT);
    uint64_t *empty = full + VP_S;
    __shared__ int abort_flag;
    if (threadIdx.x == 0) {
        for (int q = 0; q < VP_S; q++) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], VP_CT / 32);
        }
        abort_flag = 0;
        mbar_fence_init();
    }
    __syncthreads();
    // segment widths, cut at the row end (multiples of 8 floats)
    const int wH = min(VP_HW, (int)P - (c0 - 1));
    const int wW = min(VP_W, (int)P - (c0 + 7));

    if (threadIdx.x >= VP_CT) {
        // ---------------- producer warp ----------------
        const int lane = threadIdx.x - VP_CT;
        int issued = 0;
        for (int k = 0; k < nitems; k++) {
            const int s = k % VP_S;
            if (k >= VP_S) {
                // slot s held item k - VP_S; wait until the four consumer warps released it
                bool ok = true;
                if (lane == 0) ok = mbar_wait_bounded(&empty[s], (unsigned)((k / VP_S - 1) & 1));
                ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
                if (!ok || *(volatile int *)&abort_flag) {
                    if (lane == 0) {
                        atomicOr(I.flag, 2);
                        abort_flag = 1;
                    }
                    break;
                }
            }
            const long long j = j0 - R + k;
            const bool body = j >= j0 && j <= j1;   // rows the strip computes need every field
            const unsigned bytes = (unsigned)(body ? 2 * wH + 5 * wW : wH + wW) * 4;
            float *slot = smem + (size_t)s * VP_SLOT;
            if (lane == 0) mbar_arrive_expect_tx(&full[s], bytes);
            __syncwarp();
            const long long rb = j * P;
            switch (lane) {
            case 0: if (body) bulk_g2s(slot, I.sxx + rb + c0 - 8, wH * 4, &full[s]); break;
            case 1: bulk_g2s(slot + VP_HW, I.sxy + rb + c0 - 8, wH * 4, &full[s]); break;
            case 2: bulk_g2s(slot + 2 * VP_HW, I.syy + rb + c0, wW * 4, &full[s]); break;
            case 3: if (body) bulk_g2s(slot + 2 * VP_HW + VP_W, I.rip + rb + c0, wW * 4, &full[s]); break;
            case 4: if (body) bulk_g2s(slot + 2 * VP_HW + 2 * VP_W, I.rjp + rb + c0, wW * 4, &full[s]); break;
            case 5: if (body) bulk_g2s(slot + 2 * VP_HW + 3 * VP_W, I.vx + rb + c0, wW * 4, &full[s]); break;
            case 6: if (body) bulk_g2s(slot + 2 * VP_HW + 4 * VP_W, I.vy + rb + c0, wW * 4, &full[s]); break;
            default: break;
            }
            issued = k + 1;
        }
        // copies issued but maybe not consumed (abort): wait for them before the CTA exits
        if (*(volatile int *)&abort_flag && lane == 0)
            for (int k = max(0, issued - VP_S); k < issued; k++)
                mbar_wait_bounded(&full[k % VP_S], (unsigned)((k / VP_S) & 1));
        __syncthreads();
        return;
    }

    // ---------------- consumers ----------------
    const int t = threadIdx.x;
    const int i0 = c0 + 2 * t;
    const bool active = i0 <= I.nx;
    const bool two = i0 + 1 <= I.nx;
    float hc[R + 1];
#pragma unroll
    for (int m = 1; m <= R; m++) hc[m] = I.hc[m];
    const float DT = I.DT, DH = I.DH, rdh = I.rdh;
    const bool fd = I.fastdiv;
    const int mode = I.mode;
    const bool snapstep = (mode == 0) && I.store && ((nt - 1) % I.dtinv == 0);
    const int fw = I.fw, nx = I.nx, ny = I.ny, free_surf = I.free_surf;
    const bool xframe = fw > 0 && (i0 <= fw || i0 + 1 >= nx - fw + 1);
    // z windows (paired columns) for row j: wyy[q] = syy row j - R + 1 + q, wxy[q] = sxy row j - R + q
    float2 wyy[2 * R], wxy[2 * R];
#pragma unroll
    for (int q = 0; q < 2 * R; q++) wyy[q] = wxy[q] = make_float2(0.f, 0.f);
    for (int k = 0; k < nitems; k++) {
        const int s = k % VP_S;
        const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&full[s], (unsigned)((k / VP_S) & 1)));
        if (!ok) {   // only if a copy never landed: give up (the producer drains its copies)
            if ((t & 31) == 0) {
                atomicOr(I.flag, 2);
                abort_flag = 1;
            }
            break;
        }
        const float *slot = smem + (size_t)s * VP_SLOT;
        // item k is row j0 - R + k: its syy enters the syy window now (rows j - R + 1 .. j + R of
        // row j = j0 - 2R + k), its sxy after row j is computed (rows j - R .. j + R - 1)
#pragma unroll
        for (int q = 0; q < 2 * R - 1; q++) wyy[q] = wyy[q + 1];
        wyy[2 * R - 1] = *reinterpret_cast<const float2 *>(slot + 2 * VP_HW + 2 * t);
        const int j = j0 - 2 * R + k;
        const int kj = k - R;                            // the item of row j (still in its slot)
        if (j >= j0 && j <= j1 && active) {
            const float *rs = smem + (size_t)(kj % VP_S) * VP_SLOT;
            // x stencils from the halo segments: the halo index of column c is c - c0 + 8
            float2 ax[2 * R], bx[2 * R];
            {
                // sxx: columns i0 - R + 1 .. i0 + R
                const float *row = rs + 2 * t + 8 - R + 1;
                constexpr int kb = (R % 2 == 0) ? -1 : 0;
                float2 Lq[R + 1];
#pragma unroll
                for (int q = 0; q <= R; q++) Lq[q] = *reinterpret_cast<const float2 *>(row + kb + 2 * q);
#pragma unroll
                for (int m = 0; m < 2 * R; m++) {
                    if (((m - kb) & 1) == 0) ax[m] = Lq[(m - kb) / 2];
                    else ax[m] = make_float2(Lq[(m - 1 - kb) / 2].y, Lq[(m + 1 - kb) / 2].x);
                }
            }
            {
                // sxy: columns i0 - R .. i0 + R - 1
                const float *row = rs + VP_HW + 2 * t + 8 - R;
                constexpr int kb = (R % 2 == 0) ? 0 : -1;
                float2 Lq[R + 1];
#pragma unroll
                for (int q = 0; q <= R; q++) Lq[q] = *reinterpret_cast<const float2 *>(row + kb + 2 * q);
#pragma unroll
                for (int m = 0; m < 2 * R; m++) {
                    if (((m - kb) & 1) == 0) bx[m] = Lq[(m - kb) / 2];
                    else bx[m] = make_float2(Lq[(m - 1 - kb) / 2].y, Lq[(m + 1 - kb) / 2].x);
                }
            }
            // derivatives in the reference's term order (update_v_PML_PSV.c case 8 :366-480);
            // wyy[R - 1 + m] = syy row j + m, wyy[R - m] = syy row j - m + 1,
            // wxy[R + m - 1] = sxy row j + m - 1, wxy[R - m] = sxy row j - m
            float2 sxx_x = MUL2<X>(bc2(hc[1]), SUB2<X>(ax[R], ax[R - 1]));
            float2 sxy_x = MUL2<X>(bc2(hc[1]), SUB2<X>(bx[R], bx[R - 1]));
            float2 sxy_y = MUL2<X>(bc2(hc[1]), SUB2<X>(wxy[R], wxy[R - 1]));
            float2 syy_y = MUL2<X>(bc2(hc[1]), SUB2<X>(wyy[R], wyy[R - 1]));
#pragma unroll
            for (int m = 2; m <= R; m++) {
                sxx_x = ADD2<X>(sxx_x, MUL2<X>(bc2(hc[m]), SUB2<X>(ax[R - 1 + m], ax[R - m])));
                sxy_x = ADD2<X>(sxy_x, MUL2<X>(bc2(hc[m]), SUB2<X>(bx[R + m - 1], bx[R - m])));
                sxy_y = ADD2<X>(sxy_y, MUL2<X>(bc2(hc[m]), SUB2<X>(wxy[R + m - 1], wxy[R - m])));
                syy_y = ADD2<X>(syy_y, MUL2<X>(bc2(hc[m]), SUB2<X>(wyy[R - 1 + m], wyy[R - m])));
            }
            if (xframe) {
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
            const float *own = rs + 2 * VP_HW + 2 * t;
            const float2 ripv = *reinterpret_cast<const float2 *>(own + VP_W);
            const float2 rjpv = *reinterpret_cast<const float2 *>(own + 2 * VP_W);
            const float2 vxo = *reinterpret_cast<const float2 *>(own + 3 * VP_W);
            const float2 vyo = *reinterpret_cast<const float2 *>(own + 4 * VP_W);
            const float2 s1 = ADD2<X>(sxx_x, sxy_y);
            const float2 s2 = ADD2<X>(sxy_x, syy_y);
            const float2 nvx = ADD2<X>(vxo, DIVH2<X>(MUL2<X>(MUL2<X>(bc2(DT), ripv), s1), fd, DH, rdh));
            const float2 nvy = ADD2<X>(vyo, DIVH2<X>(MUL2<X>(MUL2<X>(bc2(DT), rjpv), s2), fd, DH, rdh));
            const long long o = (long long)j * P + i0;
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
#pragma unroll
        for (int q = 0; q < 2 * R - 1; q++) wxy[q] = wxy[q + 1];
        wxy[2 * R - 1] = *reinterpret_cast<const float2 *>(slot + VP_HW + 8 + 2 * t);
        // item k - R (row j) is done with: release its slot
        if (kj >= 0) {
            __syncwarp();
            if ((t & 31) == 0) mbar_arrive(&empty[kj % VP_S]);
        }
    }
    __syncthreads();
}

}   // namespace dn
