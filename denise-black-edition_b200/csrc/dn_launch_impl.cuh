// Definitions of the per-order launch functions; included once per order by
// dn_launch_rN.cu with DN_R = N.
#pragma once

#include "dn_launch.cuh"

namespace dn {

template <int R, bool X>
void launch_step_R(const LaunchCfg &c, cudaStream_t st, const Inst *d, const int *ntb, int off, long long &nl,
                          cudaEvent_t *marks)
{
    MARK(0);
    if (c.any_fused) {   // velocity, sources, stress and free surface of the fused instances
        k_step_el_fused<R, X><<<c.fgrid, FZ_NP, fz_ring_bytes(R), st>>>(d, ntb, off);
        nl++;
    }
    if (c.any_plain) {
        if (c.vpipe) k_update_v_pipe<R, X><<<c.vgrid, VP_THREADS, vpipe_smem_bytes(), st>>>(d, ntb, off, c.vsh);
        else if (c.tma)
            k_update_v_tma<R, X><<<c.tile_grid, TMA_W, pipe_smem_bytes<QV>(slot_floats_v()), st>>>(d, ntb, off);
        else if (c.pack && c.fuse_src) k_update_v2<R, X, true><<<c.tile_grid, c.bx / 2, 0, st>>>(d, ntb, off);
        else if (c.pack) k_update_v2<R, X><<<c.tile_grid, c.bx / 2, 0, st>>>(d, ntb, off);
        else k_update_v<R, X><<<c.tile_grid, c.bx, 0, st>>>(d, ntb, off);
    }
    MARK(1);
    if (c.any_plain) nl++;
    if (c.any_plain && c.need_inject_v) {
        k_inject_v<<<c.src_grid, 128, 0, st>>>(d, ntb, off);
        nl++;
    }
    MARK(2);
    if (!c.any_plain) {
        // every instance took the fused step
    } else if (c.L == 0) {
        if (c.tma)
            k_update_s_el_tma<R, X><<<c.tile_grid, TMA_W, pipe_smem_bytes<QS_EL>(slot_floats_s_el()), st>>>(d, ntb, off);
        else if (c.pack && c.fuse_src) k_update_s_el2<R, X, true><<<c.tile_grid, c.bx / 2, 0, st>>>(d, ntb, off);
        else if (c.pack) k_update_s_el2<R, X><<<c.tile_grid, c.bx / 2, 0, st>>>(d, ntb, off);
        else k_update_s_el<R, X><<<c.tile_grid, c.bx, 0, st>>>(d, ntb, off);
    } else if (c.tma) {
#define DN_VI_TMA(LL)                                                                                          \
    k_update_s_vi_tma<R, LL, X><<<c.tile_grid, TMA_W, pipe_smem_bytes<QS_VI>(slot_floats_s_vi(LL)), st>>>(d, ntb, off)
        switch (c.L) {
        case 1: DN_VI_TMA(1); break;
        case 2: DN_VI_TMA(2); break;
        case 3: DN_VI_TMA(3); break;
        case 4: DN_VI_TMA(4); break;
        default: DN_VI_TMA(5); break;
        }
#undef DN_VI_TMA
    } else {
#define DN_VI(LL)                                                                                              \
    (c.fuse_src ? k_update_s_vi<R, LL, X, true><<<c.tile_grid, c.bx, 0, st>>>(d, ntb, off)                        \
                : k_update_s_vi<R, LL, X><<<c.tile_grid, c.bx, 0, st>>>(d, ntb, off))
        switch (c.L) {
        case 1: DN_VI(1); break;
        case 2: DN_VI(2); break;
        case 3: DN_VI(3); break;
        case 4: DN_VI(4); break;
        default: DN_VI(5); break;
        }
#undef DN_VI
    }
    if (c.any_plain) nl++;
    MARK(3);
    if (c.any_src_s && c.any_plain) {
        k_inject_s<<<c.src_grid, 128, 0, st>>>(d, ntb, off);
        nl++;
    }
    MARK(4);
    if (c.any_surf && c.any_plain) {
        if (c.L == 0) {
            k_surface_el<R, X><<<c.surf_grid, 128, 0, st>>>(d, ntb, off);
        } else {
            switch (c.L) {
            case 1: k_surface_vi<R, 1, X><<<c.surf_grid, 128, 0, st>>>(d, ntb, off); break;
            case 2: k_surface_vi<R, 2, X><<<c.surf_grid, 128, 0, st>>>(d, ntb, off); break;
            case 3: k_surface_vi<R, 3, X><<<c.surf_grid, 128, 0, st>>>(d, ntb, off); break;
            case 4: k_surface_vi<R, 4, X><<<c.surf_grid, 128, 0, st>>>(d, ntb, off); break;
            default: k_surface_vi<R, 5, X><<<c.surf_grid, 128, 0, st>>>(d, ntb, off); break;
            }
        }
        nl++;
    }
    MARK(5);
    k_seismo<R><<<c.rec_grid, 128, 0, st>>>(d, ntb, off);
    nl++;
    MARK(6);
    if (c.any_store) {
        k_snap_store<<<c.tile_grid, c.bx, 0, st>>>(d, ntb, off);
        nl++;
    }
    MARK(7);
    if (c.any_adj) {
        k_correlate<<<c.tile_grid, c.bx, 0, st>>>(d, ntb, off);
        nl++;
    }
    MARK(8);
}

// opt the pipelined kernels into their dynamic shared memory (needed above 48 KB)
template <int R, bool X>
int set_smem_attrs_R()
{
    cudaFuncSetAttribute(k_update_v_tma<R, X>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)pipe_smem_bytes<QV>(slot_floats_v()));
    cudaFuncSetAttribute(k_update_s_el_tma<R, X>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)pipe_smem_bytes<QS_EL>(slot_floats_s_el()));
    cudaFuncSetAttribute(k_update_s_vi_tma<R, 1, X>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)pipe_smem_bytes<QS_VI>(slot_floats_s_vi(1)));
    cudaFuncSetAttribute(k_update_s_vi_tma<R, 2, X>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)pipe_smem_bytes<QS_VI>(slot_floats_s_vi(2)));
    cudaFuncSetAttribute(k_update_s_vi_tma<R, 3, X>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)pipe_smem_bytes<QS_VI>(slot_floats_s_vi(3)));
    cudaFuncSetAttribute(k_update_s_vi_tma<R, 4, X>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)pipe_smem_bytes<QS_VI>(slot_floats_s_vi(4)));
    cudaError_t e = cudaFuncSetAttribute(k_update_s_vi_tma<R, 5, X>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)pipe_smem_bytes<QS_VI>(slot_floats_s_vi(5)));
    return e == cudaSuccess ? 0 : -1;
}

template <int R, bool X>
int set_vpipe_attr_R()
{
    cudaError_t e = cudaFuncSetAttribute(k_update_v_pipe<R, X>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)vpipe_smem_bytes());
    return e == cudaSuccess ? 0 : -1;
}

#ifdef DN_R
template void launch_step_R<DN_R, true>(const LaunchCfg &, cudaStream_t, const Inst *, const int *, int, long long &,
                                        cudaEvent_t *);
template void launch_step_R<DN_R, false>(const LaunchCfg &, cudaStream_t, const Inst *, const int *, int, long long &,
                                         cudaEvent_t *);
template int set_smem_attrs_R<DN_R, true>();
template int set_smem_attrs_R<DN_R, false>();
template int set_vpipe_attr_R<DN_R, true>();
template int set_vpipe_attr_R<DN_R, false>();
#endif

}   // namespace dn
