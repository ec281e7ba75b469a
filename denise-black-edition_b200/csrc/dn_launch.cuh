// Launch of one time step of a batch: the kernel sequence of psv() for the
// configured stencil kernels.  The per-order launch functions are compiled in
// separate translation units (dn_launch_r1.cu .. dn_launch_r6.cu) so that the
// many kernel instantiations build in parallel.
#pragma once

#include "dn_kernels_tma.cuh"
#include "dn_kernels_vpipe.cuh"
#include "dn_kernels_fused.cuh"

namespace dn {

struct LaunchCfg {
    dim3 tile_grid, src_grid, surf_grid, rec_grid;
    int bx;
    int auto_zch;     // rows per tile of the shots whose tiles the batch chooses (0: their own)
    int R, L;
    bool exact;
    bool tma;   // stencil kernels fed by the bulk-copy row pipeline
    bool pack;  // paired-column (FP32x2) stencil kernels, bx / 2 threads per tile
    bool vpipe; // velocity update by the warp-specialised copy pipeline (k_update_v_pipe)
    dim3 vgrid; // its grid: strips of VP_W columns x vsh rows per instance
    int vsh;
    bool any_surf, any_src_s, any_store, any_adj, any_rec;
    bool fuse_src;       // forward sources applied inside the velocity / stress kernels (Inst::fsrc_*)
    bool need_inject_v;  // k_inject_v still has work (adjoint forces, or sources not in the kernels)
    bool any_fused;   // some instance runs the fused elastic step (Inst::pp)
    bool any_plain;   // some instance runs the separate velocity / stress kernels
    dim3 fgrid;       // grid of the fused step: its tiles per instance
};

// marks (optional, profiling only): 9 events recorded around the 8 kernel slots
// v, inject_v, s, inject_s, surface, seismo, snap, correlate
#define MARK(k)                                                                                    \
    do {                                                                                           \
        if (marks) cudaEventRecord(marks[k], st);                                                  \
    } while (0)


template <int R, bool X>
void launch_step_R(const LaunchCfg &c, cudaStream_t st, const Inst *d, const int *ntb, int off, long long &nl,
                   cudaEvent_t *marks);
// opts the bulk-copy pipeline kernels of order R into their dynamic shared memory
template <int R, bool X>
int set_smem_attrs_R();
template <int R, bool X>
int set_vpipe_attr_R();

}   // namespace dn
