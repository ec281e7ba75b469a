/* Internal declarations shared by the host C and CUDA translation units. */
#ifndef DN_INTERNAL_H
#define DN_INTERNAL_H

#include "denise_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Records `msg` as the thread's last error and returns `code`. */
int dn_fail(int code, const char *fmt, ...);

int dn_visc_eta(const dn_params *p, float *eta, float *pts);
float dn_visc_sum(const dn_params *p, float ws);
float dn_visc_tau_from_q(float q);
/* the sum dn_visc_cell_factors divides by: dn_visc_sum at ws = 2 pi FL[0] */
float dn_visc_sumu(const dn_params *p);
int dn_visc_cell_factors(const dn_params *p, const float *vp, const float *vs, const float *rho, const float *qp,
                         const float *qs, float *muipjp, float *tausipjp, float *mu, float *taus, float *pi,
                         float *taup);

/* Device view of a model's stacked gradient and raw model planes for the
 * gradient conditioning (dn_precond.cu) and the optimisers (dn_fwi.cu). */
typedef struct {
    int nx, ny, pitch, device, grad64;
    void *dgrad;            /* 3 x nx*ny, row-major [j][i] */
    const float *vs;        /* origin pointers: element (j, i) at vs[j * pitch + i] */
    const float *vp, *rho;
} dn_model_view;
int dn_model_view_get(dn_model *m, dn_model_view *v);

#ifdef __cplusplus
}
#endif

#ifdef __CUDACC__
/* Returns a DN_E* status from the calling function when a CUDA call fails. */
#define CU(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            return dn_fail(e_ == cudaErrorMemoryAllocation ? DN_ENOMEM : DN_EDEVICE, "%s: %s (%s:%d)", \
                           #call, cudaGetErrorString(e_), __FILE__, __LINE__);                     \
        }                                                                                          \
    } while (0)
#endif

#ifdef __CUDACC__
/* Device memory through the library's block cache (dn_alloc.cu): drop-in
 * replacements of cudaMalloc / cudaFree on the current device. */
cudaError_t dn_malloc_bytes(void **p, size_t bytes);
template <typename T>
inline cudaError_t dn_malloc(T **p, size_t bytes)
{
    return dn_malloc_bytes(reinterpret_cast<void **>(p), bytes);
}
void dn_free(void *p);
size_t dn_pool_idle_bytes(int device);
#endif

#ifdef __cplusplus
#include <nvtx3/nvToolsExt.h>
/* NVTX range for the duration of a scope (shows the library's phases in a
 * timeline profiler; the header-only NVTX calls cost nothing without one). */
struct DnRange {
    explicit DnRange(const char *name) { nvtxRangePushA(name); }
    ~DnRange() { nvtxRangePop(); }
    DnRange(const DnRange &) = delete;
    DnRange &operator=(const DnRange &) = delete;
};
#endif

/* Grid padding of every device field: HX columns left/right, HZ rows above/below
 * the interior.  HZ >= FDORDER/2 covers the free-surface image rows and the
 * stencil reach; HX = 8 keeps column i = 1 16-byte aligned. */
#define DN_HX 8
#define DN_HZ 8

#endif
