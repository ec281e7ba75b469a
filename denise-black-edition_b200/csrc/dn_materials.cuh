// Material fields of a model computed on the device from the model files:
// the same float / double operations as the host set-up (dn_setup.c:
// dn_average_materials, dn_visc_cell_factors; dn_engine.cu dn_model_create),
// so the planes are bit-identical to the ones built on the host.
//
// Reference: av_mue.c:29-44 and av_rho.c:13-22 (INVMAT1 == 1) with the
// periodic edges of matcopy (a single rank: the neighbour across an edge is
// the opposite edge), update_s_elastic_PML_PSV.c:442-444 and psv.c:333-334 for
// mu, lambda and the gradient's muss / lamss, prepare_update_s_visc_PSV.c and
// readmod_visc_PSV.c:119-120 for the viscoelastic factors.
#pragma once

#include <cuda_runtime.h>

namespace dn {

// file order (x-major: column i holds rows 1..ny) to a padded [z][x] plane, 32 x 32 tiles
__global__ void k_file_to_plane(const float *__restrict__ file, float *__restrict__ plane, int nx, int ny,
                                long long pitch)
{
    __shared__ float tile[32][33];
    const int j0 = blockIdx.x * 32, i0 = blockIdx.y * 32;   // file: i slow, j fast
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int i = i0 + k, j = j0 + threadIdx.x;
        if (i < nx && j < ny) tile[k][threadIdx.x] = file[(size_t)i * ny + j];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int j = j0 + k, i = i0 + threadIdx.x;
        if (i < nx && j < ny) plane[(long long)(j + 1) * pitch + (i + 1)] = tile[threadIdx.x][k];
    }
}

struct MatPlanes {
    const float *rho, *vs, *vp;       // origin pointers of the transposed model planes
    const float *qs, *qp;             // Q planes (honor_q), else null: Q = 30
    float *rip, *rjp, *uipjp, *mu, *lam, *gmuss, *glamss;
    float *c_muipjp, *c_tausipjp, *c_mu, *c_taus, *c_pi, *c_taup;   // viscoelastic (L > 0)
    long long pitch;
    int nx, ny, visc;
    float sumu;                       // dn_visc_sum(p, 2 pi FL[0])
};

__device__ __forceinline__ double ddv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float f2(double a) { return __double2float_rn(a); }

// tau of a Q value (readmod_visc_PSV.c:119-120: 2/Q in double, stored as float)
__device__ __forceinline__ float tau_of(const float *q, long long o) { return f2(ddv(2.0, q ? (double)q[o] : 30.0)); }

__global__ void k_materials(MatPlanes M)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y + 1;
    if (i > M.nx || j > M.ny) return;
    const long long P = M.pitch;
    // the periodic neighbours (matcopy): row ny + 1 is row 1, column nx + 1 is column 1
    const int i1 = i < M.nx ? i + 1 : 1, j1 = j < M.ny ? j + 1 : 1;
    const long long o = (long long)j * P + i, oE = (long long)j * P + i1, oS = (long long)j1 * P + i,
                    oSE = (long long)j1 * P + i1;
    const float r00 = M.rho[o], r01 = M.rho[oE], r10 = M.rho[oS], r11 = M.rho[oSE];
    const float us00 = M.vs[o], us01 = M.vs[oE], us10 = M.vs[oS], us11 = M.vs[oSE];
    // av_mue: harmonic mean of rho vs^2 over the four cells, in double
    const float u1 = __fmul_rn(__fmul_rn(r00, us00), us00);
    const float u2 = __fmul_rn(__fmul_rn(r01, us01), us01);
    const float u3 = __fmul_rn(__fmul_rn(r10, us10), us10);
    const float u4 = __fmul_rn(__fmul_rn(r11, us11), us11);
    const double hs = __dadd_rn(__dadd_rn(__dadd_rn(ddv(1.0, (double)u1), ddv(1.0, (double)u2)), ddv(1.0, (double)u3)),
                                ddv(1.0, (double)u4));
    float uipjp = f2(ddv(4.0, hs));
    if (u1 == 0.0f || u2 == 0.0f || u3 == 0.0f || u4 == 0.0f) uipjp = 0.0f;
    // av_rho: 1 / (0.5 (r + r')), the float sum promoted
    float vj = f2(ddv(1.0, __dmul_rn(0.5, (double)__fadd_rn(r00, r10))));
    float vi = f2(ddv(1.0, __dmul_rn(0.5, (double)__fadd_rn(r00, r01))));
    if ((double)r00 < 1e-4 && (double)r10 < 1e-4) vj = 0.0f;
    if ((double)r00 < 1e-4 && (double)r01 < 1e-4) vi = 0.0f;
    M.rip[o] = vi;
    M.rjp[o] = vj;
    M.uipjp[o] = uipjp;
    // mu = rho u u, lambda = rho (pi pi - 2 u u) (float), lamss = rho pi pi - 2.0 muss (double)
    const float u = us00, pi = M.vp[o], r = r00;
    const float muv = __fmul_rn(__fmul_rn(r, u), u);
    M.mu[o] = muv;
    M.lam[o] = __fmul_rn(r, __fsub_rn(__fmul_rn(pi, pi), __fmul_rn(__fmul_rn(2.0f, u), u)));
    M.gmuss[o] = muv;
    M.glamss[o] = f2(__dadd_rn((double)__fmul_rn(__fmul_rn(r, pi), pi), -__dmul_rn(2.0, (double)muv)));
    if (!M.visc) return;
    // viscoelastic factors: tau at the four cells (periodic), averaged in float, times 0.25 in double
    const float t00 = tau_of(M.qs, o), t01 = tau_of(M.qs, oE), t10 = tau_of(M.qs, oS), t11 = tau_of(M.qs, oSE);
    const float tsij = f2(__dmul_rn(0.25, (double)__fadd_rn(__fadd_rn(__fadd_rn(t00, t01), t10), t11)));
    const float tp = tau_of(M.qp, o);
    const float sumu = M.sumu;
    M.c_muipjp[o] = f2(ddv((double)uipjp, __dadd_rn(1.0, (double)__fmul_rn(sumu, tsij))));
    M.c_tausipjp[o] = tsij;
    M.c_mu[o] = f2(ddv((double)__fmul_rn(__fmul_rn(u, u), r), __dadd_rn(1.0, (double)__fmul_rn(sumu, t00))));
    M.c_taus[o] = t00;
    M.c_pi[o] = f2(ddv((double)__fmul_rn(__fmul_rn(pi, pi), r), __dadd_rn(1.0, (double)__fmul_rn(sumu, tp))));
    M.c_taup[o] = tp;
}

}   // namespace dn
