/*
 * ORACLE / TEST INFRASTRUCTURE - never part of the product.
 *
 * CPU restatement of the reference's single-shot P-SV scheme (forward,
 * adjoint, cross-correlation, gradient assembly) in two precisions:
 *   *_f : float, with the reference's double promotions spelled out, so the
 *         result is bit-identical to the reference's CPU path;
 *   *_d : double everywhere (the FP64 oracle used to state the error of every
 *         float result).
 * Parameters: ip[] = nx ny nt fdorder maxrelerror free_surf fw L quelltypb
 *             dtinv seismo eprecond honor_q
 *             fp[] = dh dt damping fpml npower k_max_pml ts fl[0..4]
 * Arrays: models in file order (x-major, z contiguous), sections [ntr][nt].
 */
#ifndef DN_PSV_ORACLE_H
#define DN_PSV_ORACLE_H

typedef struct or_ctx_f or_ctx_f;
typedef struct or_ctx_d or_ctx_d;

#define OR_DECL(SFX, REAL)                                                                                     \
    or_ctx##SFX *or_create##SFX(const int *ip, const float *fp, const float *vp, const float *vs,              \
                                const float *rho, const float *qp, const float *qs, int nsrc, const int *src_i, \
                                const int *src_j, const int *src_type, const float *src_azi,                   \
                                const float *signals, int ntr, const int *rec_i, const int *rec_j);            \
    void or_destroy##SFX(or_ctx##SFX *c);                                                                      \
    int or_forward##SFX(or_ctx##SFX *c, int store, int nt_stop);                                               \
    int or_adjoint##SFX(or_ctx##SFX *c, const float *res_vx, const float *res_vy, const float *res_p);         \
    int or_get_sections##SFX(or_ctx##SFX *c, int comp, REAL *out);                                             \
    int or_get_field##SFX(or_ctx##SFX *c, int field, REAL *out);                                               \
    int or_get_gradient##SFX(or_ctx##SFX *c, REAL *gvp, REAL *gvs, REAL *grho);                                \
    int or_get_setup##SFX(or_ctx##SFX *c, int which, REAL *out);

OR_DECL(_f, float)
OR_DECL(_d, double)

#endif
