"""ORACLE / TEST INFRASTRUCTURE - never part of the product.

numpy restatement of the reference's FWI optimisers as FWI_PSV.c:637-676 calls
them on the preconditioned, stacked gradients of one iteration:

* GRAD_METHOD 2 (L-BFGS): the LBFGS_pointer rule of FWI_PSV.c:452-466,
  store_LBFGS_PSV (src/PSV/store_LBFGS_PSV.c:37-206: gradients normalised by
  the model averages C_vp, C_vs, C_rho; y = normalised gradient minus the
  previous one, s = model minus the previous one, in the class order rho, vs,
  vp), LBFGS (src/LBFGS.c:26-93: gamma from the current pair, rho_k = 1/(y.s)
  or 0, the two loops over every slot k = NLBFGS..1 and 1..NLBFGS) and
  extract_LBFGS_PSV (src/PSV/extract_LBFGS_PSV.c:31-76: the direction r times
  C; in the first iteration the normalised gradient itself).
* GRAD_METHOD 1 (PCG): descent (src/descent.c), store_PCG_PSV, PCG
  (src/PCG.c:23-100: one beta per class, PCG_BETA 1 Fletcher-Reeves,
  2 Polak-Ribiere with reset, 3 Hestenes-Stiefel, 4 Dai-Yuan), extract_PCG_PSV,
  descent.

Vectors are float32 as in the reference.  `dots` selects the dot products:
"float" accumulates float products in a float in index order, as dotp.c and
PCG.c do (bit-identical to the reference, pinned in tests/test_optim.py);
"fp64" sums the exact double products in double and rounds the sum to float,
the device optimiser's arithmetic.  Every scalar the reference keeps in a
float (gamma, rho_k, alpha_k, beta) is rounded to float here too.

Arrays are [nx][ny] float32 (file order).  State persists between calls.
"""
import numpy as np

f32 = np.float32


def _dot(a, b, dots):
    if dots == "float":
        acc = f32(0.0)
        p = (a * b).astype(np.float32)
        for v in p:
            acc = f32(acc + v)
        return acc
    return f32(np.dot(a.astype(np.float64), b.astype(np.float64)))


class ReferenceOptimizer:
    def __init__(self, method, nx, ny, nlbfgs=20, pcg_beta=2, dots="fp64"):
        self.method, self.nx, self.ny, self.nlbfgs, self.pcg_beta, self.dots = method, nx, ny, nlbfgs, pcg_beta, dots
        self.n = 3 * nx * ny
        self.reset()
        self.gradp_old = None     # JACOBIAN_p*.old: normalised gradients of the previous iteration (rho, vs, vp)
        self.model_old = None     # JACOBIAN_p_{vp,vs,mrho}.old (rho, vs, vp)
        self.files = {}

    def reset(self):
        n = 3 * self.nx * self.ny
        if self.method == 2:
            self.y = np.zeros((self.nlbfgs, n), np.float32)
            self.s = np.zeros((self.nlbfgs, n), np.float32)
            self.ptr = 1
        else:
            self.old = np.zeros(n, np.float32)
            self.dir = np.zeros(n, np.float32)

    def step(self, it, c, model, grads):
        """One iteration; model = (vp, vs, rho), grads = (g_vp, g_vs, g_rho).
        Returns the direction (d_vp, d_vs, d_rho), all [nx][ny] float32."""
        model = [np.asarray(a, np.float32).ravel() for a in model]
        grads = [np.asarray(a, np.float32).ravel() for a in grads]
        shp = (self.nx, self.ny)
        if self.method == 2:
            return [d.reshape(shp) for d in self._lbfgs(it, c, model, grads)]
        return [d.reshape(shp) for d in self._pcg(grads)]

    def _lbfgs(self, it, c, model, grads):
        if it > 2:
            self.ptr += 1
        if self.ptr > self.nlbfgs:
            self.ptr = 1
        cvp, cvs, crho = f32(c[0]), f32(c[1]), f32(c[2])
        gn = [(cvp * grads[0]).astype(np.float32), (cvs * grads[1]).astype(np.float32),
              (crho * grads[2]).astype(np.float32)]
        q = np.concatenate([gn[2], gn[1], gn[0]])
        m = np.concatenate([model[2], model[1], model[0]])
        if it > 1:
            k = self.ptr - 1
            self.y[k] = (q - self.gradp_old).astype(np.float32)
            self.s[k] = (m - self.model_old).astype(np.float32)
            sn = _dot(self.y[k], self.s[k], self.dots)
            sd = _dot(self.y[k], self.y[k], self.dots)
            gamma = f32(sn / sd)
            rho = np.zeros(self.nlbfgs, np.float32)
            for k in range(self.nlbfgs):
                sn = _dot(self.y[k], self.s[k], self.dots)
                rho[k] = f32(1.0 / float(sn)) if abs(float(sn)) > 0.0 else f32(0.0)
            alpha = np.zeros(self.nlbfgs, np.float32)
            qq = q.copy()
            for k in range(self.nlbfgs - 1, -1, -1):
                alpha[k] = f32(rho[k] * _dot(self.s[k], qq, self.dots))
                qq = (qq - (alpha[k] * self.y[k]).astype(np.float32)).astype(np.float32)
            r = (gamma * qq).astype(np.float32)
            for k in range(self.nlbfgs):
                beta = f32(rho[k] * _dot(self.y[k], r, self.dots))
                r = (r + (self.s[k] * f32(alpha[k] - beta)).astype(np.float32)).astype(np.float32)
            nn = self.nx * self.ny
            d = [(r[2 * nn:] * cvp).astype(np.float32), (r[nn:2 * nn] * cvs).astype(np.float32),
                 (r[:nn] * crho).astype(np.float32)]
        else:
            d = gn
        self.gradp_old = q
        self.model_old = m
        self.files = {"p": gn[0], "p_u": gn[1], "p_rho": gn[2], "p_vp": model[0], "p_vs": model[1],
                      "p_mrho": model[2], "c": d[0], "c_u": d[1], "c_rho": d[2]}
        return d

    def _pcg(self, grads):
        new = np.concatenate([-g for g in grads]).astype(np.float32)
        nn = self.nx * self.ny
        for k in range(3):
            sl = slice(k * nn, (k + 1) * nn)
            a, o, d = new[sl], self.old[sl], self.dir[sl]
            diff = (a - o).astype(np.float32)
            if self.pcg_beta == 1:
                bz, bn = _dot(a, a, self.dots), _dot(o, o, self.dots)
            elif self.pcg_beta == 2:
                bz, bn = _dot(a, diff, self.dots), _dot(o, o, self.dots)
            elif self.pcg_beta == 3:
                bz, bn = -_dot(a, diff, self.dots), _dot(d, diff, self.dots)
            else:
                bz, bn = -_dot(a, a, self.dots), _dot(d, diff, self.dots)
            beta = f32(bz / bn) if bn != 0.0 else f32(0.0)
            if beta < 0.0 and self.pcg_beta == 2:
                beta = f32(0.0)
            self.dir[sl] = (a + (beta * d).astype(np.float32)).astype(np.float32)
        self.old = new
        return [(-self.dir[k * nn:(k + 1) * nn]).astype(np.float32) for k in range(3)]
