"""dn_residual_l2_noalloc (static device scratch, no allocation in the call)
against dn_residual_l2 (allocating) through the C ABI.

Both launch the same kernels, so the adjoint source must be bit-identical and
the misfit equal to 1e-12 relative.  Two different calls in a row check that
nothing from the first call leaks into the second through the shared scratch.
This file is collected last so that it also runs after every other GPU test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_TRACES = 16384
L2_RTOL = 1e-12


def _inputs(ntr, nt, seed):
    rng = np.random.default_rng(seed)
    syn_tm = rng.standard_normal((nt, ntr)).astype(np.float32)
    obs = rng.standard_normal((ntr, nt)).astype(np.float32)
    return syn_tm, obs


def _call(fn, d_syn, d_obs, d_res, ntr, nt, dt, grad_form):
    import torch

    from denise_b200 import _lib

    l2 = ctypes.c_double(-1.0)
    torch.cuda.synchronize()
    _lib.check(fn(d_syn.data_ptr(), d_obs.data_ptr(), d_res.data_ptr(), ntr, nt, ctypes.c_float(dt), grad_form,
                  ctypes.byref(l2)))
    return d_res.cpu().numpy(), l2.value


def test_noalloc_matches_allocating_entry_twice():
    import torch

    from denise_b200 import _lib

    lib = _lib.lib
    cases = [(400, 1500, 4e-4, 1, 11), (MAX_TRACES, 64, 1e-3, 2, 12)]
    for ntr, nt, dt, gf, seed in cases:
        syn_tm, obs = _inputs(ntr, nt, seed)
        d_syn = torch.from_numpy(syn_tm).cuda()
        d_obs = torch.from_numpy(obs).cuda()
        d_res_a = torch.full((ntr, nt), np.nan, dtype=torch.float32, device="cuda")
        d_res_b = torch.full((ntr, nt), np.nan, dtype=torch.float32, device="cuda")
        res_a, l2_a = _call(lib.dn_residual_l2, d_syn, d_obs, d_res_a, ntr, nt, dt, gf)
        res_b, l2_b = _call(lib.dn_residual_l2_noalloc, d_syn, d_obs, d_res_b, ntr, nt, dt, gf)
        np.testing.assert_array_equal(res_b, res_a)
        assert l2_a > 0
        assert abs(l2_b - l2_a) <= L2_RTOL * l2_a, (ntr, l2_a, l2_b)


def test_noalloc_rejects_too_many_traces():
    import torch

    from denise_b200 import _lib

    ntr, nt = MAX_TRACES + 1, 4
    d = torch.zeros((ntr, nt), dtype=torch.float32, device="cuda")
    l2 = ctypes.c_double(0.0)
    rc = _lib.lib.dn_residual_l2_noalloc(d.data_ptr(), d.data_ptr(), d.data_ptr(), ntr, nt, ctypes.c_float(1e-3),
                                         1, ctypes.byref(l2))
    assert rc == _lib.DN_EINVAL
    assert b"static scratch" in _lib.lib.dn_last_error()
