"""The library's device block cache: memory freed by a shot stays cached,
counts as free in dn_device_memory and serves the next shot; a reused block
carries nothing from its last owner into the next run; dn_device_trim frees
the cache; DN_POOL=0 (plain cudaMalloc) gives the same results."""
import os
import subprocess
import sys

import numpy as np
import pytest

import denise_b200 as dn

from test_gpu_parity import gpu_shot, small_case

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CASE = dict(nx=160, ny=96, nt=200, store_snapshots=1, snap_precision=dn.SNAP_F16)


def _sections_and_gradient():
    """Sections vx, vy and the three gradients of a forward + adjoint of one shot."""
    p, model, src, rec = small_case(**CASE)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    sec = [s.sections(c) for c in (0, 1)]
    s.set_residuals(sec[0], sec[1], None)
    dn.run([s], dn.MODE_ADJOINT)
    s.accumulate_gradient()
    g = m.gradient()
    s.close()
    m.close()
    return list(sec) + list(g)


def test_pool_reuse_reporting_and_trim():
    free0, total = dn.device_memory(0)
    out = _sections_and_gradient()
    free1, _ = dn.device_memory(0)
    # the freed shot and model are cached now, reported as free
    assert free1 >= free0 - (256 << 20), (free0, free1)
    # a dirty block from the pool must not change the next run
    p, model, src, rec = small_case(**CASE)
    junk = dn.Shot(dn.Model(p, *model[:3]), src[0], src[1], src[2] * np.float32(1e3), rec[0], rec[1])
    dn.run([junk], dn.MODE_FORWARD)
    junk.close()
    junk.model.close()
    for a, b in zip(out, _sections_and_gradient()):
        np.testing.assert_array_equal(a, b)
    dn.device_trim(0)
    free2, _ = dn.device_memory(0)
    assert abs(free2 - free1) < (256 << 20), (free1, free2)


def test_plain_cudamalloc_gives_the_same_results():
    out = _sections_and_gradient()
    root = os.path.dirname(HERE)
    code = ("import sys, numpy as np; sys.path[:0] = [%r, %r, %r]; import test_gpu_alloc as t; "
            "np.save(sys.argv[1], np.stack([a.ravel()[:4096] for a in t._sections_and_gradient()]))"
            % (HERE, root, os.path.join(root, "denise-black-edition_b200")))
    path = os.path.join(os.environ.get("TMPDIR", "/tmp"), "dn_pool_off.npy")
    env = dict(os.environ, DN_POOL="0")
    subprocess.run([sys.executable, "-c", code, path], check=True, env=env, cwd=HERE, timeout=300)
    ref = np.load(path)
    np.testing.assert_array_equal(ref, np.stack([a.ravel()[:4096] for a in out]))
