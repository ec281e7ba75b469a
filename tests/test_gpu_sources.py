"""Forward sources applied inside the paired velocity kernel and the stress
kernels (instead of k_inject_v / k_inject_s): bit-identical to the float
restatement for every source type, several sources in one cell (list order),
sources on tile edges, elastic and viscoelastic, the batch fallback to the
injection kernels above 8 source cells per shot, and DN_SRC_IN_KERNEL=0."""
import numpy as np
import pytest

import denise_b200 as dn

import oracles as O
from test_gpu_fused import _case, _check
from test_gpu_parity import gpu_shot

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("styp", [1, 2, 3, 4])
@pytest.mark.parametrize("L", [0, 3])
def test_sources_in_kernel_bitexact(styp, L):
    # two sources share (129, 9); (128, 8) and (130, 17) sit on the edges of 128-column tiles
    p, model, src, rec = _case(nx=260, ny=40, nt=160, styp=styp, src_ij=[(129, 9), (129, 9), (128, 8), (130, 17)],
                               L=L)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    _check(p, model, src, rec, s)


@pytest.mark.parametrize("env", ["default", "off"])
def test_many_source_cells_and_switch(monkeypatch, env):
    """Twelve source cells (above the in-kernel limit: the batch takes the injection
    kernels), or the switch off, and a batch beside a one-source shot: all exact."""
    if env == "off":
        monkeypatch.setenv("DN_SRC_IN_KERNEL", "0")
    cases = [_case(nx=200, ny=50, nt=120, styp=2, src_ij=[(20 + 13 * k, 5 + (k % 4)) for k in range(12)]),
             _case(nx=200, ny=50, nt=120, styp=1, seed=4)]
    pairs = [gpu_shot(*c) for c in cases]
    dn.run([s for _, s in pairs], dn.MODE_FORWARD)
    for c, (m, s) in zip(cases, pairs):
        _check(*c, s)


@pytest.mark.parametrize("quelltypb", [1, 4])
def test_adjoint_sources_of_receivers_sharing_a_cell(quelltypb):
    """Two receivers in one cell: their adjoint forces (QUELLTYPB 1) or pressures
    (QUELLTYPB 4) add one after the other in list order, as the reference's
    loop does, so the gradient is bit-identical to the restatement's."""
    from test_gpu_parity import _residuals, small_case

    p, model, src, rec = small_case(nt=200, store_snapshots=1, nx=80)
    p = p.replace(quelltypb=quelltypb)
    ri = np.concatenate([rec[0], rec[0][:3]]).astype(np.int32)   # the first three receivers twice
    rj = np.concatenate([rec[1], rec[1][:3]]).astype(np.int32)
    rec = (ri, rj)
    ref = O.Restatement(p, model, src, rec, "f")
    ref.forward(store=True)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    rvx, rvy = _residuals(p, s.sections(0), s.sections(1))
    rp = (0.5 * rvx).astype(np.float32) if quelltypb >= 4 else None
    s.set_residuals(rvx, rvy, rp)
    ref.adjoint(rvx, rvy, rp)
    dn.run([s], dn.MODE_ADJOINT)
    s.accumulate_gradient()
    for a, b in zip(m.gradient(), ref.gradient()):
        np.testing.assert_array_equal(a, b)
