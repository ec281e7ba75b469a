"""The fused elastic time step (DN_KERN_FUSED): velocity, force sources,
stress, explosive source and free surface of a step in one kernel, the fields
alternating between two buffers.  Bar: sections and final wavefields
bit-identical to the float restatement (itself pinned to the reference), over
every stencil reach, source type, free surface on and off, odd widths, several
tiles across and down (sources on the tile seams, whose velocities the
neighbouring tile recomputes), NT odd and even, mixed batches, the run queue
and partial step ranges."""
import numpy as np
import pytest

import denise_b200 as dn
from denise_b200 import _lib, synth, tune

import oracles as O
from test_gpu_parity import gpu_shot, small_case

pytestmark = pytest.mark.gpu


def _case(fdorder=8, nx=300, ny=70, nt=200, styp=1, src_ij=None, free_surf=1, seed=3, L=0, **kw):
    p, model, src, rec = small_case(L=L, fdorder=fdorder, nx=nx, ny=ny, nt=nt, styp=styp, free_surf=free_surf,
                                    seed=seed, **kw)
    if src_ij is not None:
        i, j = zip(*src_ij)
        n = len(i)
        sig = np.repeat(src[2][:1], n, axis=0) * (1.0 + 0.1 * np.arange(n, dtype=np.float32))[:, None]
        src = (np.array(i, np.int32), np.array(j, np.int32), sig.astype(np.float32), np.full(n, styp, np.int32),
               np.full(n, 30.0, np.float32))
    return p, model, src, rec


def _check(p, model, src, rec, shot):
    ref = O.Restatement(p, model, src, rec, "f")
    ref.forward(store=False)
    for comp in range(5):
        np.testing.assert_array_equal(shot.sections(comp), ref.sections(comp), err_msg=f"section {comp}")
    for name, fid in (("vx", 0), ("vy", 1), ("sxx", 2), ("syy", 3), ("sxy", 4)):
        np.testing.assert_array_equal(shot.field(fid), ref.field(fid), err_msg=name)


def _fused_launches(nt):
    """The fused step is one launch per step besides the receivers' (graph chunks of 50
    steps, the last one replayed whole, plus one step-counter launch per chunk); the
    separate kernels take at least four."""
    _, nl = dn.last_run_stats()
    chunk = min(50, nt)
    return nl <= ((nt + chunk - 1) // chunk) * (2 * chunk + 1)


# W = 2 * 64 - 2H owned columns per tile: 124 (R 1, 2), 120 (R 3, 4), 116 (R 5, 6)
SEAM = {2: 125, 4: 125, 6: 121, 8: 121, 10: 117, 12: 117}


@pytest.mark.parametrize("rows", [0, 9, 16])
@pytest.mark.parametrize("fdorder", [2, 4, 6, 8, 10, 12])
def test_fused_forward_bitexact(monkeypatch, fdorder, rows):
    """Every stencil reach, tiles of 9 and 16 rows and the default; sources on the
    column seam between two tiles and on a row seam."""
    monkeypatch.setenv("DN_FUSED", "1")
    if rows:
        monkeypatch.setenv("DN_FUSED_ROWS", str(rows))
    zc = rows if rows else 40   # a row seam when the tiles are `rows` tall (else just a row)
    seam = SEAM[fdorder]
    p, model, src, rec = _case(fdorder=fdorder, src_ij=[(seam, 5), (seam - 1, zc + 1), (seam - 2, zc)],
                               styp=1 + fdorder // 2 % 3)
    m, s = gpu_shot(p, model, src, rec)
    assert s.kernel()[1]
    dn.run([s], dn.MODE_FORWARD)
    assert _fused_launches(p.nt)
    _check(p, model, src, rec, s)


@pytest.mark.parametrize("case", [dict(nx=63, ny=41, nt=201), dict(nx=131, ny=37, free_surf=0, fdorder=12, nt=150),
                                  dict(nx=33, ny=30, styp=2, fdorder=2), dict(nx=250, ny=23, fdorder=8, nt=61, rows=5),
                                  dict(nx=245, ny=64, styp=4, free_surf=0, nt=120),
                                  dict(nx=140, ny=31, fdorder=12, nt=90, rows=3)],
                         ids=["odd63", "nofs131-fd12", "fd2-force", "rows-of-five", "azimuth-nofs", "rows-min-fd12"])
def test_fused_edges_bitexact(monkeypatch, case):
    """Odd widths (the lone last column), tiles R + 1 rows tall (the least the free
    surface allows: 3 asks for less and gets 7 at FDORDER 12), NT odd and even,
    QUELLTYP 4 without free surface."""
    monkeypatch.setenv("DN_FUSED", "1")
    case = dict(case)
    rows = case.pop("rows", 0)
    if rows:
        monkeypatch.setenv("DN_FUSED_ROWS", str(rows))
    p, model, src, rec = _case(**case)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    assert _fused_launches(p.nt)
    _check(p, model, src, rec, s)


def test_fused_by_kernel_rule_and_mixed_batch():
    """The variant comes from a kernel rule too; a batch mixing fused shots, a
    snapshot-storing shot and a moment-tensor shot (both take the separate kernels)
    gives every shot the restatement's sections and final fields."""
    tune.clear_rules()
    try:
        tune.set_rule(8, 0, 0, 1 << 40, 128, 8, store=0, variant=_lib.KERN_FUSED)
        specs = [dict(seed=3), dict(seed=4, store_snapshots=1), dict(seed=5, nt=150), dict(seed=6, styp=5)]
        cases = [_case(nx=200, ny=60, **sp) for sp in specs]
        pairs = [gpu_shot(p, model, src, rec) for p, model, src, rec in cases]
        assert [s.kernel() for _, s in pairs] == [(_lib.KERN_FUSED, True), (_lib.KERN_PAIRED, False),
                                                  (_lib.KERN_FUSED, True), (_lib.KERN_FUSED, False)]
        dn.run([s for _, s in pairs], dn.MODE_FORWARD)
        for (p, model, src, rec), (m, s) in zip(cases, pairs):
            _check(p, model, src, rec, s)
            s.close()
            m.close()
    finally:
        tune.clear_rules()


def test_fused_partial_steps(monkeypatch):
    """dn_run_steps over partial ranges takes the separate kernels on the primary
    buffers; a full range after them takes the fused step; both agree with the
    restatement."""
    monkeypatch.setenv("DN_FUSED", "1")
    p, model, src, rec = _case(nx=180, ny=50, nt=160)
    m, s = gpu_shot(p, model, src, rec)
    s.run_steps(dn.MODE_FORWARD, 1, 57)
    s.run_steps(dn.MODE_FORWARD, 58, p.nt)
    _check(p, model, src, rec, s)
    s.run_steps(dn.MODE_FORWARD, 1, p.nt)
    _check(p, model, src, rec, s)


def test_fused_in_the_serving_mix(monkeypatch):
    """Continuous batching with fused forward shots and separate-kernel gradient
    shots in the same queues, joining while others run: identical to each request
    alone."""
    monkeypatch.setenv("DN_FUSED", "1")
    import test_gpu_serve
    test_gpu_serve.test_results_are_the_same_alone_and_in_the_mix()


def test_fused_fma_mode_close(monkeypatch):
    """DN_ARITH_FMA through the fused step: within 1e-5 of the exact sections."""
    monkeypatch.setenv("DN_FUSED", "1")
    p, model, src, rec = _case(nx=200, ny=60)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    exact = s.sections(dn.SEC_VY)
    p2 = p.replace(arith=dn.ARITH_FMA)
    m2, s2 = gpu_shot(p2, model, src, rec)
    dn.run([s2], dn.MODE_FORWARD)
    assert O.rel_l2(s2.sections(dn.SEC_VY), exact) < 1e-5
