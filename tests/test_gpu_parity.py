"""GPU parity of the B200 propagator against the CPU oracles.

Bar (all on seeded inputs at sizes the CPU oracle finishes in seconds):
* DN_ARITH_EXACT (default) + FP32 snapshots + FP32 accumulation: sections,
  final wavefields, correlation accumulators and gradients are bit-identical
  to the float restatement, which is itself bit-identical to the reference's
  compiled CPU code (tests/test_oracle_pin.py);
* FP64 accumulation: gradients within 1e-6 relative L2 of the float oracle;
* FP16 snapshots: gradients within 1e-3 relative L2 of the FP64 oracle;
* DN_ARITH_FMA: sections within 1e-5 relative L2 of the exact path.
"""
import numpy as np
import pytest

import denise_b200 as dn
from denise_b200 import synth

import oracles as O

pytestmark = pytest.mark.gpu

FL5 = (2.0, 8.0, 25.0, 1.0, 60.0)   # relaxation frequencies for up to 5 mechanisms


def small_case(L=0, fdorder=8, free_surf=1, nt=300, styp=1, nx=64, ny=48, seed=3, **kw):
    p = synth.c0_params(nx=nx, ny=ny, nt=nt, fw=10, L=L, fl=FL5[:L], ts=0.1, fdorder=fdorder,
                        free_surf=free_surf, dtinv=3, seismo=4, quelltypb=1, **kw)
    vp, vs, rho = synth.base_model(p.nx, p.ny, p.dh, seed)
    qp, qs = synth.q_model(p.nx, p.ny, seed)
    sig = synth.ricker_source(p, 40.0)[None, :] * 1e3
    src = (np.array([nx // 2 - 2], np.int32), np.array([3], np.int32), sig, np.array([styp], np.int32),
           np.array([30.0], np.float32))
    nr = (nx - 10) // 4
    rec = (np.arange(5, 5 + 4 * nr, 4).astype(np.int32), np.full(nr, 4, np.int32))
    return p, (vp, vs, rho, qp, qs), src, rec


def gpu_shot(p, model, src, rec):
    m = dn.Model(p, *model[:3], model[3] if p.L else None, model[4] if p.L else None)
    s = dn.Shot(m, src[0], src[1], src[2], rec[0], rec[1], src_type=src[3], src_azi=src[4])
    return m, s


CASES = [
    dict(L=0, fdorder=8, free_surf=1),
    dict(L=0, fdorder=2, free_surf=1),
    dict(L=0, fdorder=4, free_surf=0),
    dict(L=0, fdorder=6, free_surf=1, styp=2),
    dict(L=0, fdorder=10, free_surf=1, styp=3),
    dict(L=0, fdorder=12, free_surf=0, styp=4),
    dict(L=3, fdorder=8, free_surf=1),
    dict(L=1, fdorder=4, free_surf=1),
    dict(L=2, fdorder=12, free_surf=0),
    dict(L=5, fdorder=6, free_surf=1, styp=5),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_forward_bitexact(case):
    p, model, src, rec = small_case(**case)
    ref = O.Restatement(p, model, src, rec, "f")
    ref.forward(store=False)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    for comp in range(5):
        np.testing.assert_array_equal(s.sections(comp), ref.sections(comp), err_msg=f"section {comp}")
    for name, fid in (("vx", 0), ("vy", 1), ("sxx", 2), ("syy", 3), ("sxy", 4)):
        np.testing.assert_array_equal(s.field(fid), ref.field(fid), err_msg=name)


# odd widths: the paired-column kernels own columns (i, i+1) with i odd, so the last
# column of an odd NX is computed alone and column NX+1 (halo) must stay zero;
# widths just above a tile (128 columns) leave most threads of the last tile idle
ODD = [dict(L=0, fdorder=8, nx=63, ny=41), dict(L=0, fdorder=12, nx=131, ny=37, free_surf=0),
       dict(L=3, fdorder=8, nx=129, ny=45), dict(L=0, fdorder=2, nx=33, ny=30, styp=2),
       dict(L=2, fdorder=6, nx=65, ny=33, styp=3)]


@pytest.mark.parametrize("case", ODD, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_forward_bitexact_odd_widths(case):
    p, model, src, rec = small_case(**case)
    ref = O.Restatement(p, model, src, rec, "f")
    ref.forward(store=False)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    for comp in range(5):
        np.testing.assert_array_equal(s.sections(comp), ref.sections(comp), err_msg=f"section {comp}")
    for name, fid in (("vx", 0), ("vy", 1), ("sxx", 2), ("syy", 3), ("sxy", 4)):
        np.testing.assert_array_equal(s.field(fid), ref.field(fid), err_msg=name)


@pytest.mark.parametrize("case", [dict(L=0, fdorder=8), dict(L=3, fdorder=8), dict(L=0, fdorder=4, free_surf=0)],
                         ids=["elastic8", "visco8", "elastic4-nofs"])
def test_plain_path_bitexact(case):
    p, model, src, rec = small_case(**case)
    ref = O.Restatement(p, model, src, rec, "f")
    ref.forward(store=False)
    m, s = gpu_shot(p, model, src, rec)
    dn.run_plain(s, dn.MODE_FORWARD)
    np.testing.assert_array_equal(s.sections(dn.SEC_VY), ref.sections(1))
    np.testing.assert_array_equal(s.field(2), ref.field(2))


def _residuals(p, syn_vx, syn_vy):
    # L2 residual of calc_res (GRAD_FORM 1): time-integrated, reversed, first sample zeroed,
    # against zero "observed" data scaled from the synthetics
    out = []
    for syn in (syn_vx, syn_vy):
        obs = 0.7 * syn
        d = syn - obs
        d[:, 0] = 0.0
        integ = np.zeros_like(d)
        acc = np.zeros(d.shape[0], np.float32)
        for t in range(p.nt):
            acc = (acc + np.float32(p.dt) * d[:, t]).astype(np.float32)
            integ[:, p.nt - 1 - t] = acc
        out.append(integ.astype(np.float32))
    return out


@pytest.mark.parametrize("L,nx", [(0, 64), (3, 64), (0, 63), (3, 129)])
def test_gradient_bitexact(L, nx):
    p, model, src, rec = small_case(L=L, store_snapshots=1, nx=nx)
    ref = O.Restatement(p, model, src, rec, "f")
    ref.forward(store=True)
    rvx, rvy = _residuals(p, ref.sections(0), ref.sections(1))
    ref.adjoint(rvx, rvy, None)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    np.testing.assert_array_equal(s.sections(0), ref.sections(0))
    s.set_residuals(rvx, rvy, None)
    dn.run([s], dn.MODE_ADJOINT)
    for fid in (7, 8, 9):
        np.testing.assert_array_equal(s.field(fid), ref.field(fid), err_msg=f"accumulator {fid}")
    s.accumulate_gradient()
    for a, b, n in zip(m.gradient(), ref.gradient(), ("vp", "vs", "rho")):
        np.testing.assert_array_equal(a, b, err_msg=f"gradient {n}")


def test_gradient_fp64_accumulation():
    p, model, src, rec = small_case(store_snapshots=1, grad_accum=dn.ACC_F64)
    ref = O.Restatement(p, model, src, rec, "f")
    ref.forward(store=True)
    rvx, rvy = _residuals(p, ref.sections(0), ref.sections(1))
    ref.adjoint(rvx, rvy, None)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    s.set_residuals(rvx, rvy, None)
    dn.run([s], dn.MODE_ADJOINT)
    s.accumulate_gradient()
    for a, b in zip(m.gradient(), ref.gradient()):
        assert O.rel_l2(a, b) < 1e-6


@pytest.mark.parametrize("prec,tol", [(dn.SNAP_F16, 1e-3), (dn.SNAP_BF16, 1e-2)], ids=["fp16", "bf16"])
def test_gradient_half_snapshots_vs_fp64(prec, tol):
    p, model, src, rec = small_case(store_snapshots=1, snap_precision=prec, grad_accum=dn.ACC_F64, nt=400)
    ref = O.Restatement(p, model, src, rec, "d")
    ref.forward(store=True)
    rvx, rvy = _residuals(p, ref.sections(0).astype(np.float32), ref.sections(1).astype(np.float32))
    ref.adjoint(rvx, rvy, None)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    s.set_residuals(rvx, rvy, None)
    dn.run([s], dn.MODE_ADJOINT)
    s.accumulate_gradient()
    errs = [O.rel_l2(a, b) for a, b in zip(m.gradient(), ref.gradient())]
    assert max(errs) < tol, errs


def test_fma_mode_close():
    p, model, src, rec = small_case(nt=400)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s])
    exact = s.sections(1)
    p2 = p.replace(arith=dn.ARITH_FMA)
    m2, s2 = gpu_shot(p2, model, src, rec)
    dn.run([s2])
    assert O.rel_l2(s2.sections(1), exact) < 1e-5


def test_batch_uneven_equals_individual():
    cases = [small_case(nx=64, ny=48, nt=300, seed=1), small_case(nx=80, ny=40, nt=250, seed=2),
             small_case(nx=50, ny=60, nt=320, seed=5)]
    shots, refs = [], []
    for p, model, src, rec in cases:
        m, s = gpu_shot(p, model, src, rec)
        shots.append((m, s))
        r = O.Restatement(p, model, src, rec, "f")
        r.forward()
        refs.append(r)
    dn.run([s for _, s in shots])
    for (m, s), r in zip(shots, refs):
        np.testing.assert_array_equal(s.sections(0), r.sections(0))
        np.testing.assert_array_equal(s.field(3), r.field(3))
    # a second run of the same batch replays the cached graph and must reproduce itself
    first = [s.sections(1) for _, s in shots]
    dn.run([s for _, s in shots])
    for (m, s), f in zip(shots, first):
        np.testing.assert_array_equal(s.sections(1), f)


def test_unstable_model_reports_status():
    p, model, src, rec = small_case(nt=50)
    vp = model[0].copy()
    vp[p.nx // 2 - 1, p.ny // 2 - 1] = np.nan   # a NaN planted in the model on the host
    m, s = gpu_shot(p, (vp,) + model[1:], src, rec)
    with pytest.raises(dn.DeniseError) as e:
        dn.run([s])
    assert e.value.code == -3


@pytest.mark.skipif(not O.reference_available(), reason="reference build not present")
def test_forward_matches_reference_build():
    p, model, src, rec = small_case(L=0, nt=200)

    rx, ry = O.run_isolated(O.reference_forward_sections, p, model, src, rec)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s])
    np.testing.assert_array_equal(s.sections(0), rx)
    np.testing.assert_array_equal(s.sections(1), ry)


@pytest.mark.parametrize("prec", [dn.SNAP_F16, dn.SNAP_BF16], ids=["fp16", "bf16"])
def test_half_snapshots_of_tiny_wavefields_stay_finite(prec):
    """A source 1e-40 times weaker: every snapshot tile's maximum is far below
    2^-111, where a per-tile scale without a floor would overflow on inversion."""
    p, model, src, rec = small_case(store_snapshots=1, snap_precision=prec, nt=300)
    src = (src[0], src[1], src[2] * np.float32(1e-40)) + src[3:]
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    syn = [s.sections(c) for c in (0, 1)]
    s.set_residuals(syn[0], syn[1], None)
    dn.run([s], dn.MODE_ADJOINT)
    s.accumulate_gradient()
    for g in m.gradient():
        assert np.all(np.isfinite(g))


def _encode_tiles(x, bx, zch, prec):
    """The half-precision snapshot rule on a [nx][ny] field: tiles of bx columns
    x zch rows, per tile s = 2^max(e - 15, -126) with max|x| = f 2^e, f in
    [0.5, 1) (s = 1 for an all-zero tile), stored as RN(x / s) in FP16 or BF16
    and decoded as float(h) * s."""
    out = np.empty_like(x)
    for i0 in range(0, x.shape[0], bx):
        for j0 in range(0, x.shape[1], zch):
            t = x[i0:i0 + bx, j0:j0 + zch]
            am = np.float32(np.max(np.abs(t)))
            sc = np.float32(1.0)
            if am > 0 and np.isfinite(am):
                e = int(np.frexp(am)[1])
                sc = np.ldexp(np.float32(1.0), max(e - 15, -126)).astype(np.float32)
            y = (t * (np.float32(1.0) / sc)).astype(np.float32)
            if prec == dn.SNAP_F16:
                h = y.astype(np.float16).astype(np.float32)
            else:   # bfloat16: round to nearest even on the upper 16 bits
                u = y.view(np.uint32).astype(np.uint64)
                h = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32).view(np.float32)
            out[i0:i0 + bx, j0:j0 + zch] = h * sc
    return out


@pytest.mark.parametrize("prec", [dn.SNAP_F16, dn.SNAP_BF16], ids=["fp16", "bf16"])
@pytest.mark.parametrize("zch", [4, 8, 16, 5], ids=["rows4", "rows8", "rows16", "rows5"])
def test_half_snapshot_encoding(prec, zch):
    """Decoded FP16/BF16 snapshots equal the per-tile power-of-two encoding of
    the FP32 snapshots bit for bit, on a grid with partial tiles in x and z and
    for tile heights served by the single-pass store (up to 8 rows) and by the
    general one."""
    from denise_b200 import tune

    kw = dict(nx=150, ny=45, nt=120, store_snapshots=1)
    p32, model, src, rec = small_case(**kw, snap_precision=dn.SNAP_F32)
    ph, _, _, _ = small_case(**kw, snap_precision=prec)
    tune.set_rule(ph.fdorder, ph.L, 0, 1 << 40, 128, zch)
    try:
        bx, z = tune.tile_for(ph)
        assert (bx, z) == (128, zch)
        m32, s32 = gpu_shot(p32, model, src, rec)
        mh, sh = gpu_shot(ph, model, src, rec)
        dn.run([s32, sh], dn.MODE_FORWARD)
    finally:
        tune.clear_rules()
    nsnap = -(-p32.nt // p32.dtinv)
    for k in (0, nsnap // 2, nsnap - 1):
        for f in range(5):
            ref = _encode_tiles(s32.snapshot(k, f), bx, zch, prec)
            np.testing.assert_array_equal(sh.snapshot(k, f), ref, err_msg=f"snapshot {k} field {f}")


@pytest.mark.parametrize("L,prec,ckpt", [(0, dn.SNAP_F32, 39), (2, dn.SNAP_F32, 27), (0, dn.SNAP_F16, 63)],
                         ids=["elastic-fp32", "visco-fp32-odd-segments", "elastic-fp16"])
def test_checkpointed_adjoint_equals_stored_snapshots(L, prec, ckpt):
    """Checkpointed adjoint (segments recomputed from saved states) gives the
    bit-identical gradient of the run that stores every snapshot."""
    p, model, src, rec = small_case(L=L, store_snapshots=1, snap_precision=prec, nt=300)   # DTINV 3
    out = []
    for cs in (0, ckpt):
        m, s = gpu_shot(p.replace(ckpt_steps=cs), model, src, rec)
        dn.run([s], dn.MODE_FORWARD)
        syn = [s.sections(c) for c in (0, 1)]
        rvx, rvy = _residuals(p, syn[0], syn[1])
        s.set_residuals(rvx, rvy, None)
        dn.run([s], dn.MODE_ADJOINT)
        s.accumulate_gradient()
        out.append((syn, m.gradient(), [s.field(f) for f in (7, 8, 9)]))
        s.close()
        m.close()
    (sa, ga, fa), (sb, gb, fb) = out
    for x, y in zip(sa, sb):
        np.testing.assert_array_equal(x, y)
    for x, y in zip(ga + tuple(fa), gb + tuple(fb)):
        np.testing.assert_array_equal(x, y)


def _ref_grad_ep(p, model, src, rec, rvx, rvy, c):
    r = O.Reference(p, model, src, rec, mode_global=1)
    r.run(0)
    r.set_residuals(rvx, rvy, None)
    r.run(1)
    return r.ass_grad_ep(*c)


@pytest.mark.skipif(not O.reference_available(), reason="reference build not present")
@pytest.mark.parametrize("ep", [1, 3])
def test_energy_preconditioned_gradient_matches_reference(ep):
    """grad_obj_psv.c:218-240: per-shot gradient divided by (We + 0.005 max We) C^2;
    EPRECOND 1 bit-identical; EPRECOND 3 within 1e-6 (device and host double asinh)."""
    p, model, src, rec = small_case(store_snapshots=1, eprecond=ep, nt=300)
    c = (float(np.mean(model[0])), float(np.mean(model[1])), float(np.mean(model[2])))
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    rvx, rvy = _residuals(p, s.sections(0), s.sections(1))
    s.set_residuals(rvx, rvy, None)
    dn.run([s], dn.MODE_ADJOINT)
    s.accumulate_gradient_precond(*c)
    ours = m.gradient()
    ref = O.run_isolated(_ref_grad_ep, p, model, src, rec, rvx, rvy, c)
    for a, b, n in zip(ours, ref, ("vp", "vs", "rho")):
        if ep == 1:
            np.testing.assert_array_equal(a, b, err_msg=n)
        else:
            assert O.rel_l2(a, b) < 1e-6, (n, O.rel_l2(a, b))


@pytest.mark.parametrize("kernels", ["one-column", "tma", "vpipe"])
@pytest.mark.parametrize("case", [dict(L=0, fdorder=8, nx=63), dict(L=3, fdorder=8), dict(L=0, fdorder=12, free_surf=0)],
                         ids=["elastic8-odd", "visco8", "elastic12-nofs"])
def test_alternative_kernels_bitexact(monkeypatch, kernels, case):
    """The kernels beside the default paired-column ones: the one-column
    register-streaming kernels (DN_PACK=0), the bulk-copy row pipeline
    (DN_KERNEL=tma) and the warp-specialised velocity pipeline (DN_VPIPE=1),
    all bit-identical to the reference."""
    if kernels == "one-column":
        monkeypatch.setenv("DN_PACK", "0")
    elif kernels == "vpipe":
        monkeypatch.setenv("DN_VPIPE", "1")
    else:
        monkeypatch.setenv("DN_KERNEL", "tma")
    p, model, src, rec = small_case(**case)
    ref = O.Restatement(p, model, src, rec, "f")
    ref.forward(store=False)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    for comp in range(2):
        np.testing.assert_array_equal(s.sections(comp), ref.sections(comp), err_msg=f"section {comp}")
    np.testing.assert_array_equal(s.field(2), ref.field(2))


@pytest.mark.parametrize("L,ckpt", [(0, 39), (2, 27)], ids=["elastic", "visco-odd-segments"])
def test_checkpointed_batch_equals_single_shots(L, ckpt):
    """Checkpointed shots run as one batch (segments of all shots in the same
    launches; different models and source positions) give, shot for shot, the
    bit-identical sections and gradients of stored-snapshot runs of each shot alone."""
    cases = [small_case(L=L, store_snapshots=1, nt=300, seed=sd, nx=72) for sd in (3, 4, 6)]
    cases = [(p, model, (src[0] + 5 * k,) + tuple(src[1:]), rec) for k, (p, model, src, rec) in enumerate(cases)]
    want = []
    for p, model, src, rec in cases:
        m, s = gpu_shot(p, model, src, rec)
        dn.run([s], dn.MODE_FORWARD)
        syn = [s.sections(c) for c in (0, 1)]
        rvx, rvy = _residuals(p, syn[0], syn[1])
        s.set_residuals(rvx, rvy, None)
        dn.run([s], dn.MODE_ADJOINT)
        s.accumulate_gradient()
        want.append((syn, m.gradient(), (rvx, rvy)))
        s.close()
        m.close()
    pairs = [gpu_shot(p.replace(ckpt_steps=ckpt), model, src, rec) for p, model, src, rec in cases]
    shots = [s for _, s in pairs]
    dn.run(shots, dn.MODE_FORWARD)
    for (m, s), (syn, _, (rvx, rvy)) in zip(pairs, want):
        for c in (0, 1):
            np.testing.assert_array_equal(s.sections(c), syn[c])
        s.set_residuals(rvx, rvy, None)
    dn.run(shots, dn.MODE_ADJOINT)
    for (m, s), (_, g, _) in zip(pairs, want):
        s.accumulate_gradient()
        for x, y in zip(m.gradient(), g):
            np.testing.assert_array_equal(x, y)
        s.close()
        m.close()


@pytest.mark.parametrize("rows", [0, 7, 32])
@pytest.mark.parametrize("fdorder,nx,ny", [(8, 300, 70), (12, 257, 41), (2, 131, 33), (6, 64, 48)])
def test_vpipe_forward_and_gradient_bitexact(monkeypatch, rows, fdorder, nx, ny):
    """The warp-specialised velocity pipeline over strip heights (automatic, 7 and
    32 rows: strips that end inside the grid, one strip taller than the grid),
    several tiles across (nx > 256, odd nx) and every stencil reach: forward
    sections and the adjoint's gradient bit-identical to the oracle."""
    monkeypatch.setenv("DN_VPIPE", "1")
    if rows:
        monkeypatch.setenv("DN_VPIPE_ROWS", str(rows))
    p, model, src, rec = small_case(fdorder=fdorder, nx=nx, ny=ny, nt=200, store_snapshots=1)
    ref = O.Restatement(p, model, src, rec, "f")
    ref.forward(store=True)
    m, s = gpu_shot(p, model, src, rec)
    dn.run([s], dn.MODE_FORWARD)
    for comp in range(2):
        np.testing.assert_array_equal(s.sections(comp), ref.sections(comp), err_msg=f"section {comp}")
    rvx, rvy = _residuals(p, s.sections(0), s.sections(1))
    s.set_residuals(rvx, rvy, None)
    ref.adjoint(rvx, rvy, None)
    dn.run([s], dn.MODE_ADJOINT)
    s.accumulate_gradient()
    for a, b in zip(m.gradient(), ref.gradient()):
        np.testing.assert_array_equal(a, b)
