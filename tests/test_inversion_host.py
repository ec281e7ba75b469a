"""Host side of the parameter-file FWI driver (denise_b200/inversion.py),
without a GPU: the test-shot selection of grad_obj_psv.c:179 / obj_psv.c:50,
the propagator parameters of a MODE 1 file, the refusal of switches the GPU
path does not provide, and the per-iteration model file names."""
import numpy as np
import pytest

import inp_case
from denise_b200 import inversion, io, workflow


@pytest.mark.parametrize("ts,nshots,want", [((1, 1, 1), 3, [0]), ((1, 3, 1), 3, [0, 1, 2]), ((2, 7, 2), 8, [1, 3, 5]),
                                            ((3, 9, 3), 5, [2]), ((1, 8, 4), 8, [0, 4])])
def test_test_shots_follow_testshot_start_end_incr(tmp_path, monkeypatch, ts, nshots, want):
    monkeypatch.chdir(tmp_path)   # paths inside the parameter file are relative, as in the reference
    inp_case.write_case(str(tmp_path), nshots=nshots, MODE=1, TESTSHOT=list(ts))
    acq = inversion.Acquisition(io.read_inp(str(tmp_path / "case.inp")))
    assert acq.nshots == nshots
    assert acq.test_shots() == want


def test_params_and_unsupported_switches(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    inp_case.write_case(str(tmp_path), nshots=2, MODE=1, DTINV=3, FDORDER=6, L=2)
    inp = io.read_inp(str(tmp_path / "case.inp"))
    acq = inversion.Acquisition(inp)
    p = inversion.params_from_inp(inp, acq.ts, store_snapshots=1)
    assert (p.nx, p.ny, p.fdorder, p.dtinv, p.L, p.store_snapshots) == (120, 80, 6, 3, 2, 1)
    assert p.nt == io.inp_nt(inp) and len(p.fl) == 2
    assert np.float32(p.ts) == np.float32(acq.ts)
    inversion._check_supported(inp)
    for key in ("SWS_TAPER_FILE", "TRKILL", "TIMELAPSE", "GRAVITY"):
        inp_case.write_case(str(tmp_path), nshots=2, MODE=1, **{key: 1})
        with pytest.raises(NotImplementedError):
            inversion._check_supported(io.read_inp(str(tmp_path / "case.inp")))


def test_model_file_names():
    assert workflow.stage_files("m/inv", 2) == ("m/inv_vp_stage_2.bin", "m/inv_vs_stage_2.bin", "m/inv_rho_stage_2.bin")
    assert workflow.iteration_files("m/inv", 1, 3)[0] == "m/inv_vp_stage_1_it_3.bin"


def test_memory_batches_spread_evenly(monkeypatch):
    """Batches hold at most the shots that fit 90 % of the free memory and are
    spread evenly; every shot appears once, in order."""
    from denise_b200 import api, shard

    shots = [(None, None, None, np.zeros(40, np.int32), None)] * 32
    monkeypatch.setattr(api, "shot_footprint", lambda p, ntr, store: 18 << 30)
    for free_gb, want in ((178, [8] * 4), (90, [4] * 8), (19, [1] * 32), (1000, [32])):
        monkeypatch.setattr(api, "device_memory", lambda device=0, f=free_gb: (f << 30, 183 << 30))
        parts = shard.memory_batches(None, shots, range(32), 1, 0)
        assert [len(b) for b in parts] == want, free_gb
        assert sum(parts, []) == list(range(32))
    monkeypatch.setattr(api, "device_memory", lambda device=0: (178 << 30, 183 << 30))
    assert [len(b) for b in shard.memory_batches(None, shots, range(30), 1, 0)] == [8, 8, 8, 6]
    assert shard.memory_batches(None, shots, [], 1, 0) == []
    # a shot larger than the free memory is refused before anything runs
    monkeypatch.setattr(api, "device_memory", lambda device=0: (10 << 30, 183 << 30))
    with pytest.raises(MemoryError):
        shard.memory_batches(None, shots, range(32), 1, 0)
