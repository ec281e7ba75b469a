"""Workflow files (read_par_inv.c): the stage reader against the reference's
own read_par_inv, and the model averages of the energy preconditioning."""
import ctypes

import numpy as np
import pytest

import oracles as O
from denise_b200.workflow import STAGE_KEYS, model_averages, read_workflow

needs_ref = pytest.mark.skipif(not O.reference_available(), reason="reference build not present")

HEADER = " ".join(STAGE_KEYS) + "\n"
STAGES = [
    "0.01 1 0.0 5.0 4 0 20.0 0.4 0.3 1 1 2 0 0 0.5 0.5 3 2 0 0 50.0 0.1 0 0 0.0 1.0 1.0 0 0.0 0\n",
    # a stage broken over two lines, hexadecimal and octal integers (fscanf %i)
    "0.005 1 2.0 10.0 0x6 5 10.0 0.2 0.1\n 1 1 1 0 2 1.5 0.7 1 7 0 0 20.0 0.1 0 1 150.0 0.8 1.0 0 0.0 01\n",
    "0.001 0 0.0 15.0 4 0 0.0 0.0 0.0 1 1 1 0 4 0.3 0.2 0 5 0 0 0.0 0.0 0 2 80.0 1.0 1.0 0 0.0 2\n",
]


def _ref_stage(path, k, kmax):
    lib = ctypes.CDLL(O.REF_SO)
    out = (ctypes.c_double * 30)()
    lib.refh_read_par_inv(path.encode(), k, kmax, out)
    return list(out)


@needs_ref
def test_read_workflow_matches_reference(tmp_path):
    path = tmp_path / "workflow.inp"
    # the second stage's line break adds a newline, so the reference counts one stage more
    # than there are; its fscanf finds no values for it and keeps those of stage 3
    path.write_text(HEADER + "".join(STAGES))
    stages = read_workflow(str(path))
    assert len(stages) == 4 and stages[3] == stages[2]
    for k in range(1, 5):
        ref = O.run_isolated(_ref_stage, str(path), k, len(stages))
        got = [float(np.float32(stages[k - 1][key])) if isinstance(stages[k - 1][key], float) else
               float(stages[k - 1][key]) for key in STAGE_KEYS]
        assert got == ref, (k, [(n, a, b) for n, a, b in zip(STAGE_KEYS, got, ref) if a != b])


def test_stage_count_and_values(tmp_path):
    path = tmp_path / "wf.inp"
    path.write_text(HEADER + STAGES[0] + STAGES[2])
    st = read_workflow(str(path))
    assert len(st) == 2
    assert st[0]["EPRECOND"] == 3 and st[0]["INV_RHO_ITER"] == 2 and st[1]["SPATFILTER"] == 4
    assert st[1]["N_ORDER"] == 2 and st[1]["OFFSET_MUTE"] == 2 and st[1]["OFFSETC"] == 80.0


def test_model_averages_in_float_sequence():
    rng = np.random.default_rng(1)
    a = (3000 + 500 * rng.random((37, 23))).astype(np.float32)
    acc = np.float32(0.0)
    for v in a.ravel():
        acc = np.float32(acc + v)
    want = float(np.float32(acc / np.float32(a.size)))
    assert model_averages(a, a, a)[0] == want
