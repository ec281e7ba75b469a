"""Time-domain Butterworth filter (apply_tdfilt): the oracle restatement of
libcseife's recursive filters (oracle/tdfilt_oracle.py) against the
reference's own apply_tdfilt; and the device filter against the oracle."""
import os
import sys

import numpy as np
import pytest

import oracles as O

sys.path.insert(0, os.path.join(O.ROOT, "oracle"))
import tdfilt_oracle as tf  # noqa: E402

needs_ref = pytest.mark.skipif(not O.reference_available(), reason="reference build not present")

# (order, fc_low, fc_high): odd and even orders, low-pass only and band-pass; a
# negative high-pass corner (FC_SPIKE_1 = -5 in the reference's example files)
# means no high-pass, as apply_tdfilt only high-passes for fc1 > 0
CASES = [(4, 20.0, 0.0), (5, 30.0, 3.0), (2, 12.5, 1.0), (1, 40.0, 5.0), (6, 8.0, 2.0), (3, 45.0, 0.0),
         (5, 15.0, -5.0)]


def traces(seed=0, ntr=6, ns=500):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((ntr, ns)).astype(np.float32)


@needs_ref
@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference(case):
    d = traces(case[0])
    want = O.run_isolated(O.ref_apply_tdfilt, d, 1e-3, *case)
    got = tf.apply_tdfilt(d, 1e-3, *case)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    assert got[0, -1] == d[0, -1]          # the reference leaves the last sample as it is


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_device_filter_matches_oracle(case):
    import denise_b200 as dn

    d = traces(case[0] + 10, ntr=37, ns=2001)
    got = dn.tdfilt(d, 5e-4, *case)
    want = tf.apply_tdfilt(d, 5e-4, *case)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
def test_device_filter_on_device_buffer_and_errors():
    import ctypes

    import torch

    import denise_b200 as dn
    from denise_b200 import _lib

    d = traces(3, ntr=8, ns=1000)
    t = torch.as_tensor(d).cuda()
    _lib.check(_lib.lib.dn_tdfilt(t.data_ptr(), 8, 1000, ctypes.c_float(1e-3), 4, ctypes.c_float(25.0),
                                  ctypes.c_float(2.0)))
    np.testing.assert_array_equal(t.cpu().numpy(), tf.apply_tdfilt(d, 1e-3, 4, 25.0, 2.0))
    for bad in ((0, 25.0, 0.0), (17, 25.0, 0.0), (4, 0.0, 0.0), (4, 25.0, float("nan"))):
        with pytest.raises(dn.DeniseError, match="DN_EINVAL"):
            dn.tdfilt(d, 1e-3, *bad)
