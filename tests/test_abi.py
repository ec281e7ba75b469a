"""The C ABI library loads on a CPU-only host and exports every symbol that
include/denise_b200.h declares; argument validation answers without a GPU."""
import ctypes
import os
import re

import pytest

import denise_b200 as dn
from denise_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "denise_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(dn_\w+)\s*\(", src, flags=re.M)))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_version_and_errors():
    ma, mi = ctypes.c_int(), ctypes.c_int()
    assert _lib.lib.dn_version(ctypes.byref(ma), ctypes.byref(mi)) == 0
    assert (ma.value, mi.value) == (0, 1)


@pytest.mark.parametrize("bad,code", [(dict(fdorder=7), -1), (dict(nt=1), -1), (dict(boundary=1), -6),
                                      (dict(grad_form=2), -6), (dict(L=6), -1), (dict(L=2, fl=(1.0,)), -1)])
def test_model_validation_without_gpu(bad, code):
    import numpy as np

    base = dict(nx=16, ny=12, dh=5.0, dt=4e-4, nt=10)
    base.update(bad)
    p = dn.PsvParams(**base)
    z = np.ones((16, 12), np.float32)
    with pytest.raises(dn.DeniseError) as e:
        dn.Model(p, z * 2000, z * 1000, z * 2000, z * 50, z * 50)
    assert e.value.code == code


def test_kernel_shim_library_loads_beside_the_reference():
    """lib/libdenise_b200_fd.so defines update_v_PML_PSV, update_s_elastic_PML_PSV and
    update_s_visc_PML_PSV;
    its references to the reference's globals and err() resolve in a process that
    holds the reference (here, its build)."""
    import oracles as O

    shim = os.path.join(os.path.dirname(_lib.LIB_PATH), "libdenise_b200_fd.so")
    assert os.path.exists(shim)
    if not O.reference_available():
        pytest.skip("the reference build (oracle/_ref) is not there")
    ctypes.CDLL(O.REF_SO, mode=ctypes.RTLD_GLOBAL)
    lib = ctypes.CDLL(shim)
    for name in ("update_v_PML_PSV", "update_s_elastic_PML_PSV", "update_s_visc_PML_PSV"):
        assert hasattr(lib, name)
