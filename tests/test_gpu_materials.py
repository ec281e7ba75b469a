"""Material planes built on the device (k_materials) against the host set-up
(DN_HOST_MATERIALS=1, the functions tests/test_setup_parity.py pins to the
reference): bit-identical for elastic and viscoelastic models, constant and
per-cell Q, odd and tiny grids (the periodic edges of matcopy)."""
import numpy as np
import pytest

import denise_b200 as dn
from denise_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nx,ny,L,honor_q", [(64, 48, 0, 0), (37, 29, 3, 0), (41, 33, 2, 1), (1, 7, 0, 0),
                                             (5, 1, 1, 1), (300, 120, 3, 1)])
def test_device_materials_equal_host(monkeypatch, nx, ny, L, honor_q):
    p = synth.c0_params(nx=nx, ny=ny, nt=10, fw=0, L=L, fl=(2.0, 8.0, 25.0)[:L], ts=0.1, honor_q=honor_q,
                        free_surf=0)
    vp, vs, rho = synth.base_model(nx, ny, p.dh, 7)
    rng = np.random.default_rng(5)
    vs = vs.copy()
    vs.flat[rng.integers(0, vs.size, max(1, vs.size // 50))] = 0.0   # fluid cells: the u == 0 branch of av_mue
    qp, qs = synth.q_model(nx, ny, 7) if L else (None, None)
    planes = {}
    for host in ("1", "0"):
        monkeypatch.setenv("DN_HOST_MATERIALS", host)
        m = dn.Model(p, vp, vs, rho, qp, qs)
        planes[host] = [m.material(k) for k in range(16 if L else 10)]
        m.close()
    for k, (a, b) in enumerate(zip(planes["1"], planes["0"])):
        np.testing.assert_array_equal(a, b, err_msg=dn.Model.MATERIALS[k])
