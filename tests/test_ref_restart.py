"""Restart records of the compiled reference (oracle/_ref): Save_Restart_udf
written through the record writer and read back by the resumed-run path
(one step, then Force_restore_parameters) continue a run exactly.  This pins
the record format and semantics the GPU library's save/load follow."""
import os

import numpy as np
import pytest

from oracle import ref, udf

pytestmark = pytest.mark.ref


@pytest.fixture(scope="module", autouse=True)
def _need_ref():
    if not ref.available():
        pytest.skip("oracle/_ref not built")


def test_reference_restart_continues_exactly(tmp_path):
    cfg = udf.ns_config((5, 5, 5), 3, seed=5, kbt=0.0, min_gap=1.0, gravity_g=0.5, mass_ratio=1.5)
    a = ref.RefSim(cfg)
    a.step(4)
    path = os.path.join(tmp_path, "r.res")
    a.save_restart(path)
    z4, p4 = a.zeta().copy(), a.particles()
    a.step(3)
    b = ref.RefSim(cfg)
    b.resume(path)
    assert b.ts() == 4
    assert np.array_equal(b.zeta(), z4)
    assert np.array_equal(b.particles()["x"], p4["x"]) and np.array_equal(b.particles()["v"], p4["v"])
    b.step(3)
    assert np.abs(a.zeta()).max() > 0
    assert np.array_equal(b.zeta(), a.zeta())
    assert np.array_equal(b.particles()["x"], a.particles()["x"])
