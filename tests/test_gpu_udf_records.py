"""Output_udf records (avs_output.cxx:343-450) from device state against the
compiled reference's own Output_udf (oracle/_ref, stand-in record manager):
same paths, values within 1e-10 relative (FP64), at ts = 0 and after steps;
the records also round-trip through udf_io.write_records / read_records."""
import numpy as np
import pytest

from oracle import ref, udf

pytestmark = pytest.mark.gpu


def test_udf_records_match_reference(tmp_path):
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    import kapsel_old_b200 as kg
    from kapsel_old_b200 import udf_io

    cfg = udf.ns_config((5, 5, 5), 3, seed=3, kbt=1e-3, gravity_g=0.2, mass_ratio=1.5)
    R = ref.RefSim(cfg)
    g = kg.Simulation(cfg, precision=kg.FP64)
    mine = []
    for nstep in (0, 3, 2):
        R.step(nstep)
        g.step(nstep)
        R.output_udf()
        mine.append(g.udf_record())
    theirs = R.udf_records()[1:]  # record 0 is the echoed input
    assert len(theirs) == 3
    for a, b in zip(mine, theirs):
        flat = udf_io.flatten(a)
        assert set(flat) == set(b), set(flat) ^ set(b)
        for k, x in flat.items():
            y = float(b[k])
            assert abs(float(x) - y) <= 1e-10 * max(abs(y), 1e-6), (k, x, y)
    assert mine[2]["t"] == 5
    (tmp_path / "d.udf").write_text(
        "\\begin{def}\nclass Vector3d:{x: float, y: float, z: float}\n"
        "class Quaternion:{q0: float, q1: float, q2: float, q3: float}\n"
        "class outParticle:{R:Vector3d, R_raw:Vector3d, v:Vector3d, q:Quaternion, omega:Vector3d,"
        " f_hydro:Vector3d, torque_hydro:Vector3d, f_r:Vector3d, torque_r:Vector3d,"
        " f_slip:Vector3d, torque_slip:Vector3d}\nE: float\nt: float\nParticles[]: outParticle\n\\end{def}\n")
    out = tmp_path / "out.udf"
    udf_io.write_records(str(out), mine, str(tmp_path / "d.udf"))
    back = udf_io.read_records(str(out))
    assert [float(r["t"]) for r in back] == [0.0, 3.0, 5.0]
    assert np.isclose(back[1]["Particles[2].v.y"], mine[1]["Particles"][2]["v"]["y"], rtol=0, atol=0)
