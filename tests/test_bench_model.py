"""The measurement model of bench.py, checked on the CPU.

The roofline figures of the bench line rest on three pieces of arithmetic:
the Sekibun point count of a sphere (the reference prints it at start-up as
"#sekibun_mesh= 1935" for a=5, xi=2; Particle_domain, profile.cxx:25-74),
the compulsory bytes of one step (40.6 field passes of N*R bytes at 128^3
with 256 spheres) and the compulsory bytes of each launch.  The whole-job
value of replicas is all ranks' steps over the slowest rank's time."""
import bench
from kapsel_old_b200 import workload


def test_sekibun_counts_match_the_reference_domain():
    # a = 4, 5, 6, 10 with xi = 2: the point counts of the reference's
    # Particle_domain for these radii
    assert [bench.sekibun_count({"a": a, "a_xi": 2.0}) for a in (4, 5, 6, 10)] == [1309, 1935, 2801, 8709]


def test_step_bytes_model_of_the_headline_workload():
    cfg = workload.mixed_128_256()
    b, passes = bench.step_bytes_model(cfg, 4)
    assert abs(passes - 40.6) < 0.01
    assert b == passes * 128 ** 3 * 4


def test_kernel_bytes_of_the_fused_kernels():
    cfg = workload.mixed_128_256()
    kb = bench.kernel_bytes(cfg, 4)
    N = 128 ** 3
    I1 = 128 * 85 * 43 * 8  # one component after the x pass: NX x KYc x TZ complex floats
    # the force kernel reads phi, up and u* (7 real fields) and writes 3 x-pass inputs
    assert kb["k_zyw_force"] == 7 * N * 4 + 3 * I1
    # the c2r kernel reads 3 x-pass outputs and writes u* (3 real fields)
    assert kb["k_yzw_c2r"] == 3 * I1 + 3 * N * 4


def test_replica_value_is_all_ranks_over_the_slowest():
    assert bench.replica_value(200, 4, 0.5) == 200 * 4 / 0.5
    assert bench.reduce_max(1.25) == 1.25  # one rank: its own time
