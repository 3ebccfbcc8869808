"""GPU tests of the batched ensemble: boxes of different shapes advanced by
one CUDA graph per step must match the same boxes advanced one by one, and
the oracle; the per-box mean-square displacement is checked against the
particle records."""
import numpy as np
import pytest

from oracle import spm, udf

pytestmark = pytest.mark.gpu


def _cfgs():
    return [udf.ns_config((5, 5, 5), 2, seed=21, a=4.5, kbt=1e-3),
            udf.ns_config((5, 5, 6), 3, seed=22, a=5.0, kbt=1e-3),
            udf.ns_config((6, 6, 6), 4, seed=23, a=5.5, kbt=1e-3)]


def rel(a, b):
    n = np.linalg.norm(b)
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / (n if n > 0 else 1.0)


@pytest.mark.parametrize("autotune", [False, True])
def test_batch_matches_single_boxes_and_oracle(autotune):
    import kapsel_old_b200 as kg

    cfgs = _cfgs()
    batch_sims = [kg.Simulation(c, precision=kg.FP64) for c in cfgs]
    solo = [kg.Simulation(c, precision=kg.FP64) for c in cfgs]
    b = kg.Batch(batch_sims, autotune=autotune)
    b.step(5)
    for s in solo:
        s.step(5)
    for bs, ss in zip(batch_sims, solo):
        assert rel(bs.zeta(), ss.zeta()) < 1e-12
        assert rel(bs.particles()["v"], ss.particles()["v"]) < 1e-12
    o = spm.SpmOracle(cfgs[2])
    o.run(5)
    zt = spm.SpmOracle.to_ooura(np.stack([o.S.truncate(o.zeta[d]) for d in range(2)]))
    assert rel(batch_sims[2].zeta(), zt) < 1e-10
    assert np.abs(batch_sims[2].particles()["x"] - o.p.x).max() < 1e-10
    b.close()


def test_batch_msd():
    import kapsel_old_b200 as kg

    cfgs = _cfgs()
    sims = [kg.Simulation(c, precision=kg.MIXED) for c in cfgs]
    x0 = [s.particles()["x_nopbc"] for s in sims]
    b = kg.Batch(sims)
    b.step(6)
    msd = b.msd()
    for i, s in enumerate(sims):
        d = s.particles()["x_nopbc"] - x0[i]
        assert abs(msd[i] - np.mean(np.sum(d * d, axis=1))) <= 1e-12 * max(msd[i], 1e-300)
    assert np.all(msd > 0)
    b.close()


def test_batch_autotune_after_stepping_matches_single_boxes():
    """Boxes stepped on their own before the batch is built: the autotuner's
    timing passes overwrite the spectrum buffer that a stepped box keeps for
    its next step, which must then be recomputed, not reused."""
    import kapsel_old_b200 as kg

    cfgs = _cfgs()
    batch_sims = [kg.Simulation(c, precision=kg.FP64) for c in cfgs]
    solo = [kg.Simulation(c, precision=kg.FP64) for c in cfgs]
    for s in batch_sims + solo:
        s.step(3)
    b = kg.Batch(batch_sims, autotune=True)
    b.step(4)
    for s in solo:
        s.step(4)
    for bs, ss in zip(batch_sims, solo):
        assert bs.time()[0] == ss.time()[0] == 7
        assert rel(bs.zeta(), ss.zeta()) < 1e-12
        assert rel(bs.particles()["v"], ss.particles()["v"]) < 1e-12
    b.close()


def test_batch_pass_variants_match():
    """Every z / y pass variant the autotuner may choose gives the same step
    (FP64, to roundoff) as the default one, on a box whose shape allows all
    of them (64x64x128)."""
    import kapsel_old_b200 as kg

    cfg = udf.ns_config((6, 6, 7), 5, seed=24, a=5.0, kbt=1e-3)
    ref = kg.Simulation(cfg, precision=kg.FP64)
    ref.step(4)
    for zmode, ymode in [(0, 0), (0, 1), (0, 2), (0, 3), (1, 0), (1, 1), (1, 2)]:
        if True:
            s = kg.Simulation(cfg, precision=kg.FP64)
            _set_variant(s, zmode, ymode)
            s.step(4)
            assert rel(s.zeta(), ref.zeta()) < 1e-12, (zmode, ymode)
            assert rel(s.particles()["v"], ref.particles()["v"]) < 1e-12, (zmode, ymode)
            s.close()
    ref.close()


@pytest.mark.parametrize("shape", [(5, 5, 6), (6, 6, 7), (7, 7, 7), (6, 5, 6)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_x_split_matches_default(shape, precision):
    """The other radix split of the block-level x transforms (32 = 4 x 8,
    64 = 16 x 4, 128 = 16 x 8), which the batch autotuner may choose, gives
    the same steps to roundoff (FP64 1e-12, mixed 1e-5); 256-point x lines
    have no other split."""
    import ctypes

    import kapsel_old_b200 as kg

    prec = kg.FP64 if precision == "fp64" else kg.MIXED
    tol = 1e-12 if precision == "fp64" else 1e-5
    cfg = udf.ns_config(shape, 4, seed=26, a=5.0, kbt=1e-3)
    a = kg.Simulation(cfg, precision=prec)
    b = kg.Simulation(cfg, precision=prec)
    fn = b.L.kapsel_gpu_set_x_split
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int]
    assert fn(b.h, 1) == 0
    a.step(4)
    b.step(4, graph=True)
    assert 0 < rel(b.zeta(), a.zeta()) < tol
    assert rel(b.particles()["v"], a.particles()["v"]) < tol
    a.close()
    b.close()
    big = kg.Simulation(udf.ns_config((8, 5, 5), 1, seed=27, a=5.0), precision=kg.FP64)
    assert fn(big.h, 1) == -1
    big.close()


def _set_variant(sim, zmode, ymode):
    import ctypes

    fn = sim.L.kapsel_gpu_set_pass_variant
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    assert fn(sim.h, zmode, ymode) == 0


@pytest.mark.parametrize("shape,n", [((7, 7, 7), 256), ((6, 6, 7), 12), ((6, 6, 6), 6), ((5, 5, 6), 3),
                                     ((6, 7, 6), 10)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_yz_planes_bitwise(shape, n, precision):
    """Pass variant 3 runs the inverse y + z c2r and the force's z + y passes
    as one launch each over (component, x) planes in shared memory; its
    transforms and sums are those of the separate passes, so every step is
    bitwise the same as variant (0, 0), including the clearing of phi/up
    that the next step's scatter relies on."""
    import kapsel_old_b200 as kg

    prec = kg.FP64 if precision == "fp64" else kg.MIXED
    cfg = udf.ns_config(shape, n, seed=25, a=5.0, kbt=1e-3)
    a = kg.Simulation(cfg, precision=prec)
    b = kg.Simulation(cfg, precision=prec)
    _set_variant(a, 0, 0)
    _set_variant(b, 0, 3)
    a.step(2)
    b.step(2)
    a.step(4, graph=True)
    b.step(4, graph=True)
    assert np.array_equal(a.zeta(), b.zeta())
    pa, pb = a.particles(), b.particles()
    for k in ("x", "v", "omega"):
        assert np.array_equal(pa[k], pb[k]), k
    assert np.array_equal(a.velocity(), b.velocity())
    a.close()
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_larger_box_created_before_smaller_one(precision):
    """The dynamic shared-memory limit of a kernel is one value per process:
    a box created after a larger one must not lower it below what the larger
    box's launches ask for (64x64x128 with the block-level z passes, then
    32^3), alone and in a batch built largest box first."""
    import kapsel_old_b200 as kg

    prec = kg.FP64 if precision == "fp64" else kg.MIXED
    big = udf.ns_config((6, 6, 7), 6, seed=26, a=5.0, kbt=1e-3)
    small = udf.ns_config((5, 5, 5), 2, seed=27, a=4.5, kbt=1e-3)
    a = kg.Simulation(big, precision=prec)
    b = kg.Simulation(small, precision=prec)
    a.step(3)
    b.step(3)
    c = kg.Simulation(big, precision=prec)
    c.step(3)
    assert np.array_equal(a.zeta(), c.zeta())
    sims = [kg.Simulation(cfg, precision=prec) for cfg in (big, big, small, small)]
    solo = kg.Simulation(big, precision=prec)
    bt = kg.Batch(sims, autotune=True)
    bt.step(4)
    solo.step(4)
    assert rel(sims[0].zeta(), solo.zeta()) < (1e-12 if precision == "fp64" else 1e-5)
    bt.close()
    for s in sims + [a, b, c, solo]:
        s.close()
