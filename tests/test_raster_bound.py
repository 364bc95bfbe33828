"""The raster's early rejection of sample points (sum_exceeds_one in tdi_kernels.cu) skips the
two divisions of the barycentric test only when fl(fl(na/denom) + fl(nb/denom)) is certainly
above 1. This checks that claim in IEEE float32 arithmetic (numpy rounds to nearest, as the
device does) on points spread over the float range and packed around alpha + beta = 1."""
import numpy as np

F32 = np.float32
GROW = F32(1.0) + F32(16.0) * F32(5.9604644775390625e-8)


def predicate(na, nb, d):
    """The device predicate, restated: na, nb of d's sign."""
    with np.errstate(all="ignore"):
        s = (na + nb).astype(F32)
        lim = (d * GROW).astype(F32)
    beyond = np.where(d > 0, s > lim, s < lim)
    return beyond & (np.abs(d) >= F32(1e-30)) & (np.abs(s) <= F32(3.4028234663852886e38))


def test_rejected_points_fail_the_exact_test():
    rng = np.random.default_rng(11)
    rejected = 0
    for _ in range(20):
        n = 200_000
        d = (rng.uniform(-1, 1, n) * 10.0 ** rng.uniform(-29, 30, n)).astype(F32)
        t = rng.uniform(0, 1, n)
        scale = 1 + rng.normal(0, 1, n) * 10.0 ** rng.uniform(-8, -1, n)
        na = (d.astype(np.float64) * t * scale).astype(F32)
        nb = (d.astype(np.float64) * (1 - t) * scale).astype(F32)
        same = (np.sign(na) == np.sign(d)) & (np.sign(nb) == np.sign(d)) & (na != 0) & (nb != 0)
        p = predicate(na, nb, d) & same
        with np.errstate(all="ignore"):
            total = ((na / d).astype(F32) + (nb / d).astype(F32)).astype(F32)
        assert not np.any(p & ~(total > F32(1))), "a rejected point passes alpha + beta <= 1"
        rejected += int(p.sum())
    assert rejected > 100_000  # the bound does reject most points beyond the edge
