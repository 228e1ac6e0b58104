"""CPU check of the integer form of RobustPrune's test in the tensor-core prune.

The kernel decides "t prunes u" as fl(Y * alpha) <= d(node, u), where Y is the exact
integer squared distance between t and u (below 2^24, so FP32 holds it exactly) and
fl() is FP32 rounding.  fl(Y * alpha) does not decrease as Y grows, so the kernel
finds once per candidate u the largest integer Ymax with fl(Ymax * alpha) <= d(node, u)
and compares integers: Y <= Ymax.  This restates that search in FP32 numpy, as the
kernel does it, and checks the equivalence over random and boundary distances.
"""
import numpy as np

F = np.float32
LIMIT = (1 << 24) - 1


def ymax(sd: np.float32, alpha: np.float32) -> int:
    """The kernel's threshold: start at floor(sd / alpha) (FP32), then step."""
    y = int(min(np.floor(F(sd) / F(alpha)), F(LIMIT)))
    while y < LIMIT and F(F(y + 1) * F(alpha)) <= sd:
        y += 1
    while y > 0 and F(F(y) * F(alpha)) > sd:
        y -= 1
    return y


def _check(sd, alpha, ys):
    t = ymax(sd, alpha)
    scaled = (ys.astype(np.float32) * F(alpha)).astype(np.float32)
    assert np.array_equal(scaled <= F(sd), ys <= t), (sd, alpha, t)


def test_threshold_equals_the_float_test():
    rng = np.random.default_rng(7)
    for alpha in (F(1.0), F(1.2), F(1.5), F(1.2000000476837158), *rng.uniform(1.0, 2.0, 8).astype(np.float32)):
        # distances of the kind the prune sees: integers (integer rows) and their neighbours
        base = rng.integers(0, LIMIT, 200)
        sds = np.concatenate([base.astype(np.float32),
                              (base.astype(np.float32) * alpha).astype(np.float32),
                              rng.uniform(0, 2.0e7, 100).astype(np.float32), np.float32([0.0, 1.0, 2.0e7])])
        for sd in sds:
            sd = F(sd)
            t = ymax(sd, alpha)
            window = np.arange(max(0, t - 64), min(LIMIT, t + 64) + 1, dtype=np.int64)
            _check(sd, alpha, np.concatenate([window, rng.integers(0, LIMIT + 1, 64)]))


def test_threshold_at_exact_products():
    """sd equal to fl(Y * alpha) for some Y, and one ulp either side of it."""
    rng = np.random.default_rng(11)
    alpha = F(1.2)
    for y in rng.integers(0, LIMIT, 300):
        p = F(F(y) * alpha)
        for sd in (np.nextafter(p, F(0)), p, np.nextafter(p, F(np.inf))):
            t = ymax(F(sd), alpha)
            window = np.arange(max(0, t - 8), min(LIMIT, t + 8) + 1, dtype=np.int64)
            _check(F(sd), alpha, window)
            if sd >= p:
                assert t >= y
