"""CPU: the oracle's restatement of the uint8 copy's grid (vo_u8_grid, vo_u8_codes)
against an independent numpy statement of the same rule, on float rows (a fitted
grid), byte rows (the identity) and rows beyond a fitted grid's range (clamped)."""
import numpy as np

from vann import workload


def _numpy_grid(rows):
    rows = rows.astype(np.float32)
    fitted = not bool(np.all((rows >= 0) & (rows <= 255) & (np.rint(rows) == rows)))
    if not fitted:
        return False, np.zeros(rows.shape[1], np.float32), np.float32(1), np.float32(1)
    lo = rows.min(0)
    rng = (rows.max(0) - lo).max()
    s = np.float32(rng) / np.float32(255.0) if rng > 0 else np.float32(1.0)
    return True, lo, np.float32(s), np.float32(1.0) / np.float32(s)


def _numpy_codes(x, lo, inv):
    return np.clip(np.rint((x.astype(np.float32) - lo) * np.float32(inv)), 0, 255).astype(np.uint8)


def test_fitted_grid_and_codes_match(oracle):
    for D, seed in ((96, 1), (48, 2), (128, 3)):
        rows = workload.mixture(3000, D, 20, seed=seed, sigma=0.05, integer=False, unit_norm=True)
        fitted, lo, s, inv = oracle.u8_grid(rows)
        nf, nlo, ns, ninv = _numpy_grid(rows)
        assert fitted and nf
        assert np.array_equal(lo, nlo) and s == ns and inv == ninv
        assert np.array_equal(oracle.u8_codes(rows, lo, inv), _numpy_codes(rows, lo, inv))
        # rows beyond the range clamp to the end codes
        wide = rows[:100] * np.float32(1.7)
        c = oracle.u8_codes(wide, lo, inv)
        assert np.array_equal(c, _numpy_codes(wide, lo, inv))
        assert c.min() == 0 and c.max() == 255


def test_byte_rows_keep_the_identity():
    import oracle.oracle as O

    rows = workload.mixture(2000, 128, 20, seed=4)
    fitted, lo, s, inv = O.u8_grid(rows)
    assert not fitted and not lo.any() and s == 1 and inv == 1
    assert np.array_equal(O.u8_codes(rows, None, 1.0), rows.astype(np.uint8))
    # one non-integer value makes the grid fitted
    rows[5, 7] += 0.25
    assert O.u8_grid(rows)[0]
