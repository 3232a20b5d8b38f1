"""The arithmetic facts the stencil kernels rely on, checked on the CPU with IEEE
float32 arithmetic (numpy's float32 division and multiplication round to nearest,
like the GPU's __fdiv_rn / __fmul_rn):

* receivers (csrc/pff_core.cu, rcv_off_fast): a drop d < dmax whose quotient by dx
  rounds to the same float32 as dmax's is never below RN(dmax * (1 - 2^-21)), so
  directions under that bound can be skipped when looking for a tie;
* labels and list passes (csrc/pff_lake.cu, divmod_nx): umulhi(n, m) with
  m = floor(2^32 / d) or floor((2^32 - 1) / d) is floor(n / d) or one less for
  0 <= n < 2^31, and one correction of the remainder makes it exact;
* the exact-division range (csrc/pff_div.cuh, make_divc) keeps the numerator and the
  quotient inside [2^-100, 2^100].
"""
import numpy as np

F = np.float32


def test_near_tie_bound_covers_every_rounding_tie():
    rng = np.random.default_rng(3)
    one_minus = F(1.0) - F(2.0 ** -21)
    ties = 0
    for dx in [30.0, 10.0, 3.0, 1.0, 0.3, 7.77, 1e-3, 3e-20, 1e4]:
        dx = F(dx)
        # largest drops spread over many binades, and drops a few ulps below them
        m = (rng.random(200_000) * F(2.0) ** rng.integers(-40, 40, 200_000)).astype(np.float32)
        m = m[m > 0]
        for k in (1, 2, 3, 4, 6, 8, 16, 64):
            bits = m.view(np.uint32)
            keep = bits > np.uint32(k)
            mm = m[keep]
            d = (bits[keep] - np.uint32(k)).view(np.float32)
            tie = (d / dx) == (mm / dx)  # a different drop whose rounded quotient ties
            near = mm * one_minus
            assert np.all(d[tie] >= near[tie]), (float(dx), k)
            ties += int(tie.sum())
    assert ties > 100_000  # the bound was exercised


def test_divmod_by_multiply_high():
    rng = np.random.default_rng(5)
    ds = np.concatenate([np.arange(2, 70), [127, 128, 129, 1000, 1024, 2047, 2048, 4095, 4096, 4097, 65535, 65536,
                                            (1 << 20) + 7, (1 << 29) + 1], rng.integers(2, 1 << 30, 200)])
    for d, m in [(d, (1 << 32) // d) for d in ds.tolist()] + [(d, ((1 << 32) - 1) // d) for d in ds.tolist()]:
        n = np.concatenate([np.arange(0, 3 * d if d < 5000 else 5000, dtype=np.int64),
                            rng.integers(0, 1 << 31, 20000), [(1 << 31) - 1, (1 << 31) - d, ((1 << 31) // d) * d - 1]])
        n = n[(n >= 0) & (n < (1 << 31))].astype(np.uint64)
        q = (n * np.uint64(m)) >> np.uint64(32)
        r = n.astype(np.int64) - q.astype(np.int64) * d
        assert np.all((r >= 0) & (r < 2 * d)), d
        fix = r >= d
        q = q.astype(np.int64) + fix
        r = r - d * fix
        assert np.array_equal(q, n.astype(np.int64) // d) and np.array_equal(r, n.astype(np.int64) % d), d


def test_exact_division_range():
    for dx in [30.0, 10.0, 3.0, 1.0, 0.3, 7.77, 123.456, 1e-3, 3e-20, 1e4, 0.1, 2.0 ** -20, 1e30, 1e-30]:
        dx = F(dx)
        with np.errstate(over="ignore", under="ignore"):
            mlo = max(F(dx * F(2.0 ** -100)), F(2.0 ** -100))
            mhi = min(F(dx * F(2.0 ** 100)), F(2.0 ** 100))
        assert mlo <= mhi
        for m in (mlo, mhi):
            q = np.float64(m) / np.float64(dx)
            assert 2.0 ** -100 <= q <= 2.0 ** 100 * (1 + 2.0 ** -20), (float(dx), float(m))
            assert 2.0 ** -100 <= float(m) <= 2.0 ** 100
