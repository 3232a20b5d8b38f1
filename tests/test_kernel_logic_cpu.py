"""The decision logic of two GPU kernels, restated in numpy float32 and checked on
the CPU at scale against the reference semantics (no GPU needed):

* the lean receivers kernel's choice (csrc/pff_core.cu, rcv_off_fast): the largest
  drop, the first direction at or above RN(dmax (1 - 2^-21)), the ordered scan for
  near ties and drops outside the exact-division range -- against the reference's
  ordered scan with a strict '>' (receivers.py:43-52) on drops with exact ties, near
  ties, NaN and invalid links;
* the fill's settled-round skip (csrc/pff_gf.cu, k_fill_round_late): running the
  packed rounds only until a round whose input is all settled gives the same records
  as running all ceil(log2 N) rounds, and the oracle's fill (fill_topo.py:17-45) --
  on forests with long chains, receiver cycles and increments too small to move z.
"""
import numpy as np
import pytest

F = np.float32
NEG = F(-np.inf)


def ordered_scan(d, dx):
    """receivers.py:43-52 on drops d[:, k] (k = top, left, right, bottom)."""
    best = np.zeros(d.shape[0], np.float32)
    kk = np.full(d.shape[0], -1, np.int64)
    for k in range(4):
        with np.errstate(invalid="ignore"):
            t = d[:, k] / dx
            up = t > best
        best = np.where(up, t, best)
        kk = np.where(up, k, kk)
    return kk, best


def fast_choice(d, dx):
    """rcv_off_fast: (direction, gradient, ok); where ok is False the kernel runs the
    ordered scan instead."""
    with np.errstate(invalid="ignore"):
        m = np.fmax(np.fmax(d[:, 0], d[:, 1]), np.fmax(d[:, 2], d[:, 3]))
        near = m * (F(1.0) - F(2.0 ** -21))
        p = [d[:, k] >= near for k in range(3)]
    dsel = np.where(p[0], d[:, 0], np.where(p[1], d[:, 1], np.where(p[2], d[:, 2], d[:, 3])))
    k = np.where(p[0], 0, np.where(p[1], 1, np.where(p[2], 2, 3)))
    mlo = max(F(dx * F(2.0 ** -100)), F(2.0 ** -100))
    mhi = min(F(dx * F(2.0 ** 100)), F(2.0 ** 100))
    with np.errstate(invalid="ignore", over="ignore"):
        pit = ~(m > 0)
        ok = pit | ((dsel == m) & (m >= mlo) & (m <= mhi))
        q = m / dx  # the kernel's Markstein quotient equals this on [mlo, mhi] (exhaustive GPU test)
    return np.where(pit, -1, k), np.where(pit, F(0.0), q).astype(np.float32), ok


@pytest.mark.parametrize("dx", [30.0, 3.0, 0.3, 1e-3, 3e-20, 1e4])
def test_receivers_fast_choice_matches_ordered_scan(dx):
    dx = F(dx)
    rng = np.random.default_rng(int(abs(np.log2(dx))) + 7)
    n = 400_000
    base = (rng.random(n) * 50).astype(np.float32)
    d = np.stack([base + (rng.random(n) * 10 - 5).astype(np.float32) for _ in range(4)], 1).astype(np.float32)
    # exact ties, near ties (a few ulps), flats, NaN and invalid links
    sel = rng.random(n) < 0.2
    d[sel, 2] = d[sel, 0]
    sel = rng.random(n) < 0.2
    j = rng.integers(0, 4, n)
    for k in range(4):
        s = sel & (j == k)
        o = (k + 1) % 4
        d[s, k] = (d[s, o].view(np.uint32) - rng.integers(1, 5, s.sum()).astype(np.uint32)).view(np.float32)
    d[rng.random(n) < 0.05] = 0.0
    d[rng.random((n, 4)) < 0.02] = np.nan
    d[rng.random((n, 4)) < 0.05] = NEG
    d[rng.random(n) < 0.01, 1] = np.float32(1e-40)  # subnormal drops
    k_ref, s_ref = ordered_scan(d, dx)
    k_fast, s_fast, ok = fast_choice(d, dx)
    assert np.array_equal(k_fast[ok], k_ref[ok])
    assert np.array_equal(s_fast[ok].view(np.uint32), s_ref[ok].view(np.uint32))
    assert ok.mean() > 0.5  # most cells take the fast path


ROOT = np.uint32(0x80000000)


def packed_fill(zh, rec, inc, vote0=None):
    """The packed fill rounds of csrc/pff_gf.cu (k_fill_round_packed / _late) in numpy:
    records {pointer | root flag, z}; with vote0, a round after one whose input was
    all settled is skipped, as k_fill_round_late does."""
    N = zh.size
    idx = np.arange(N)
    r0 = np.where((rec >= 0) & (rec < N), rec, idx)
    ptr = r0.astype(np.int64)
    root = r0 == idx
    z = zh.astype(np.float32).copy()
    prev_settled = False
    ran = 0
    for it in range(inc.size):
        if vote0 is not None and it > vote0 and prev_settled:
            break
        r = ptr
        rr = ptr[r]
        zr = z[r]
        zref = np.where(root[r], zr, zh[r])
        keep = (idx == r) | ((rr == r) & (z > zref))
        with np.errstate(over="ignore"):
            zn = np.where(keep, z, np.maximum(z, (zr + inc[it]).astype(np.float32)))
        if vote0 is not None and it >= vote0:
            prev_settled = bool(keep.all())
        ptr, z = rr, zn.astype(np.float32)
        ran += 1
    return z, ran


def forest(kind, n, rng):
    idx = np.arange(n)
    if kind == "line":  # one long chain: needs every round
        rec = idx - 1
        rec[0] = 0
    elif kind == "random":  # each cell points to an earlier cell or itself
        rec = np.where(rng.random(n) < 0.01, idx, (idx * rng.random(n)).astype(np.int64))
    else:  # random with 2-cycles injected (never settled)
        rec = np.where(rng.random(n) < 0.01, idx, (idx * rng.random(n)).astype(np.int64))
        a = rng.choice(n - 1, 20, replace=False) + 1
        rec[a] = a - 1
        rec[a - 1] = a
    return rec.astype(np.int32)


@pytest.mark.parametrize("kind", ["line", "random", "cycles"])
@pytest.mark.parametrize("eps,scale", [(1e-3, 100.0), (1e-6, 1000.0), (0.0, 10.0), (1e-9, 1e6)])
def test_fill_settled_skip_is_exact(orc, kind, eps, scale):
    rng = np.random.default_rng(11)
    n = 70_000  # 17 rounds
    rec = forest(kind, n, rng)
    zh = (rng.random(n) * scale).astype(np.float32)
    inc = orc.fill_increments(n, eps)
    z_all, ran_all = packed_fill(zh, rec, inc)
    z_skip, ran_skip = packed_fill(zh, rec, inc, vote0=10)
    assert ran_all == inc.size
    assert np.array_equal(z_all.view(np.uint32), z_skip.view(np.uint32))
    _, _, z_orc = orc.fill_z_add_delta(zh.copy(), np.zeros(n, np.float32), rec, eps)
    assert np.array_equal(z_all.view(np.uint32), z_orc.view(np.uint32))
    if kind == "random" and eps > 0 and scale < 1e5:
        assert ran_skip < ran_all  # the skip happened
