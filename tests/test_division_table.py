"""The degree-centrality mean's division table, restated and checked on the CPU.

The long-list mean (``k_degree_long``) replaces ``x / d`` for ``0 <= x < 2^31`` by
``mulhi32(M, x) >> (l - 1)`` with ``l = ceil(log2 d)`` and ``M = ceil(2^(31 + l) / d)``, the table
``tga_open`` uploads for every count ``2 <= d <= max outdegree + 1`` (the Java mean,
cpu_java/src/main/java/gr/uoa/di/networkanalysis/BaselineRunner.java:316-322, divides by the
running count at every step and truncates).  The proof
(Granlund and Montgomery, PLDI 1994): ``M d = 2^(31 + l) + e`` with ``0 <= e < d <= 2^l``, so the
product exceeds ``x 2^(31 + l) / d`` by ``x e / d < 2^(31 + l) / d``: less than 1/d of one
quotient step (``2^(31 + l)``), and ``x / d`` lies at least 1/d of a step below the next integer.  This test checks the arithmetic on the hardest inputs of each divisor: the largest
``x`` below 2^31 with the largest remainder, every multiple boundary near the top of the range, and
random ``x``.  The GPU parity tests check the kernel's means bit for bit against the oracle.
"""
import numpy as np

MASK32 = (1 << 32) - 1


def table_entry(d):
    l = (d - 1).bit_length()  # ceil(log2 d) for d >= 2
    m = ((1 << (31 + l)) + d - 1) // d
    assert m <= MASK32, (d, m)
    return m, l - 1


def divisors():
    ds = set(range(2, 4097))
    for k in range(2, 30):
        for off in (-3, -1, 0, 1, 3):
            d = (1 << k) + off
            if d >= 2:
                ds.add(d)
    rng = np.random.default_rng(7)
    ds.update(int(d) for d in rng.integers(2, 1 << 29, size=2000))
    ds.update((163154, 163155, 5_000_000, 5_000_001, (1 << 31) // 4 - 1))
    return sorted(ds)


def test_division_table_exact_below_2_31():
    rng = np.random.default_rng(11)
    top = (1 << 31) - 1
    for d in divisors():
        m, s = table_entry(d)
        k_hi = top // d
        xs = [0, 1, d - 1, d, d + 1, top, top - 1]
        for k in range(max(k_hi - 4, 1), k_hi + 1):
            xs += [k * d - 1, k * d, min(k * d + d - 1, top)]
        x = np.array(xs + list(rng.integers(0, 1 << 31, size=64)), dtype=np.uint64)
        x = x[x <= top]
        q = ((x * np.uint64(m)) >> np.uint64(32)) >> np.uint64(s)
        assert np.array_equal(q, x // np.uint64(d)), d


def test_division_table_exhaustive_small_range():
    # Every x below 2^20 for a few divisors of each kind (power of two, one above, odd, large).
    x = np.arange(1 << 20, dtype=np.uint64)
    for d in (2, 3, 7, 64, 65, 1000, 4095, 4097, 163155, (1 << 29) + 1):
        m, s = table_entry(d)
        q = ((x * np.uint64(m)) >> np.uint64(32)) >> np.uint64(s)
        assert np.array_equal(q, x // np.uint64(d)), d
