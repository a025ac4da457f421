"""CPU restatement of the roughness walk's per-chunk moment arithmetic (analysis.cu,
walk_kernel<0>): the heights of a 64-site chunk are b + d_i with d_i a +-1 walk from 0, the
power sums of d are taken in 32-bit (k <= 4) and 64-bit (k = 5..7) integers, and the sums
of h^k follow by the binomial expansion in FP64 once per chunk.  The test checks the integer
ranges the kernel relies on (worst case: a monotone walk) and the expansion against exact
integer sums, with the tolerance the GPU roughness tests use (rtol 1e-12)."""
import numpy as np
import pytest

RTOL = 1e-12
I32 = 2**31 - 1
I64 = 2**63 - 1


def chunk_power_sums(bits, skip_first):
    """The kernel's integer accumulators a1..a7 and the count n over one chunk."""
    d = 0
    a = [0] * 8
    n = 0
    for i, bit in enumerate(bits):
        d += 2 * int(bit) - 1
        if i == 0 and skip_first:
            continue
        n += 1
        for k in range(1, 8):
            a[k] += d ** k
    return n, a


def expand(b, n, a):
    """sum_i (b + d_i)^k for k = 3..7 from the power sums of d, in FP64 as the kernel does."""
    B = float(b)
    A = [float(n)] + [float(v) for v in a[1:]]
    out = []
    for k in range(3, 8):
        s = 0.0
        c = 1
        for j in range(k + 1):
            s += c * B ** (k - j) * A[j]
            c = c * (k - j) // (j + 1)
        out.append(s)
    return out


def test_integer_ranges_worst_case():
    """A monotone walk (d = 1..64) gives the largest power sums: a1..a4 stay in int32 and the
    per-site products d^4 * d, d^3 * d^3, d^4 * d^3 and their sums in int64."""
    for bit in (0, 1):
        n, a = chunk_power_sums([bit] * 64, False)
        for k in range(1, 5):
            assert abs(a[k]) <= I32, k
        for k in range(5, 8):
            assert abs(a[k]) <= I64, k
        assert 64 ** 4 <= I32 and 64 ** 3 <= I32  # d^3, d^4 per site in int32


@pytest.mark.parametrize("b", [0, 7, -13, 64, -100, 1_000, -250_000, 3_000_000])
@pytest.mark.parametrize("skip_first", [False, True])
def test_expansion_matches_exact_sums(b, skip_first):
    rng = np.random.default_rng(abs(b) + int(skip_first))
    walks = [np.zeros(64, dtype=int), np.ones(64, dtype=int)]  # monotone: heights cross 0 near |b| = 64
    walks += [rng.integers(0, 2, size=64) for _ in range(20)]
    for bits in walks:
        n, a = chunk_power_sums(bits, skip_first)
        d, exact = 0, [0] * 8
        for i, bit in enumerate(bits):
            d += 2 * int(bit) - 1
            if i == 0 and skip_first:
                continue
            for k in range(1, 8):
                exact[k] += (b + d) ** k
        # S1, S2 exact in int64, as the kernel forms them
        assert n * b + a[1] == exact[1]
        assert n * b * b + 2 * b * a[1] + a[2] == exact[2]
        for k, got in zip(range(3, 8), expand(b, n, a)):
            assert got == pytest.approx(exact[k], rel=RTOL, abs=1e-9), (k, b)
