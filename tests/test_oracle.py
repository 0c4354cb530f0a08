"""The CPU oracle against the reference crate's own tests and golden vectors.

Ports, case for case, src/fp.rs:314-367 (barrett_matches_division),
tests/test_rank.rs, tests/test_linear_complexity.rs, tests/test_prng.rs,
tests/test_stats.rs and the README's end-to-end runs.
"""
import json
import os

import numpy as np
import pytest

from conftest import M61

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
REF = GOLD["reference"]


def mix2(x):  # src/fp.rs:318-322
    z = (x * 0x9E3779B97F4A7C15) & (2**64 - 1)
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & (2**64 - 1)
    return z ^ (z >> 31)


def test_barrett_matches_division(O):
    """src/fp.rs:314-367."""
    for p in [2, 3, 97, 65537, (1 << 31) - 1, (1 << 61) - 1, M61, (1 << 62) + 135, (1 << 63) - 25]:
        f = O.Field(p)
        corners = [0, 1, p - 1, p, p + 1, 2**128 - 1, 2**128 - 2, 1 << 127, (1 << 127) | 1]
        corners += [(mix2(i) << 64) | mix2(i ^ 0xABCD) for i in range(256)]
        for t in corners:
            assert f.reduce_u128(t) == t % p, (p, t)
        for x in [0, 1, p - 1, p, 2**64 - 1, 2**64 - 2]:
            assert f.reduce(x) == x % p
        for i in range(256):
            a, b = mix2(i) % p, mix2(i ^ 0x1234) % p
            assert f.mul(a, b) == a * b % p


def test_safe_batch(O):
    """src/fp.rs:53-59: 64 for 2^61-1, 4 for p near 2^63."""
    assert O.Field(M61).safe_batch == 64
    assert O.Field((1 << 63) - 25).safe_batch == 4


def test_rank_of_known_matrices(O):
    """tests/test_rank.rs:74-97."""
    assert O.rank(M61, np.eye(3, dtype=np.uint64), 3) == 3
    assert O.rank(M61, [1, 2, 3, 4, 5, 6, 5, 7, 9], 3) == 2
    assert O.rank(M61, np.zeros(16, dtype=np.uint64), 4) == 0
    assert O.rank(2, [1, 1, 0, 0, 1, 1, 1, 0, 1], 3) == 2


def test_blocked_matches_reference(O):
    """tests/test_rank.rs:99-149: blocked rank == naive rank on the panel-boundary grid."""
    ts = O.TestStream()
    for p in [2, 97, M61]:
        for n in [1, 2, 5, 63, 64, 65, 129, 200, 257, 300]:
            for target in [n, n // 2, n // 3, 1, 0]:
                a = ts.rank_case(p, n, target)
                expected = O.rank_naive(p, a, n)
                assert O.rank(p, a, n) == expected, (p, n, target)
                assert expected <= min(target, n)


def test_linear_complexity_of_lfsr_sequence(O):
    """tests/test_linear_complexity.rs:72-91."""
    s = [1, 2, 3]
    for i in range(3, 40):
        s.append((3 * s[i - 1] + 5 * s[i - 2] + 7 * s[i - 3]) % M61)
    assert O.linear_complexity(M61, s) == 3
    assert O.linear_complexity(M61, [4] * 20) == 1
    assert O.linear_complexity(M61, [0] * 20) == 0


def test_lc_matches_reference(O):
    """tests/test_linear_complexity.rs:93-133."""
    ts = O.TestStream()
    for p in [2, 3, 97, 65537, M61]:
        for n in [1, 2, 3, 5, 16, 50, 100, 200]:
            s = ts.lc_random(p, n)
            assert O.linear_complexity(p, s) == O.lc_naive(p, s), (p, n)
        for k in [1, 4, 10, 25]:
            s = ts.lc_lfsr(p, k)
            got = O.linear_complexity(p, s)
            assert got == O.lc_naive(p, s) and got <= k, (p, k, got)


@pytest.mark.parametrize("kind,key", [("mixmax17", "mixmax17"), ("mixmax", "mixmax240"), ("mixmax256", "mixmax256")])
def test_matches_official_mixmax(O, kind, key):
    """tests/test_prng.rs:13-72."""
    raw = [int(x) >> 3 for x in O.prng(kind, REF["mixmax_seed"], 10)]
    assert raw == REF[key]


def test_matches_reference_xoroshiro(O):
    """tests/test_prng.rs:81-111."""
    assert [int(x) for x in O.prng("xoroshiro128pp", 0, 10)] == REF["xoroshiro_seed0"]


def test_mixmax_rejects_zero_seed(O):
    """src/prng.rs:153-155."""
    with pytest.raises(ValueError):
        O.prng("mixmax17", 0, 1)


def test_corank_distribution_sane(O):
    """tests/test_stats.rs:11-23."""
    p0 = O.corank_prob(M61, 64, 0)
    assert abs(p0 - (1.0 - 1.0 / M61)) / p0 < 1e-12
    p1 = O.corank_prob(M61, 64, 1)
    assert abs(p1 - 1.0 / M61) / p1 < 1e-6
    assert abs(O.corank_prob(2, 256, 0) - 0.2887880951) < 1e-6
    assert abs(sum(O.corank_prob(M61, 64, d) for d in range(65)) - 1.0) < 1e-12


def test_single_observation_tails(O):
    """tests/test_stats.rs:25-37 (exact equalities)."""
    n = 305
    assert O.corank_tail_pvalue(M61, n, 0) == 1.0
    p1 = O.corank_tail_pvalue(M61, n, 1)
    assert abs(p1 - 1.0 / M61) / p1 < 1e-6
    assert O.corank_tail_pvalue(M61, n, 33) == 1e-307
    assert O.lc_left_tail_pvalue(M61, 10_000, 5000) == 1.0
    assert O.lc_left_tail_pvalue(M61, 10_000, 272) == 1e-307
    p = O.lc_left_tail_pvalue(2, 100, 40)
    assert 0.0 < p < 1.0


def test_lc_left_tail_is_exact_finite_n(O):
    """tests/test_stats.rs:39-71."""
    assert abs(O.lc_left_tail_pvalue(2, 2, 1) - 0.75) < 1e-12
    assert abs(O.lc_left_tail_pvalue(2, 5, 2) - 0.34375) < 1e-12
    assert abs(O.lc_left_tail_pvalue(2, 5, 3) - 0.84375) < 1e-12

    def pmf(q, n, l):
        if l == 0:
            return q ** -n
        if 2 * l <= n:
            return (q - 1.0) * q ** (2 * l - n - 1)
        return (q - 1.0) * q ** (n - 2 * l)

    for q in [2, 3, 5, 7]:
        for n in range(1, 25):
            cdf = 0.0
            for ell in range(n + 1):
                cdf += pmf(float(q), n, ell)
                got = O.lc_left_tail_pvalue(q, n, ell)
                assert abs(got - min(cdf, 1.0)) <= 1e-9 * cdf + 1e-15, (q, n, ell)


def test_readme_runs_small(O):
    """README.md:61-158 end-to-end known answers (the sizes that run in seconds)."""
    for kind, test, size, p, seed, stat, pstr in REF["readme_runs"]:
        if size > 10000:
            continue
        count = size * size if test == "R" else size
        x = np.array([int(v) % p for v in O.prng(kind, seed, count)], dtype=np.uint64)
        if test == "R":
            c = size - O.rank(p, x, size)
            assert c == stat
            assert O.pretty_p_value(O.corank_tail_pvalue(p, size, c)) == pstr
        else:
            lc = O.linear_complexity(p, x)
            assert lc == stat
            assert O.pretty_p_value(O.lc_left_tail_pvalue(p, size, lc)) == pstr


def test_pretty_matches_rust_debug(O):
    for hx, s in GOLD["oracle"]["pretty"]:
        assert O.pretty_p_value(float.fromhex(hx)) == s


def test_is_prime(O):
    small = [q for q in range(2, 500) if all(q % d for d in range(2, int(q ** 0.5) + 1))]
    assert [q for q in range(500) if O.is_prime(q)] == small
    for q in [M61, (1 << 62) + 135, (1 << 63) - 25, 2147483647, 65521]:
        assert O.is_prime(q)
    for c in [(1 << 61) + 1, (1 << 62) - 1, 3215031751, 341550071728321, 3825123056546413051]:
        assert not O.is_prime(c)
