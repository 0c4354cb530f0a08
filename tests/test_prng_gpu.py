"""Device fill of the generators (modlin_prng_fill_device) against the host
stream (modlin_prng_fill, itself pinned to the oracle and to the reference's
golden outputs): bit-identical outputs and generator state, raw and reduced,
interleaved with host fills, and from planted states that make ROOT's folds
leave 2^61 - 1 where the residue is 0 (src/prng.rs:117-222)."""
import numpy as np
import pytest
import torch

from mixmax_model import M61, MIX, plant, set_mix_state

pytestmark = pytest.mark.gpu

KINDS = ["xoroshiro128pp", "mixmax17", "mixmax", "mixmax256"]


def dev_fill(g, count, p=0):
    t = torch.empty(max(count, 1), dtype=torch.int64, device="cuda")
    g.fill_device(t.data_ptr(), count, p)
    torch.cuda.synchronize()
    return t[:count].cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("kind", KINDS)
def test_fill_matches_host_stream(M, kind):
    for seed in (1, 0x9E3779B97F4A7C15):
        for count in (1, 7, 255, 256, 257, 4097, 100_003, 3_000_017):
            h, d = M.prng.Prng(kind, seed), M.prng.Prng(kind, seed)
            assert np.array_equal(dev_fill(d, count), h.fill(count)), (kind, seed, count)
            assert np.array_equal(d.get_state(), h.get_state()), (kind, seed, count)


@pytest.mark.parametrize("kind", KINDS)
def test_fill_interleaves_with_host(M, kind):
    """Host and device fills share one position (src/main.rs:82: reps read
    disjoint stretches of the orbit)."""
    ref = M.prng.Prng(kind, 7).fill(2_000_000)
    g = M.prng.Prng(kind, 7)
    parts, pos = [], 0
    for n, where in [(3, "h"), (500, "d"), (1, "d"), (254, "h"), (77_777, "d"), (12, "h"), (1_000_000, "d"),
                     (5, "d"), (921_448, "h")]:
        parts.append(dev_fill(g, n) if where == "d" else g.fill(n))
        pos += n
    assert np.array_equal(np.concatenate(parts), ref[:pos])


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("p", [2, 65521, 4294967291, M61, (1 << 62) - 57])
def test_fill_reduced(M, kind, p):
    """Field::reduce of each output, as the -R/-L fill does (src/main.rs:94-104)."""
    raw = M.prng.Prng(kind, 3).fill(300_001)
    got = dev_fill(M.prng.Prng(kind, 3), 300_001, p)
    assert np.array_equal(got, raw % np.uint64(p))


def test_fill_large_mixmax256(M):
    """A long stream: 2^26 outputs spread over every resident warp."""
    n = 1 << 26
    h, d = M.prng.Prng("mixmax256", 1), M.prng.Prng("mixmax256", 1)
    assert np.array_equal(dev_fill(d, n, M61), h.fill(n) % np.uint64(M61))
    assert np.array_equal(d.get_state(), h.get_state())


def test_fill_zero_count_and_errors(M):
    g = M.prng.Prng("mixmax17", 1)
    s = g.get_state()
    g.fill_device(0, 0)
    assert np.array_equal(g.get_state(), s)
    with pytest.raises(M.ModlinError):
        g.fill_device(0, 10)
    t = torch.empty(4, dtype=torch.int64, device="cuda")
    with pytest.raises(M.ModlinError):
        g.fill_device(t.data_ptr(), 4, 1)  # p = 1 is not a field


# ---- planted states: the exact path and the segment repair -----------------

@pytest.mark.parametrize("kind", ["mixmax17", "mixmax", "mixmax256"])
def test_planted_zero_entries(M, kind):
    """Entries = 0 planted at block ends (ROOT then holds 2^61 - 1 there and
    outputs (2^61 - 1) << 3), in the middle of a multi-iteration block, and
    2^61 - 1 entries in the starting state itself. With few blocks every
    block is its own segment, so block-end plants exercise the repair of the
    next segment's start."""
    N, _, skip, _ = MIX[kind]
    per = skip + 1
    rng = np.random.default_rng(N)
    zeros = [(per * 1, 5), (per * 2, 1), (per * 7, N - 1), (per * 40 + (1 if per > 1 else 0), 9)]
    x = plant(kind, rng, zeros)
    count = 60 * (N - 1) + 11
    for counter in (N, 2, N - 1):
        h, d = M.prng.Prng(kind, 1), M.prng.Prng(kind, 1)
        set_mix_state(h, kind, x, counter)
        set_mix_state(d, kind, x, counter)
        ref = h.fill(count)
        assert np.count_nonzero(ref == np.uint64((M61 << 3) & ((1 << 64) - 1))) >= 2
        assert np.array_equal(dev_fill(d, count), ref), (kind, counter)
        assert np.array_equal(d.get_state(), h.get_state())
    # 2^61 - 1 and 0 entries in the starting state
    y = list(x)
    y[0], y[4], y[6] = M61, M61, 0
    h, d = M.prng.Prng(kind, 1), M.prng.Prng(kind, 1)
    set_mix_state(h, kind, y, N)
    set_mix_state(d, kind, y, N)
    assert np.array_equal(dev_fill(d, count), h.fill(count))
    assert np.array_equal(d.get_state(), h.get_state())


def test_rank_prng_matches_host_matrix(M, O):
    """modlin_rank_prng: the -R matrix generated and ranked on the device."""
    for kind, n, p in [("mixmax17", 300, M61), ("xoroshiro128pp", 257, 65521), ("mixmax256", 600, 7)]:
        g = M.prng.Prng(kind, 11)
        r = M.fp.rank_prng(p, g, n)
        x = M.prng.Prng(kind, 11).fill(n * n) % np.uint64(p)
        assert r == M.fp.rank(p, x, n)
        h = M.prng.Prng(kind, 11)
        h.fill(n * n)
        assert np.array_equal(g.get_state(), h.get_state())
