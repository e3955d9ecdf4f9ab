"""The sampled chance mode on the CPU (ChanceMode::Sampled,
crates/solver/src/tree.rs:128-136, 302-334; sampling.rs:9-54).

The reference draws the sample from rand 0.9.5's StdRng (rand_chacha 0.9.0's
ChaCha12Rng, keyed by rand_core 0.9's PCG32 expansion of the u64 seed). Rust
cannot run here, so the sampled cards themselves are not pinned against the
reference's output. What is pinned:

- the ChaCha block function and its counter and stream words, against an
  independent ChaCha20 (the `cryptography` package's), at 20 rounds; StdRng
  runs the same function at 12;
- the reference's own test of the sampler (sampling.rs:63-76: seed 1, flop
  AsKs7d, 12 picks, two or three spades, all available);
- the stratification rules of sampling.rs for many seeds, boards and sizes;
- the tree counts of libdcfr's host builder against the oracle's
  (test_abi.py), including a tree whose size depends on the drawn turn cards.
"""
import numpy as np
import pytest

import spots
from oracle_api import chacha_block, estimate, rng_u64, sample_cards
from poker_trainer_b200 import abi


def test_chacha20_block_matches_an_independent_implementation():
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms

    rng = np.random.default_rng(11)
    for t in range(8):
        key = rng.integers(0, 2**32, 8, dtype=np.uint64).astype(np.uint32)
        counter = 0 if t == 0 else int(rng.integers(0, 2**40))
        stream = 0 if t < 2 else int(rng.integers(0, 2**63))
        # Words 12-15 as little-endian bytes: the 64-bit counter, then the stream.
        nonce = counter.to_bytes(8, "little") + stream.to_bytes(8, "little")
        enc = Cipher(algorithms.ChaCha20(key.tobytes(), nonce), mode=None).encryptor()
        want = np.frombuffer(enc.update(bytes(64 * 4)), dtype="<u4")
        got = np.concatenate([chacha_block(key, counter + b, stream, 20) for b in range(4)])
        assert np.array_equal(got, want), t


def test_twelve_rounds_differ_from_twenty():
    key = np.arange(8, dtype=np.uint32)
    assert not np.array_equal(chacha_block(key, 0, 0, 12), chacha_block(key, 0, 0, 20))


def test_rng_is_deterministic_and_seed_dependent():
    a, b, c = rng_u64(3, 100), rng_u64(3, 100), rng_u64(4, 100)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)
    # 100 draws cross the four-block buffer (32 draws per buffer) three times.
    assert len(set(a.tolist())) == 100
    # Top 53 bits uniform: the mean of the f64 draws is near 1/2.
    f = (rng_u64(9, 4096) >> np.uint64(11)).astype(np.float64) / 2.0**53
    assert 0.0 <= f.min() and f.max() < 1.0 and abs(f.mean() - 0.5) < 0.02


def cards_off(board: str) -> list[int]:
    used = set(abi.parse_cards(board))
    return [c for c in range(52) if c not in used]


def test_stratified_by_suit_reference_case():
    """sampling.rs:63-76."""
    available = cards_off("AsKs7d")
    picks = sample_cards(available, 12, 1)
    assert len(picks) == 12
    spades = sum(1 for c in picks if c % 4 == 3)
    assert 2 <= spades <= 3, spades
    assert all(c in available for c in picks)


@pytest.mark.parametrize("board", ["AsKs7d", "Kh7d2c", "Qs9s4d2d", "Qh9d4c2s", "2c3c4c5c"])
def test_stratification_rules(board):
    available = cards_off(board)
    per_suit = [sum(1 for c in available if c % 4 == s) for s in range(4)]
    for k in (1, 4, 6, 8, 12, 20, len(available) - 1):
        for seed in range(12):
            picks = sample_cards(available, k, seed)
            assert picks == sorted(set(picks)), "sorted and distinct"
            assert len(picks) == k
            assert all(c in available for c in picks)
            for s in range(4):
                exact = k * per_suit[s] / len(available)
                got = sum(1 for c in picks if c % 4 == s)
                assert int(np.floor(exact)) <= got <= int(np.floor(exact)) + 1, (k, seed, s)
                # Within a suit, ranks spread evenly: consecutive picks are
                # floor(step) or ceil(step) apart in rank order, step = m / q.
                suit_cards = [c for c in available if c % 4 == s]
                pos = [suit_cards.index(c) for c in picks if c % 4 == s]
                if got >= 2:
                    gaps = np.diff(pos)
                    step = per_suit[s] / got
                    assert gaps.min() >= np.floor(step) and gaps.max() <= np.ceil(step), (gaps, step)
    assert sample_cards(available, len(available), 0) == available
    assert sample_cards(available, len(available) + 5, 0) == available


def test_seeds_draw_different_samples():
    available = cards_off("Kh7d2c")
    samples = {tuple(sample_cards(available, 8, seed)) for seed in range(40)}
    assert len(samples) > 20


def test_sampled_tree_sizes():
    """Sampled trees are smaller than exact ones, chance nodes deal k cards,
    and all-in runouts stay exact (tree.rs:327-333)."""
    ex = spots.turn_config()
    sm = spots.sampled_turn_config()
    e, s = estimate(ex), estimate(sm)
    # 48 rivers against 6: every post-river subtree shrinks by 8x.
    assert s.storage_cells < e.storage_cells and s.chance_nodes == e.chance_nodes
    allin = estimate(spots.allin_turn_config())
    sallin = estimate(spots.sampled_allin_turn_config())
    assert sallin.chance_nodes == allin.chance_nodes
    assert sallin.terminal_nodes < allin.terminal_nodes


def test_sampled_flop_estimate_reference_case():
    """tests.rs:151-170: Solver::estimate of the sampled flop has player nodes."""
    st = estimate(spots.sampled_flop_config())
    assert st.player_nodes > 0
    ex = spots.sampled_flop_config()
    ex.chance = abi.CHANCE_EXACT
    assert estimate(ex).storage_cells > 10 * st.storage_cells
