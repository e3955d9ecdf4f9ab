"""16-bit compressed storage on the GPU (Storage::Compressed,
crates/solver/src/storage.rs:87-330) against the CPU oracle's restatement
of it (tests/test_oracle_compressed.py pins that one).

In exact precision the GPU performs the oracle's f32 operations in its
order, decode, update, block max and encode included, so the stored i16 /
u16 values and the per-node scales must be identical. In fast precision the
bar is the reference's own GPU compressed tests (gpu/engine/tests.rs:
201-240, one iteration from random storage within 1e-5; exploitability
within 1e-4). The mode stays close to f32 as the reference's
compressed_storage_is_close (tests.rs:273-303) asks."""
import numpy as np
import pytest

import spots
from oracle_api import OracleSolver
from poker_trainer_b200 import abi
from poker_trainer_b200.solver import Solver, SolveOptions

pytestmark = pytest.mark.gpu

SPOTS = {
    "river": spots.river_config,
    "turn": spots.turn_config,
    "iso_turn": spots.iso_turn_config,
    "mid_street_raked": lambda: spots.mid_street_config(True),
}


def compressed(cfg, precision=abi.PRECISION_EXACT):
    cfg.storage = abi.STORAGE_COMPRESSED
    cfg.precision = precision
    return cfg


def random_compressed(n, k, seed):
    rng = np.random.default_rng(seed)
    rq = rng.integers(-32767, 32768, n).astype(np.int16)
    rq[rng.random(n) < 0.3] = 0
    sq = rng.integers(0, 65536, n).astype(np.uint16)
    sq[rng.random(n) < 0.2] = 0
    rs = (rng.random(k) * 100).astype(np.float32)
    ss = (rng.random(k) * 20).astype(np.float32)
    return rq, sq, rs, ss


def assert_storage_equal(g, o, what):
    grq, gsq, grs, gss = g.download_storage_compressed()
    orq, osq, ors, oss = o.compressed_storage()
    for name, a, b in (("regrets", grq, orq), ("sums", gsq, osq)):
        diff = np.nonzero(a != b)[0]
        if len(diff):
            i = diff[0]
            pytest.fail(f"{what}: {name}: {len(diff)} of {len(a)} differ; first at {i}: gpu {a[i]} oracle {b[i]}")
    for name, a, b in (("regret scales", grs, ors), ("sum scales", gss, oss)):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), f"{what}: {name} differ"


@pytest.mark.parametrize("name", list(SPOTS))
def test_iterations_bit_identical(gpu, name):
    o = OracleSolver(compressed(SPOTS[name]()))
    g = Solver.new(compressed(SPOTS[name]()))
    assert o.compressed and g.stats().compressed
    assert g.storage_len() == len(o.compressed_storage()[0])
    for done in (1, 4):
        o.iterate(done if done == 1 else 3)
        g.iterate(done if done == 1 else 3)
        assert_storage_equal(g, o, f"{name} after {done} iterations")
    assert g.exploitability() == o.exploitability()


@pytest.mark.parametrize("name", ["river", "turn", "mid_street_raked"])
def test_one_iteration_from_random_storage(gpu, name):
    """gpu/engine/tests.rs:201-240 for compressed spots: the same random
    storage on both sides, one CFR iteration, the same storage after."""
    o = OracleSolver(compressed(SPOTS[name]()))
    g = Solver.new(compressed(SPOTS[name]()))
    n, k = g.storage_len(), g.storage_slots()
    st = random_compressed(n, k, 101)
    o.set_compressed_storage(*st)
    g.upload_storage_compressed(*st)
    o.set_iterations(3)
    g.set_iterations(3)
    o.iterate(1)
    g.iterate(1)
    assert_storage_equal(g, o, f"{name} one iteration from random storage")


@pytest.mark.parametrize("name", ["turn", "iso_turn"])
def test_fast_precision_matches_oracle(gpu, name):
    o = OracleSolver(compressed(SPOTS[name]()))
    g = Solver.new(compressed(SPOTS[name](), abi.PRECISION_FAST))
    o.iterate(20)
    g.iterate(20)
    eo, eg = o.exploitability(), g.exploitability()
    assert abs(eg - eo) <= 1e-4 * max(abs(eo), 1e-3), (eg, eo)
    # Decoded values within 1e-5 relative of the block scale.
    grq, gsq, grs, gss = g.download_storage_compressed()
    orq, osq, ors, oss = o.compressed_storage()
    assert np.allclose(grs, ors, rtol=1e-5, atol=1e-6)
    assert np.allclose(gss, oss, rtol=1e-5, atol=1e-6)


def test_fp64_oracle_and_decoded_download(gpu):
    g = Solver.new(compressed(spots.turn_config(), abi.PRECISION_FAST))
    g.iterate(30)
    e32 = g.exploitability()
    e64, _ = g.exploitability_fp64()
    assert abs(e64 - e32) <= 1e-4 * max(abs(e64), 1e-3), (e64, e32)
    # The f32 download of a compressed solver is its decoded storage.
    r, s = g.download_storage()
    rq, sq, rs, ss = g.download_storage_compressed()
    o = OracleSolver(compressed(spots.turn_config()))
    ints, offs, _, _ = o.nodes()
    nh = [o.num_hands(0), o.num_hands(1)]
    for v in np.nonzero(ints[:, 0] == 0)[0]:
        off, slot = int(offs[v, 0]), int(offs[v, 1])
        m = int(ints[v, 3]) * nh[int(ints[v, 1])]
        assert np.array_equal(r[off:off + m], rq[off:off + m].astype(np.float32) * np.float32(rs[slot] / np.float32(32767)))
        assert np.array_equal(s[off:off + m], sq[off:off + m].astype(np.float32) * np.float32(ss[slot] / np.float32(65535)))


def test_compressed_close_to_f32(gpu):
    """tests.rs:273-303 on the GPU: both modes solve below 0.5% of the pot,
    the root's range strategies agree within 0.03, and the compressed tree
    is the smaller one (4 bytes per cell against 8)."""
    a = Solver.new(compressed(spots.turn_config(), abi.PRECISION_FAST))
    f = spots.turn_config()
    f.precision = abi.PRECISION_FAST
    b = Solver.new(f)
    opts = SolveOptions(max_iterations=300, target_exploitability_pct=0.2, check_every=20)
    pa, pb = a.solve(opts), b.solve(opts)
    assert pa.exploitability_pct < 0.5 and pb.exploitability_pct < 0.5, (pa, pb)
    ra, rb = a.query().range_strategy(), b.query().range_strategy()
    assert max(abs(x - y) for x, y in zip(ra, rb)) < 0.03, (ra, rb)
    sa, sb = a.stats(), b.stats()
    assert sa.compressed and not sb.compressed
    assert sa.storage_cells == sb.storage_cells and sa.memory_bytes < sb.memory_bytes
