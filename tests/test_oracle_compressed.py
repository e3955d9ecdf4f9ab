"""16-bit compressed storage in the oracle (storage.rs:87-330): pinned by
the reference's own test of the mode, compressed_storage_is_close
(crates/solver/src/tests.rs:273-303), and by its storage rules restated on
a single node."""
import numpy as np

from oracle_api import OracleSolver, parse_range
from poker_trainer_b200 import abi

OOP = "AQ, KQ, QJs, JTs, 99, 44, T9s, 87s, A5s, KJs"
IP = "AA, KK, AQ, QT, 99, JJ, TT, 98s, KJs, 65s, AJs"


def turn_config(storage):
    """tests.rs:275-287: Qh9d4c2s, pot 600, stacks 4000, the default menu."""
    return abi.make_config("Qh9d4c2s", [parse_range(OOP), parse_range(IP)], pot=600, stack=4000,
                           menu_=abi.default_menu(), storage=storage)


def range_strategy(node):
    s = np.asarray(node["strategy"], np.float64)
    w = np.asarray(node["reach"], np.float64)
    return (s * w[None, :]).sum(1) / w.sum()


def test_compressed_storage_is_close():
    a = OracleSolver(turn_config(abi.STORAGE_COMPRESSED))
    b = OracleSolver(turn_config(abi.STORAGE_F32))
    assert a.compressed and not b.compressed
    assert a.stats().memory_bytes < b.stats().memory_bytes
    pa = a.solve(300, 0.2, 20)
    pb = b.solve(300, 0.2, 20)
    assert pa.exploitability_pct < 0.5, pa
    assert pb.exploitability_pct < 0.5, pb
    ra, rb = range_strategy(a.query()), range_strategy(b.query())
    assert np.max(np.abs(ra - rb)) < 0.03, (ra, rb)


def test_compressed_storage_scales_and_rounding():
    """After a CFR iteration every player node's scale is the max |value| of
    its block, and the block's largest value encodes to 32767 (regrets) or
    65535 (sums): the encoding of storage.rs:272-330."""
    s = OracleSolver(turn_config(abi.STORAGE_COMPRESSED))
    s.iterate(3)
    rq, sq, rs, ss = s.compressed_storage()
    ints, offs, fl, am = s.nodes()
    kind, player, nchild = ints[:, 0], ints[:, 1], ints[:, 3]
    nh = [s.num_hands(0), s.num_hands(1)]
    checked = 0
    for v in np.nonzero(kind == 0)[0][:200]:
        off, slot = int(offs[v, 0]), int(offs[v, 1])
        n = nchild[v] * nh[player[v]]
        r = rq[off:off + n].astype(np.int32)
        q = sq[off:off + n].astype(np.int32)
        if rs[slot] > 0:
            assert np.abs(r).max() == 32767
            checked += 1
        else:
            assert not r.any()
        if ss[slot] > 0:
            assert q.max() == 65535
        else:
            assert not q.any()
    assert checked > 0
