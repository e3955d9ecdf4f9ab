"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) for the tests.

The oracle is test infrastructure: a C++ restatement of the reference's CPU
DCFR solver. Tests use it as the checker of libdcfr; the product never loads
it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from poker_trainer_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        P = C.c_void_p
        L.oracle_create.restype = P
        L.oracle_create.argtypes = [C.POINTER(abi.Config), C.POINTER(C.c_int)]
        L.oracle_destroy.argtypes = [P]
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_estimate.argtypes = [C.POINTER(abi.Config), C.POINTER(abi.TreeStats)]
        L.oracle_set_batch_river.argtypes = [P, C.c_int]
        L.oracle_storage_len.restype = C.c_uint64
        L.oracle_storage_len.argtypes = [P]
        L.oracle_get_storage.argtypes = [P, P, P]
        L.oracle_is_compressed.argtypes = [P]
        L.oracle_num_slots.restype = C.c_uint64
        L.oracle_num_slots.argtypes = [P]
        L.oracle_get_storage_compressed.argtypes = [P, P, P, P, P]
        L.oracle_set_storage_compressed.argtypes = [P, P, P, P, P]
        L.oracle_set_storage.argtypes = [P, P, P]
        L.oracle_set_iterations.argtypes = [P, C.c_uint32]
        L.oracle_iterations.restype = C.c_uint32
        L.oracle_iterations.argtypes = [P]
        L.oracle_hands.argtypes = [P, C.c_int, P, P]
        L.oracle_stats.argtypes = [P, C.POINTER(abi.TreeStats)]
        L.oracle_isomorphic_pairs.argtypes = [P]
        L.oracle_num_nodes.restype = C.c_uint64
        L.oracle_num_nodes.argtypes = [P]
        L.oracle_nodes.argtypes = [P, P, P, P, P]
        L.oracle_iterate.argtypes = [P, C.c_uint32]
        L.oracle_exploitability.restype = C.c_double
        L.oracle_exploitability.argtypes = [P]
        L.oracle_root_values.argtypes = [P, P]
        L.oracle_traverse.argtypes = [P, C.c_int, C.c_int, C.c_uint32, P]
        L.oracle_solve.argtypes = [P, C.POINTER(abi.SolveOptions), abi.PROGRESS_CB, P, C.POINTER(abi.Progress)]
        L.oracle_query.argtypes = [P, P, C.c_size_t, C.POINTER(abi.NodeInfoHeader), P, P, P, P, P]
        L.oracle_query_sizes.argtypes = [P, P, C.c_size_t, P, P]
        L.oracle_ranges_after.argtypes = [P, P, C.c_size_t, P]
        L.oracle_actions_at.argtypes = [P, P, C.c_size_t, P, C.c_size_t, P]
        L.oracle_is_decision.argtypes = [P, P, C.c_size_t]
        L.oracle_evaluate.restype = C.c_uint32
        L.oracle_evaluate.argtypes = [P, C.c_int]
        L.oracle_five_card_counts.argtypes = [P]
        L.oracle_combos.argtypes = [P]
        L.oracle_combo_class.argtypes = [P]
        L.oracle_class_combos.argtypes = [C.c_int, P]
        L.oracle_parse_range.argtypes = [C.c_char_p, P]
        L.oracle_parse_cards.argtypes = [C.c_char_p, P, C.c_int]
        L.oracle_menu_actions.argtypes = [C.POINTER(abi.Menu), C.c_int, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                                          C.c_int64, C.c_uint32, C.c_int64, P, C.c_int]
        L.oracle_default_menu.argtypes = [C.POINTER(abi.Menu)]
        L.oracle_parse_bet_size.argtypes = [C.c_char_p, P, P]
        L.oracle_next_check_gap.restype = C.c_uint32
        L.oracle_next_check_gap.argtypes = [C.c_int, C.c_uint32, C.c_double, C.c_uint32, C.c_double, C.c_double,
                                            C.c_uint32]
        L.oracle_discount.argtypes = [C.c_uint32, C.POINTER(abi.Params), P]
        L.oracle_board_symmetric_pairs.argtypes = [P, C.c_int, P]
        L.oracle_iso_orbit.argtypes = [P, C.c_int, C.c_int, P]
        L.oracle_handset_create.restype = P
        L.oracle_handset_create.argtypes = [P, P, P, C.c_int]
        L.oracle_handset_destroy.argtypes = [P]
        L.oracle_handset_len.argtypes = [P, C.c_int]
        L.oracle_handset_num_combinations.restype = C.c_double
        L.oracle_handset_num_combinations.argtypes = [P]
        L.oracle_handset_cards.argtypes = [P, C.c_int, P]
        L.oracle_compatible_reach.argtypes = [P, C.c_int, P, P]
        L.oracle_eval_fold.argtypes = [P, C.c_int, P, C.c_double, P]
        L.oracle_eval_showdown.argtypes = [P, C.c_int, P, C.c_double, C.c_double, C.c_double, P]
        L.oracle_fold_batch.argtypes = [P, C.c_int, C.c_int, P, P, P]
        L.oracle_showdown_batch.argtypes = [P, C.c_int, C.c_int, P, P, P, P, P, P, P]
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_get_threads.restype = C.c_int
        L.oracle_chacha_block.argtypes = [P, C.c_uint64, C.c_uint64, C.c_int, P]
        L.oracle_chacha_block.restype = None
        L.oracle_rng_u64.argtypes = [C.c_uint64, C.c_uint64, P]
        L.oracle_rng_u64.restype = None
        L.oracle_sample_cards.argtypes = [P, C.c_int32, C.c_int32, C.c_uint64, P]
        L.oracle_sample_cards.restype = C.c_int
        _lib = L
    return _lib


def ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def parse_range(s: str) -> np.ndarray:
    out = np.zeros(1326, np.float32)
    rc = lib().oracle_parse_range(s.encode(), ptr(out))
    if rc:
        raise ValueError(lib().oracle_last_error().decode())
    return out


def chacha_block(key: np.ndarray, counter: int, stream: int, rounds: int) -> np.ndarray:
    """One ChaCha block as 16 u32 words (the sampled chance mode's core)."""
    key = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(16, np.uint32)
    lib().oracle_chacha_block(ptr(key), counter, stream, rounds, ptr(out))
    return out


def rng_u64(seed: int, n: int) -> np.ndarray:
    """The first n 64-bit draws of StdRng::seed_from_u64(seed)."""
    out = np.zeros(n, np.uint64)
    lib().oracle_rng_u64(seed, n, ptr(out))
    return out


def sample_cards(available, k: int, seed: int) -> list[int]:
    """sampling.rs:9-54 with a fresh StdRng::seed_from_u64(seed)."""
    a = np.ascontiguousarray(available, dtype=np.int32)
    out = np.zeros(max(len(a), 1), np.int32)
    n = lib().oracle_sample_cards(ptr(a), len(a), k, seed, ptr(out))
    return [int(x) for x in out[:n]]


def estimate(cfg: abi.Config) -> abi.TreeStats:
    st = abi.TreeStats()
    rc = lib().oracle_estimate(C.byref(cfg), C.byref(st))
    if rc:
        raise RuntimeError(f"estimate failed ({rc}): {lib().oracle_last_error().decode()}")
    return st


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class OracleSolver:
    """The oracle's Solver (crates/solver/src/lib.rs:288-913 restated)."""

    def __init__(self, cfg: abi.Config):
        err = C.c_int(0)
        self.h = lib().oracle_create(C.byref(cfg), C.byref(err))
        if not self.h:
            raise OracleError(err.value, lib().oracle_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    def set_batch_river(self, on: bool):
        lib().oracle_set_batch_river(self.h, int(on))

    def hands(self, p):
        n = lib().oracle_hands(self.h, p, None, None)
        combos = np.zeros(n, np.uint16)
        w = np.zeros(n, np.float32)
        lib().oracle_hands(self.h, p, ptr(combos), ptr(w))
        return combos, w

    def num_hands(self, p):
        return lib().oracle_hands(self.h, p, None, None)

    def stats(self):
        st = abi.TreeStats()
        lib().oracle_stats(self.h, C.byref(st))
        return st

    def isomorphic_pairs(self):
        return lib().oracle_isomorphic_pairs(self.h)

    def storage(self):
        n = lib().oracle_storage_len(self.h)
        r = np.zeros(n, np.float32)
        s = np.zeros(n, np.float32)
        lib().oracle_get_storage(self.h, ptr(r), ptr(s))
        return r, s

    def set_storage(self, r, s):
        r = np.ascontiguousarray(r, np.float32)
        s = np.ascontiguousarray(s, np.float32)
        assert len(r) == lib().oracle_storage_len(self.h)
        lib().oracle_set_storage(self.h, ptr(r), ptr(s))

    @property
    def compressed(self) -> bool:
        return bool(lib().oracle_is_compressed(self.h))

    def compressed_storage(self):
        """(i16 regrets, u16 sums, regret scales, sum scales) of a compressed
        solver (storage.rs:92-97)."""
        n = lib().oracle_storage_len(self.h)
        k = lib().oracle_num_slots(self.h)
        rq = np.zeros(n, np.int16)
        sq = np.zeros(n, np.uint16)
        rs = np.zeros(k, np.float32)
        ss = np.zeros(k, np.float32)
        assert lib().oracle_get_storage_compressed(self.h, ptr(rq), ptr(sq), ptr(rs), ptr(ss)) == 0
        return rq, sq, rs, ss

    def set_compressed_storage(self, rq, sq, rs, ss):
        rq = np.ascontiguousarray(rq, np.int16)
        sq = np.ascontiguousarray(sq, np.uint16)
        rs = np.ascontiguousarray(rs, np.float32)
        ss = np.ascontiguousarray(ss, np.float32)
        assert lib().oracle_set_storage_compressed(self.h, ptr(rq), ptr(sq), ptr(rs), ptr(ss)) == 0

    def set_iterations(self, t):
        lib().oracle_set_iterations(self.h, t)

    @property
    def iterations(self):
        return lib().oracle_iterations(self.h)

    def nodes(self):
        n = lib().oracle_num_nodes(self.h)
        ints = np.zeros((n, 9), np.int32)
        offs = np.zeros((n, 2), np.uint64)
        fl = np.zeros((n, 2), np.float32)
        am = np.zeros(n, np.int64)
        lib().oracle_nodes(self.h, ptr(ints), ptr(offs), ptr(fl), ptr(am))
        return ints, offs, fl, am

    def iterate(self, n):
        lib().oracle_iterate(self.h, n)

    def exploitability(self):
        return lib().oracle_exploitability(self.h)

    def root_values(self):
        out = np.zeros(2, np.float64)
        lib().oracle_root_values(self.h, ptr(out))
        return out

    def traverse(self, p, mode, t):
        out = np.zeros(self.num_hands(p), np.float32)
        lib().oracle_traverse(self.h, p, mode, t, ptr(out))
        return out

    def solve(self, max_iterations, target_pct, check_every, history=None):
        opts = abi.SolveOptions(max_iterations, check_every, target_pct)

        def cb(p, _user):
            if history is not None:
                history.append((p.contents.iteration, p.contents.exploitability))
            return 1

        cbf = abi.PROGRESS_CB(cb)
        out = abi.Progress()
        lib().oracle_solve(self.h, C.byref(opts), cbf, None, C.byref(out))
        return out

    def query(self, path=()):
        steps, n = abi.path_steps(path)
        na = C.c_int32(0)
        nh = C.c_int32(0)
        rc = lib().oracle_query_sizes(self.h, steps, n, C.byref(na), C.byref(nh))
        if rc:
            raise OracleError(rc, lib().oracle_last_error().decode())
        info = abi.NodeInfoHeader()
        acts = (abi.ActionT * na.value)()
        combos = np.zeros(nh.value, np.uint16)
        strat = np.zeros(na.value * nh.value, np.float32)
        ev = np.zeros(na.value * nh.value, np.float32)
        reach = np.zeros(nh.value, np.float32)
        rc = lib().oracle_query(self.h, steps, n, C.byref(info), acts, ptr(combos), ptr(strat), ptr(ev), ptr(reach))
        if rc:
            raise OracleError(rc, lib().oracle_last_error().decode())
        return dict(player=info.player, actions=[(a.kind, a.amount) for a in acts], combos=combos,
                    strategy=strat.reshape(na.value, nh.value), ev=ev.reshape(na.value, nh.value), reach=reach,
                    reach_fraction=(info.reach_fraction[0], info.reach_fraction[1]), pot=info.pot,
                    invest=(info.invest[0], info.invest[1]))

    def ranges_after(self, path=()):
        steps, n = abi.path_steps(path)
        out = np.zeros((2, 1326), np.float32)
        rc = lib().oracle_ranges_after(self.h, steps, n, ptr(out))
        if rc:
            raise OracleError(rc, lib().oracle_last_error().decode())
        return out

    def actions_at(self, path=()):
        steps, n = abi.path_steps(path)
        acts = (abi.ActionT * 16)()
        cnt = C.c_size_t(0)
        rc = lib().oracle_actions_at(self.h, steps, n, acts, 16, C.byref(cnt))
        if rc:
            raise OracleError(rc, lib().oracle_last_error().decode())
        return [(acts[i].kind, acts[i].amount) for i in range(cnt.value)]

    def is_decision(self, path=()):
        steps, n = abi.path_steps(path)
        return bool(lib().oracle_is_decision(self.h, steps, n))


class HandSetOracle:
    """hands.rs HandSet + StrengthTable on a board, for evaluator tests."""

    def __init__(self, r0, r1, board):
        b = np.array(board, np.int32)
        self.r0 = np.ascontiguousarray(r0, np.float32)
        self.r1 = np.ascontiguousarray(r1, np.float32)
        self.h = lib().oracle_handset_create(ptr(self.r0), ptr(self.r1), ptr(b), len(b))

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_handset_destroy(self.h)

    def len(self, p):
        return lib().oracle_handset_len(self.h, p)

    def num_combinations(self):
        return lib().oracle_handset_num_combinations(self.h)

    def cards(self, p):
        out = np.zeros((self.len(p), 2), np.uint8)
        lib().oracle_handset_cards(self.h, p, ptr(out))
        return out

    def compatible_reach(self, p, r):
        r = np.ascontiguousarray(r, np.float32)
        out = np.zeros(self.len(p), np.float64)
        lib().oracle_compatible_reach(self.h, p, ptr(r), ptr(out))
        return out

    def eval_fold(self, p, r, payoff):
        r = np.ascontiguousarray(r, np.float32)
        out = np.zeros(self.len(p), np.float32)
        lib().oracle_eval_fold(self.h, p, ptr(r), payoff, ptr(out))
        return out

    def eval_showdown(self, p, r, w, l, t):
        r = np.ascontiguousarray(r, np.float32)
        out = np.zeros(self.len(p), np.float32)
        lib().oracle_eval_showdown(self.h, p, ptr(r), w, l, t, ptr(out))
        return out

    def fold_batch(self, p, reaches, payoffs):
        k = len(reaches)
        rs = [np.ascontiguousarray(r, np.float32) for r in reaches]
        outs = [np.zeros(self.len(p), np.float32) for _ in range(k)]
        rp = (C.c_void_p * k)(*[r.ctypes.data for r in rs])
        op = (C.c_void_p * k)(*[o.ctypes.data for o in outs])
        pay = np.array(payoffs, np.float64)
        lib().oracle_fold_batch(self.h, p, k, rp, ptr(pay), op)
        return outs

    def showdown_batch(self, p, reaches, win, lose, tie, fold_pay=None):
        k = len(reaches)
        rs = [np.ascontiguousarray(r, np.float32) for r in reaches]
        outs = [np.zeros(self.len(p), np.float32) for _ in range(k)]
        fouts = [np.zeros(self.len(p), np.float32) for _ in range(k)]
        rp = (C.c_void_p * k)(*[r.ctypes.data for r in rs])
        op = (C.c_void_p * k)(*[o.ctypes.data for o in outs])
        if fold_pay is not None:
            fp = (C.c_void_p * k)(*[fouts[t].ctypes.data if fold_pay[t] is not None else None for t in range(k)])
            fpay = np.array([x if x is not None else 0.0 for x in fold_pay], np.float64)
        else:
            fp, fpay = None, None
        w, l, t = (np.array(x, np.float64) for x in (win, lose, tie))
        lib().oracle_showdown_batch(self.h, p, k, rp, ptr(w), ptr(l), ptr(t), op,
                                    ptr(fpay) if fpay is not None else None, fp)
        return outs, fouts
