"""Python mirror of the reference solver crate's public API over libdcfr.

Same names, argument meaning and error behaviour as
AhanDatta/Poker-Trainer crates/solver/src/lib.rs: `Solver.new(config)`
raises the SolverError variants (EmptyRange, InvalidBoard, TooLarge,
BadPath), `solve(opts, on_progress)` runs DCFR with the exploitability-check
schedule, `query(path)` returns a NodeInfo, and so on. Every call goes to
the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdcfr.so")
_lib = None

# Every entry point of include/dcfr.h.
EXPORTS = [
    "dcfr_last_error", "dcfr_config_init", "dcfr_estimate", "dcfr_create", "dcfr_destroy", "dcfr_solve",
    "dcfr_iterate", "dcfr_synchronize", "dcfr_exploitability", "dcfr_root_values", "dcfr_iterations",
    "dcfr_last_exploitability", "dcfr_stats", "dcfr_isomorphic_pairs", "dcfr_hands", "dcfr_is_decision",
    "dcfr_actions_at", "dcfr_query_sizes", "dcfr_query", "dcfr_ranges_after", "dcfr_storage_len",
    "dcfr_download_storage", "dcfr_upload_storage", "dcfr_set_iterations", "dcfr_traverse",
    "dcfr_kernel_launches", "dcfr_last_iterate_ms", "dcfr_iteration_bytes", "dcfr_iterate_profiled",
    "dcfr_terminal_kernel", "dcfr_last_solve_ms", "dcfr_setup_profile_get",
    "dcfr_showdown_values_noalloc", "dcfr_exploitability_fp64",
    "dcfr_batch_create", "dcfr_batch_destroy", "dcfr_batch_iterate", "dcfr_batch_exploitability",
    "dcfr_batch_storage_len", "dcfr_batch_download_storage", "dcfr_batch_autotune", "dcfr_batch_get_tuning",
    "dcfr_batch_set_tuning", "dcfr_batch_last_iterate_ms", "dcfr_batch_iterations", "dcfr_batch_kernel_launches",
    "dcfr_batch_iteration_bytes",
    "dcfr_mlp_create", "dcfr_mlp_destroy", "dcfr_mlp_num_params", "dcfr_mlp_get_params", "dcfr_mlp_set_params",
    "dcfr_mlp_forward", "dcfr_mlp_gradients", "dcfr_mlp_train_step",
    "dcfr_mlp_backward", "dcfr_mlp_gradients_device", "dcfr_mlp_adam_step", "dcfr_gemm_bf16", "dcfr_gemm_bf16_timed",
    "dcfr_create_depth_limited", "dcfr_node_storage", "dcfr_write_node",
    "dcfr_storage_slots", "dcfr_download_storage_compressed", "dcfr_upload_storage_compressed",
]


def lib():
    """Loads libdcfr.so (built in-tree by poker_trainer_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libdcfr.so is not built ({LIB_PATH}); run python -m poker_trainer_b200.build")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.dcfr_last_error.restype = C.c_char_p
        L.dcfr_config_init.argtypes = [C.POINTER(abi.Config)]
        L.dcfr_estimate.argtypes = [C.POINTER(abi.Config), C.POINTER(abi.TreeStats)]
        L.dcfr_create.argtypes = [C.POINTER(abi.Config), C.POINTER(P)]
        L.dcfr_destroy.argtypes = [P]
        L.dcfr_destroy.restype = None
        L.dcfr_solve.argtypes = [P, C.POINTER(abi.SolveOptions), P, abi.PROGRESS_CB, P, C.POINTER(abi.Progress)]
        L.dcfr_iterate.argtypes = [P, C.c_uint32]
        L.dcfr_synchronize.argtypes = [P]
        L.dcfr_exploitability.argtypes = [P, C.POINTER(C.c_double)]
        L.dcfr_exploitability_fp64.argtypes = [P, C.POINTER(C.c_double), P]
        L.dcfr_create_depth_limited.argtypes = [C.POINTER(abi.Config), P, C.POINTER(P)]
        L.dcfr_node_storage.argtypes = [P, P, C.c_size_t, C.POINTER(C.c_uint64), C.POINTER(C.c_int32),
                                        C.POINTER(C.c_int32)]
        L.dcfr_write_node.argtypes = [P, P, C.c_size_t, P, P]
        L.dcfr_batch_create.argtypes = [P, C.c_int32, C.POINTER(P)]
        L.dcfr_batch_destroy.argtypes = [P]
        L.dcfr_batch_destroy.restype = None
        L.dcfr_batch_iterate.argtypes = [P, C.c_uint32]
        L.dcfr_batch_exploitability.argtypes = [P, P]
        L.dcfr_batch_storage_len.argtypes = [P, C.c_int32, C.POINTER(C.c_uint64)]
        L.dcfr_batch_download_storage.argtypes = [P, C.c_int32, P, P, C.c_uint64]
        L.dcfr_batch_autotune.argtypes = [P, C.c_uint32, C.POINTER(abi.BatchTuning)]
        L.dcfr_batch_get_tuning.argtypes = [P, C.POINTER(abi.BatchTuning)]
        L.dcfr_batch_set_tuning.argtypes = [P, C.POINTER(abi.BatchTuning)]
        L.dcfr_batch_last_iterate_ms.argtypes = [P, C.POINTER(C.c_double)]
        L.dcfr_batch_iterations.argtypes = [P, C.POINTER(C.c_uint32)]
        L.dcfr_batch_kernel_launches.argtypes = [P, C.POINTER(C.c_uint64)]
        L.dcfr_batch_iteration_bytes.argtypes = [P, C.POINTER(C.c_double)]
        L.dcfr_root_values.argtypes = [P, P]
        L.dcfr_iterations.argtypes = [P, C.POINTER(C.c_uint32)]
        L.dcfr_last_exploitability.argtypes = [P, C.POINTER(C.c_double)]
        L.dcfr_stats.argtypes = [P, C.POINTER(abi.TreeStats)]
        L.dcfr_isomorphic_pairs.argtypes = [P, C.POINTER(C.c_int32)]
        L.dcfr_hands.argtypes = [P, C.c_int32, P, P, C.POINTER(C.c_int32)]
        L.dcfr_is_decision.argtypes = [P, P, C.c_size_t, C.POINTER(C.c_int32)]
        L.dcfr_actions_at.argtypes = [P, P, C.c_size_t, P, C.c_size_t, C.POINTER(C.c_size_t)]
        L.dcfr_query_sizes.argtypes = [P, P, C.c_size_t, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.dcfr_query.argtypes = [P, P, C.c_size_t, C.POINTER(abi.NodeInfoHeader), P, P, P, P, P]
        L.dcfr_ranges_after.argtypes = [P, P, C.c_size_t, P]
        L.dcfr_storage_len.argtypes = [P, C.POINTER(C.c_uint64)]
        L.dcfr_download_storage.argtypes = [P, P, P, C.c_uint64]
        L.dcfr_upload_storage.argtypes = [P, P, P, C.c_uint64]
        L.dcfr_storage_slots.argtypes = [P, C.POINTER(C.c_uint64)]
        L.dcfr_download_storage_compressed.argtypes = [P, P, P, P, P, C.c_uint64, C.c_uint64]
        L.dcfr_upload_storage_compressed.argtypes = [P, P, P, P, P, C.c_uint64, C.c_uint64]
        L.dcfr_set_iterations.argtypes = [P, C.c_uint32]
        L.dcfr_traverse.argtypes = [P, C.c_int32, C.c_int32, C.c_uint32, P]
        L.dcfr_kernel_launches.argtypes = [P, C.POINTER(C.c_uint64)]
        L.dcfr_terminal_kernel.argtypes = [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.dcfr_last_solve_ms.argtypes = [P, C.POINTER(C.c_double)]
        L.dcfr_setup_profile_get.argtypes = [P, C.POINTER(abi.SetupProfile)]
        L.dcfr_last_iterate_ms.argtypes = [P, C.POINTER(C.c_double)]
        L.dcfr_iteration_bytes.argtypes = [P, C.POINTER(C.c_double)]
        L.dcfr_iterate_profiled.argtypes = [P, C.c_uint32, C.POINTER(abi.KernelProfile)]
        _lib = L
    return _lib


# ------------------------------------------------------------------ errors
class SolverError(Exception):
    """SolverError (crates/solver/src/lib.rs:186-208)."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


class EmptyRange(SolverError):
    pass


class InvalidBoard(SolverError):
    pass


class TooLarge(SolverError):
    pass


class BadPath(SolverError):
    pass


class GpuError(SolverError):
    """A CUDA failure (no CPU fallback exists)."""


_ERRORS = {abi.ERR_EMPTY_RANGE: EmptyRange, abi.ERR_INVALID_BOARD: InvalidBoard, abi.ERR_TOO_LARGE: TooLarge,
           abi.ERR_BAD_PATH: BadPath, abi.ERR_CUDA: GpuError, abi.ERR_OUT_OF_MEMORY: GpuError,
           abi.ERR_DEVICE_TIMEOUT: GpuError}


def check(rc: int):
    if rc != abi.OK:
        msg = lib().dcfr_last_error().decode(errors="replace")
        raise _ERRORS.get(rc, SolverError)(rc, msg)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


# ------------------------------------------------------------------ types
@dataclass
class SolveOptions:
    """SolveOptions (lib.rs:137-153)."""
    max_iterations: int = 1000
    target_exploitability_pct: float = 0.5
    check_every: int = 10


@dataclass
class Progress:
    iteration: int
    max_iterations: int
    exploitability: float
    exploitability_pct: float
    finished: bool


@dataclass
class NodeInfo:
    """NodeInfo (lib.rs:220-275); strategy/ev are [actions, hands]."""
    player: int
    actions: list
    combos: np.ndarray
    strategy: np.ndarray
    ev: np.ndarray
    reach: np.ndarray
    reach_fraction: tuple
    pot: int
    invest: tuple

    def num_hands(self) -> int:
        return len(self.combos)

    def hand_index(self, combo: int):
        idx = np.nonzero(self.combos == combo)[0]
        return int(idx[0]) if len(idx) else None

    def hand_strategy(self, i: int) -> np.ndarray:
        return self.strategy[:, i]

    def hand_ev(self, i: int) -> np.ndarray:
        return self.ev[:, i]

    def range_strategy(self) -> list:
        total = float(np.sum(self.reach.astype(np.float64)))
        if total <= 0:
            return [0.0] * len(self.actions)
        r = self.reach.astype(np.float64)
        return [float(np.sum(r * self.strategy[a].astype(np.float64)) / total) for a in range(len(self.actions))]


@dataclass
class TreeStats:
    player_nodes: int
    chance_nodes: int
    terminal_nodes: int
    storage_cells: int
    compressed: bool
    memory_bytes: int

    def total_nodes(self) -> int:
        return self.player_nodes + self.chance_nodes + self.terminal_nodes


def _stats(st: abi.TreeStats) -> TreeStats:
    return TreeStats(st.player_nodes, st.chance_nodes, st.terminal_nodes, st.storage_cells, bool(st.compressed),
                     st.memory_bytes)


class Solver:
    """A built game on the GPU (Solver, crates/solver/src/lib.rs:288-913)."""

    def __init__(self, handle):
        self._h = handle

    @staticmethod
    def new(config: abi.Config) -> "Solver":
        h = C.c_void_p()
        check(lib().dcfr_create(C.byref(config), C.byref(h)))
        return Solver(h)

    @staticmethod
    def new_depth_limited(config: abi.Config, net) -> "Solver":
        """A flop solve cut at the turn deal, its leaves valued by `net`
        (poker_trainer_b200.mlp.LeafNet, kept alive by the solver)."""
        h = C.c_void_p()
        check(lib().dcfr_create_depth_limited(C.byref(config), net._h, C.byref(h)))
        s = Solver(h)
        s._net = net
        return s

    def node_storage(self, path=()):
        """(offset, actions, hands) of a decision node's block in the
        reference storage layout."""
        steps, n = abi.path_steps(path)
        off = C.c_uint64()
        na = C.c_int32()
        nh = C.c_int32()
        check(lib().dcfr_node_storage(self._h, steps, n, C.byref(off), C.byref(na), C.byref(nh)))
        return off.value, na.value, nh.value

    def write_node(self, path, regrets=None, sums=None):
        """Overwrites a decision node's blocks ([actions][hands] arrays)."""
        steps, n = abi.path_steps(path)
        r = None if regrets is None else np.ascontiguousarray(regrets, np.float32)
        sm = None if sums is None else np.ascontiguousarray(sums, np.float32)
        check(lib().dcfr_write_node(self._h, steps, n, _ptr(r) if r is not None else None,
                                    _ptr(sm) if sm is not None else None))

    @staticmethod
    def estimate(config: abi.Config) -> TreeStats:
        st = abi.TreeStats()
        check(lib().dcfr_estimate(C.byref(config), C.byref(st)))
        return _stats(st)

    def close(self):
        if getattr(self, "_h", None):
            lib().dcfr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # ------------------------------------------------------------ solve
    def solve(self, opts: SolveOptions | None = None, on_progress=None, cancel=None) -> Progress:
        """solve / solve_cancellable (lib.rs:475-494). `on_progress(progress)`
        returning False cancels; `cancel` is a ctypes c_int32 flag."""
        opts = opts or SolveOptions()
        o = abi.SolveOptions(opts.max_iterations, opts.check_every, opts.target_exploitability_pct)

        def cb(p, _u):
            if on_progress is None:
                return 1
            pp = p.contents
            r = on_progress(Progress(pp.iteration, pp.max_iterations, pp.exploitability, pp.exploitability_pct,
                                     bool(pp.finished)))
            return 0 if r is False else 1

        cbf = abi.PROGRESS_CB(cb)
        out = abi.Progress()
        flag = C.byref(cancel) if cancel is not None else None
        check(lib().dcfr_solve(self._h, C.byref(o), flag, cbf, None, C.byref(out)))
        return Progress(out.iteration, out.max_iterations, out.exploitability, out.exploitability_pct,
                        bool(out.finished))

    def iterate(self, n: int):
        check(lib().dcfr_iterate(self._h, n))

    def synchronize(self):
        check(lib().dcfr_synchronize(self._h))

    def exploitability(self) -> float:
        x = C.c_double()
        check(lib().dcfr_exploitability(self._h, C.byref(x)))
        return x.value

    def exploitability_fp64(self):
        """The FP64 best-response oracle: (exploitability, best-response
        root values of both players), all in chips."""
        x = C.c_double()
        br = np.zeros(2, np.float64)
        check(lib().dcfr_exploitability_fp64(self._h, C.byref(x), _ptr(br)))
        return x.value, br

    def root_values(self) -> np.ndarray:
        out = np.zeros(2, np.float64)
        check(lib().dcfr_root_values(self._h, _ptr(out)))
        return out

    def iterations(self) -> int:
        x = C.c_uint32()
        check(lib().dcfr_iterations(self._h, C.byref(x)))
        return x.value

    def last_exploitability(self) -> float:
        x = C.c_double()
        check(lib().dcfr_last_exploitability(self._h, C.byref(x)))
        return x.value

    def stats(self) -> TreeStats:
        st = abi.TreeStats()
        check(lib().dcfr_stats(self._h, C.byref(st)))
        return _stats(st)

    def isomorphic_pairs(self) -> int:
        x = C.c_int32()
        check(lib().dcfr_isomorphic_pairs(self._h, C.byref(x)))
        return x.value

    def num_hands(self, p: int) -> int:
        n = C.c_int32()
        check(lib().dcfr_hands(self._h, p, None, None, C.byref(n)))
        return n.value

    def hands(self, p: int):
        n = self.num_hands(p)
        combos = np.zeros(n, np.uint16)
        w = np.zeros(n, np.float32)
        nn = C.c_int32()
        check(lib().dcfr_hands(self._h, p, _ptr(combos), _ptr(w), C.byref(nn)))
        return combos, w

    # ------------------------------------------------------------ queries
    def is_decision(self, path=()) -> bool:
        steps, n = abi.path_steps(path)
        x = C.c_int32()
        check(lib().dcfr_is_decision(self._h, steps, n, C.byref(x)))
        return bool(x.value)

    def actions_at(self, path=()) -> list:
        steps, n = abi.path_steps(path)
        acts = (abi.ActionT * 32)()
        cnt = C.c_size_t()
        check(lib().dcfr_actions_at(self._h, steps, n, acts, 32, C.byref(cnt)))
        return [(acts[i].kind, acts[i].amount) for i in range(cnt.value)]

    def query(self, path=()) -> NodeInfo:
        steps, n = abi.path_steps(path)
        na, nh = C.c_int32(), C.c_int32()
        check(lib().dcfr_query_sizes(self._h, steps, n, C.byref(na), C.byref(nh)))
        info = abi.NodeInfoHeader()
        acts = (abi.ActionT * max(1, na.value))()
        combos = np.zeros(nh.value, np.uint16)
        strat = np.zeros(na.value * nh.value, np.float32)
        ev = np.zeros(na.value * nh.value, np.float32)
        reach = np.zeros(nh.value, np.float32)
        check(lib().dcfr_query(self._h, steps, n, C.byref(info), acts, _ptr(combos), _ptr(strat), _ptr(ev),
                               _ptr(reach)))
        return NodeInfo(info.player, [(acts[i].kind, acts[i].amount) for i in range(na.value)], combos,
                        strat.reshape(na.value, nh.value), ev.reshape(na.value, nh.value), reach,
                        (info.reach_fraction[0], info.reach_fraction[1]), info.pot, (info.invest[0], info.invest[1]))

    def ranges_after(self, path=()) -> np.ndarray:
        steps, n = abi.path_steps(path)
        out = np.zeros((2, abi.NUM_COMBOS), np.float32)
        check(lib().dcfr_ranges_after(self._h, steps, n, _ptr(out)))
        return out

    # ------------------------------------------------------------ storage
    def storage_len(self) -> int:
        x = C.c_uint64()
        check(lib().dcfr_storage_len(self._h, C.byref(x)))
        return x.value

    def download_storage(self, out=None):
        """Regrets and strategy sums (the reference's HostStorage). `out` may
        supply two contiguous float32 arrays of storage_len() (for instance
        views of pinned host memory)."""
        n = self.storage_len()
        if out is None:
            r = np.zeros(n, np.float32)
            s = np.zeros(n, np.float32)
        else:
            r, s = out
            if r.dtype != np.float32 or s.dtype != np.float32 or len(r) < n or len(s) < n:
                raise ValueError("out arrays must be float32 with storage_len() entries")
            if not (r.flags.c_contiguous and s.flags.c_contiguous):
                raise ValueError("out arrays must be contiguous")
        check(lib().dcfr_download_storage(self._h, _ptr(r), _ptr(s), n))
        return r, s

    def storage_slots(self) -> int:
        n = C.c_uint64()
        check(lib().dcfr_storage_slots(self._h, C.byref(n)))
        return n.value

    def download_storage_compressed(self):
        """Compressed storage (storage.rs:92-97): i16 regrets, u16 sums and
        the per-slot scales."""
        n, k = self.storage_len(), self.storage_slots()
        rq = np.zeros(n, np.int16)
        sq = np.zeros(n, np.uint16)
        rs = np.zeros(k, np.float32)
        ss = np.zeros(k, np.float32)
        check(lib().dcfr_download_storage_compressed(self._h, _ptr(rq), _ptr(sq), _ptr(rs), _ptr(ss), n, k))
        return rq, sq, rs, ss

    def upload_storage_compressed(self, rq, sq, rs, ss):
        rq = np.ascontiguousarray(rq, np.int16)
        sq = np.ascontiguousarray(sq, np.uint16)
        rs = np.ascontiguousarray(rs, np.float32)
        ss = np.ascontiguousarray(ss, np.float32)
        check(lib().dcfr_upload_storage_compressed(self._h, _ptr(rq), _ptr(sq), _ptr(rs), _ptr(ss), len(rq), len(rs)))

    def upload_storage(self, regrets, sums):
        r = np.ascontiguousarray(regrets, np.float32)
        s = np.ascontiguousarray(sums, np.float32)
        check(lib().dcfr_upload_storage(self._h, _ptr(r), _ptr(s), len(r)))

    def set_iterations(self, t: int):
        check(lib().dcfr_set_iterations(self._h, t))

    def traverse(self, p: int, mode: int, t: int) -> np.ndarray:
        out = np.zeros(self.num_hands(p), np.float32)
        check(lib().dcfr_traverse(self._h, p, mode, t, _ptr(out)))
        return out

    def last_solve_ms(self) -> float:
        """Device time of the last solve() (CUDA events on the handle's
        stream around it), milliseconds."""
        x = C.c_double()
        check(lib().dcfr_last_solve_ms(self._h, C.byref(x)))
        return x.value

    def setup_profile(self) -> dict:
        """Host milliseconds of each setup phase (dcfr_setup_profile)."""
        sp = abi.SetupProfile()
        check(lib().dcfr_setup_profile_get(self._h, C.byref(sp)))
        return {f[0]: getattr(sp, f[0]) for f in abi.SetupProfile._fields_}

    def terminal_kernel(self) -> tuple:
        """(kernel name, terminals per panel) of this handle's f32 terminal
        evaluation: "panel", "warp", "block", "group" (two warps per
        terminal) or "exact"."""
        k = C.c_int32()
        t = C.c_int32()
        check(lib().dcfr_terminal_kernel(self._h, C.byref(k), C.byref(t)))
        return ("panel", "warp", "block", "exact", "group")[k.value], t.value

    def kernel_launches(self) -> int:
        x = C.c_uint64()
        check(lib().dcfr_kernel_launches(self._h, C.byref(x)))
        return x.value

    def last_iterate_ms(self) -> float:
        x = C.c_double()
        check(lib().dcfr_last_iterate_ms(self._h, C.byref(x)))
        return x.value

    def iteration_bytes(self) -> float:
        x = C.c_double()
        check(lib().dcfr_iteration_bytes(self._h, C.byref(x)))
        return x.value

    def iterate_profiled(self, n: int) -> dict:
        """Runs n iterations with CUDA events at every kernel-class boundary;
        returns per class (down, terminal, up, other) launches, device ms and
        compulsory bytes, plus the first-to-last-event total."""
        prof = abi.KernelProfile()
        check(lib().dcfr_iterate_profiled(self._h, n, C.byref(prof)))
        classes = {}
        for c, name in enumerate(abi.KERNEL_CLASSES):
            classes[name] = dict(launches=int(prof.launches[c]), ms=float(prof.ms[c]), bytes=float(prof.bytes[c]))
        return dict(iterations=int(prof.iterations), total_ms=float(prof.total_ms), classes=classes)


class BatchSolver:
    """Batched river solves (dcfr_batch_*): many independent river spots
    solved together by a persistent kernel under a captured CUDA graph."""

    def __init__(self, handle, count):
        self._h = handle
        self.count = count

    @staticmethod
    def new(configs) -> "BatchSolver":
        arr = (abi.Config * len(configs))(*configs)
        h = C.c_void_p()
        check(lib().dcfr_batch_create(arr, len(configs), C.byref(h)))
        return BatchSolver(h, len(configs))

    def close(self):
        if getattr(self, "_h", None):
            lib().dcfr_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def iterate(self, n: int):
        check(lib().dcfr_batch_iterate(self._h, n))

    def exploitability(self) -> np.ndarray:
        out = np.zeros(self.count, np.float64)
        check(lib().dcfr_batch_exploitability(self._h, _ptr(out)))
        return out

    def storage_len(self, spot: int) -> int:
        n = C.c_uint64()
        check(lib().dcfr_batch_storage_len(self._h, spot, C.byref(n)))
        return n.value

    def download_storage(self, spot: int):
        n = self.storage_len(spot)
        r = np.zeros(n, np.float32)
        s = np.zeros(n, np.float32)
        check(lib().dcfr_batch_download_storage(self._h, spot, _ptr(r), _ptr(s), n))
        return r, s

    def autotune(self, trial_iterations: int = 10) -> abi.BatchTuning:
        t = abi.BatchTuning()
        check(lib().dcfr_batch_autotune(self._h, trial_iterations, C.byref(t)))
        return t

    def tuning(self) -> abi.BatchTuning:
        t = abi.BatchTuning()
        check(lib().dcfr_batch_get_tuning(self._h, C.byref(t)))
        return t

    def set_tuning(self, t: abi.BatchTuning):
        check(lib().dcfr_batch_set_tuning(self._h, C.byref(t)))

    def last_iterate_ms(self) -> float:
        x = C.c_double()
        check(lib().dcfr_batch_last_iterate_ms(self._h, C.byref(x)))
        return x.value

    def iterations(self) -> int:
        x = C.c_uint32()
        check(lib().dcfr_batch_iterations(self._h, C.byref(x)))
        return x.value

    def kernel_launches(self) -> int:
        x = C.c_uint64()
        check(lib().dcfr_batch_kernel_launches(self._h, C.byref(x)))
        return x.value

    def iteration_bytes(self) -> float:
        x = C.c_double()
        check(lib().dcfr_batch_iteration_bytes(self._h, C.byref(x)))
        return x.value
