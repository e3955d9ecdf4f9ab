"""ctypes mirror of include/dcfr.h and builders for its config structs.

The structs follow the reference solver crate's public types
(AhanDatta/Poker-Trainer, crates/solver/src/lib.rs:74-240,
crates/solver/src/tree.rs:19-34, crates/holdem/src/menu.rs:16-133); the
helpers here build them from the same notation the reference uses
("75%", "3x", "allin", board strings such as "Ks7s2dTh4c").
"""
from __future__ import annotations

import ctypes as C

NUM_COMBOS = 1326
MAX_SIZES = 8

# Status codes (include/dcfr.h).
OK = 0
ERR_EMPTY_RANGE = 1
ERR_INVALID_BOARD = 2
ERR_TOO_LARGE = 3
ERR_BAD_PATH = 4
ERR_INVALID_ARG = 5
ERR_CUDA = 6
ERR_OUT_OF_MEMORY = 7
ERR_UNSUPPORTED = 8
ERR_DEVICE_TIMEOUT = 9

PREFLOP, FLOP, TURN, RIVER = 0, 1, 2, 3
SIZE_POT, SIZE_MULT, SIZE_ALLIN = 0, 1, 2
FOLD, CHECK, CALL, RAISE = 0, 1, 2, 3
STORAGE_F32, STORAGE_COMPRESSED, STORAGE_AUTO = 0, 1, 2
PRECISION_FAST, PRECISION_EXACT = 0, 1  # GpuPrecision (crates/solver/src/gpu/mod.rs:51-63)
PRECISIONS = {"fast": PRECISION_FAST, "exact": PRECISION_EXACT}
CHANCE_EXACT, CHANCE_SAMPLED = 0, 1  # ChanceMode (crates/solver/src/tree.rs:128-136)
MODE_CFR, MODE_BEST_RESPONSE, MODE_AVERAGE = 0, 1, 2


class BetSize(C.Structure):
    _fields_ = [("kind", C.c_int32), ("_pad", C.c_int32), ("value", C.c_double)]


class StreetSizes(C.Structure):
    _fields_ = [
        ("n_bet", C.c_int32),
        ("n_raise", C.c_int32),
        ("bet", BetSize * MAX_SIZES),
        ("raise_", BetSize * MAX_SIZES),
    ]


class Menu(C.Structure):
    _fields_ = [
        ("flop", StreetSizes),
        ("turn", StreetSizes),
        ("river", StreetSizes),
        ("max_raises", C.c_uint32),
        ("_pad", C.c_uint32),
        ("add_allin_threshold", C.c_double),
        ("force_allin_threshold", C.c_double),
        ("merge_threshold", C.c_double),
    ]


class BettingState(C.Structure):
    _fields_ = [
        ("street", C.c_int32),
        ("to_act", C.c_int32),
        ("pot", C.c_int64),
        ("commit", C.c_int64 * 2),
        ("stack", C.c_int64 * 2),
        ("current_bet", C.c_int64),
        ("last_raise_inc", C.c_int64),
        ("num_raises", C.c_uint32),
        ("needs", C.c_uint8 * 2),
        ("_pad", C.c_uint8 * 2),
    ]


class Params(C.Structure):
    _fields_ = [
        ("alpha", C.c_double),
        ("beta", C.c_double),
        ("gamma", C.c_double),
        ("beta_clip", C.c_int32),
        ("restart_average", C.c_int32),
        ("unweighted_average", C.c_int32),
        ("_pad", C.c_int32),
    ]


class Config(C.Structure):
    _fields_ = [
        ("board", C.c_uint8 * 5),
        ("_pad0", C.c_uint8 * 3),
        ("board_len", C.c_int32),
        ("_pad1", C.c_int32),
        ("ranges", (C.c_float * NUM_COMBOS) * 2),
        ("root", BettingState),
        ("menu", Menu),
        ("has_future_menu", C.c_int32),
        ("_pad2", C.c_int32),
        ("future_menu", Menu),
        ("big_blind", C.c_int64),
        ("prune", C.c_float),
        ("n_keep", C.c_int32 * 2),
        ("_pad3", C.c_int32),
        ("keep", (C.c_uint16 * NUM_COMBOS) * 2),
        ("max_memory_bytes", C.c_uint64),
        ("rake_rate", C.c_double),
        ("rake_cap", C.c_double),
        ("storage", C.c_int32),
        ("isomorphism", C.c_int32),
        ("dcfr", Params),
        ("precision", C.c_int32),
        ("chance", C.c_int32),
        ("chance_turn", C.c_int32),
        ("chance_river", C.c_int32),
        ("chance_seed", C.c_uint64),
    ]


KERNEL_CLASSES = ("down", "terminal", "up", "other")  # DCFR_KERNEL_* order


class KernelProfile(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint32),
        ("_pad", C.c_uint32),
        ("launches", C.c_uint64 * 4),
        ("ms", C.c_double * 4),
        ("bytes", C.c_double * 4),
        ("total_ms", C.c_double),
    ]


class SetupProfile(C.Structure):
    """dcfr_setup_profile (include/dcfr.h): host milliseconds per setup phase."""
    _fields_ = [(n, C.c_double) for n in ("game_ms", "device_ms", "tables_ms", "plans_ms", "rows_ms", "create_ms",
                                          "iteration_graph_ms", "eval_graphs_ms")]


class BatchTuning(C.Structure):
    """dcfr_batch_tuning (include/dcfr.h)."""
    _fields_ = [
        ("warps", C.c_int32),
        ("blocks_per_sm", C.c_int32),
        ("iterations_per_launch", C.c_uint32),
        ("longest_first", C.c_int32),
        ("candidates", C.c_int32),
        ("_pad", C.c_int32),
        ("trial_ms", C.c_double),
    ]


class TreeStats(C.Structure):
    _fields_ = [
        ("player_nodes", C.c_uint64),
        ("chance_nodes", C.c_uint64),
        ("terminal_nodes", C.c_uint64),
        ("storage_cells", C.c_uint64),
        ("compressed", C.c_int32),
        ("_pad", C.c_int32),
        ("memory_bytes", C.c_uint64),
    ]


class SolveOptions(C.Structure):
    _fields_ = [
        ("max_iterations", C.c_uint32),
        ("check_every", C.c_uint32),
        ("target_exploitability_pct", C.c_double),
    ]


class Progress(C.Structure):
    _fields_ = [
        ("iteration", C.c_uint32),
        ("max_iterations", C.c_uint32),
        ("exploitability", C.c_double),
        ("exploitability_pct", C.c_double),
        ("finished", C.c_int32),
        ("_pad", C.c_int32),
    ]


PROGRESS_CB = C.CFUNCTYPE(C.c_int, C.POINTER(Progress), C.c_void_p)


class Step(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("action_kind", C.c_int32),
        ("amount", C.c_int64),
        ("card", C.c_uint8),
        ("_pad", C.c_uint8 * 7),
    ]


class ActionT(C.Structure):
    _fields_ = [("kind", C.c_int32), ("_pad", C.c_int32), ("amount", C.c_int64)]


class NodeInfoHeader(C.Structure):
    _fields_ = [
        ("player", C.c_int32),
        ("num_actions", C.c_int32),
        ("num_hands", C.c_int32),
        ("_pad", C.c_int32),
        ("reach_fraction", C.c_double * 2),
        ("pot", C.c_int64),
        ("invest", C.c_int64 * 2),
    ]


# --------------------------------------------------------------- notation
RANKS = "23456789TJQKA"
SUITS = "cdhs"


def parse_card(s: str) -> int:
    """Card id rank*4+suit (crates/holdem/src/card.rs:46-48, 108-121)."""
    s = s.strip()
    if len(s) != 2 or s[0].upper() not in RANKS or s[1].lower() not in SUITS:
        raise ValueError(f"invalid card: {s!r}")
    return RANKS.index(s[0].upper()) * 4 + SUITS.index(s[1].lower())


def parse_cards(s: str) -> list[int]:
    """Card list such as "AhKd7c" (crates/holdem/src/card.rs:124-132)."""
    compact = "".join(ch for ch in s if not ch.isspace() and ch != ",")
    if len(compact) % 2:
        raise ValueError(f"invalid card list: {s!r}")
    return [parse_card(compact[i:i + 2]) for i in range(0, len(compact), 2)]


def card_str(c: int) -> str:
    return RANKS[c >> 2] + SUITS[c & 3]


def combo_index(a: int, b: int) -> int:
    """crates/holdem/src/combo.rs:14-17."""
    lo, hi = (a, b) if a < b else (b, a)
    return hi * (hi - 1) // 2 + lo


def combo_cards(i: int) -> tuple[int, int]:
    """COMBOS entry (higher card id, lower card id) (combo.rs:19-35)."""
    hi = 1
    while (hi + 1) * hi // 2 <= i:
        hi += 1
    return hi, i - hi * (hi - 1) // 2


def parse_size(s: str) -> tuple[int, float]:
    """BetSize::from_str (crates/holdem/src/menu.rs:26-50)."""
    t = s.strip().lower()
    if t in ("a", "allin", "all-in", "all in", "shove"):
        return SIZE_ALLIN, 0.0
    if t.endswith("%"):
        v = float(t[:-1])
        if v <= 0:
            raise ValueError(s)
        return SIZE_POT, v / 100.0
    if t.endswith("x"):
        v = float(t[:-1])
        if v <= 1:
            raise ValueError(s)
        return SIZE_MULT, v
    raise ValueError(f"invalid bet size {s!r}")


def street_sizes(bet, raise_) -> StreetSizes:
    ss = StreetSizes()
    bet, raise_ = list(bet), list(raise_)
    if len(bet) > MAX_SIZES or len(raise_) > MAX_SIZES:
        raise ValueError("too many sizes")
    ss.n_bet, ss.n_raise = len(bet), len(raise_)
    for i, b in enumerate(bet):
        ss.bet[i].kind, ss.bet[i].value = parse_size(b)
    for i, r in enumerate(raise_):
        ss.raise_[i].kind, ss.raise_[i].value = parse_size(r)
    return ss


def menu(bet=("50%", "100%"), raise_=("3x",), *, flop=None, turn=None, river=None, max_raises=3,
         add_allin=0.0, force_allin=0.0, merge=0.0) -> Menu:
    """A PostflopMenu. With only `bet`/`raise_` every street gets the same
    sizes and the three thresholds default to 0, as the reference's test
    helper `menu_one` does (crates/solver/src/tests.rs:6-17)."""
    m = Menu()
    m.flop = street_sizes(*(flop or (bet, raise_)))
    m.turn = street_sizes(*(turn or (bet, raise_)))
    m.river = street_sizes(*(river or (bet, raise_)))
    m.max_raises = max_raises
    m.add_allin_threshold = add_allin
    m.force_allin_threshold = force_allin
    m.merge_threshold = merge
    return m


def default_menu() -> Menu:
    """PostflopMenu::default (crates/holdem/src/menu.rs:119-133)."""
    return menu(flop=(("33%", "75%"), ("3x",)), turn=(("50%", "100%"), ("3x",)),
                river=(("50%", "100%"), ("3x",)), max_raises=3, add_allin=1.5, force_allin=0.15, merge=0.1)


def street_start(street: int, pot: int, stack0: int, stack1: int | None = None, big_blind: int = 100) -> BettingState:
    """BettingState::street_start (crates/solver/src/tree.rs:49-61)."""
    if stack1 is None:
        stack1 = stack0
    b = BettingState()
    b.street, b.pot = street, pot
    b.commit[0] = b.commit[1] = 0
    b.stack[0], b.stack[1] = stack0, stack1
    b.current_bet, b.last_raise_inc, b.num_raises, b.to_act = 0, big_blind, 0, 0
    b.needs[0], b.needs[1] = int(stack0 > 0), int(stack1 > 0)
    return b


def betting_state(street, pot, commit, stack, current_bet, last_raise_inc, num_raises, to_act, needs) -> BettingState:
    b = BettingState()
    b.street, b.pot = street, pot
    b.commit[0], b.commit[1] = commit
    b.stack[0], b.stack[1] = stack
    b.current_bet, b.last_raise_inc, b.num_raises, b.to_act = current_bet, last_raise_inc, num_raises, to_act
    b.needs[0], b.needs[1] = int(needs[0]), int(needs[1])
    return b


def street_of_board(n: int) -> int:
    return {0: PREFLOP, 3: FLOP, 4: TURN}.get(n, RIVER)


def make_config(board, ranges, *, root=None, pot=None, stack=None, menu_: Menu | None = None,
                future_menu: Menu | None = None, big_blind=100, prune=0.0, keep=((), ()),
                max_memory_bytes=8 << 30, rake_rate=0.0, rake_cap=0.0, storage=STORAGE_AUTO,
                isomorphism=True, alpha=1.5, beta=0.0, beta_clip=False, gamma=3.0,
                restart_average=True, unweighted_average=True, precision="fast",
                sampled: tuple[int, int, int] | None = None) -> Config:
    """SolveConfig (crates/solver/src/lib.rs:74-135), defaults as
    SolveConfig::new and DcfrParams::default (cfr.rs:72-80). `sampled` =
    (turn, river, seed) selects ChanceMode::Sampled."""
    cfg = Config()
    cards = parse_cards(board) if isinstance(board, str) else list(board)
    if len(cards) > 5:
        raise ValueError("board has more than 5 cards")
    for i, c in enumerate(cards):
        cfg.board[i] = c
    cfg.board_len = len(cards)
    for p in range(2):
        r = ranges[p]
        if len(r) != NUM_COMBOS:
            raise ValueError("a range has 1326 weights")
        C.memmove(cfg.ranges[p], (C.c_float * NUM_COMBOS)(*[float(x) for x in r]), 4 * NUM_COMBOS)
    if root is None:
        root = street_start(street_of_board(len(cards)), pot, stack, stack, big_blind)
    cfg.root = root
    cfg.menu = menu_ if menu_ is not None else default_menu()
    if future_menu is not None:
        cfg.has_future_menu = 1
        cfg.future_menu = future_menu
    cfg.big_blind = big_blind
    cfg.prune = prune
    for p in range(2):
        cfg.n_keep[p] = len(keep[p])
        for i, c in enumerate(keep[p]):
            cfg.keep[p][i] = c
    cfg.max_memory_bytes = max_memory_bytes
    cfg.rake_rate, cfg.rake_cap = rake_rate, rake_cap
    cfg.storage = storage
    cfg.isomorphism = int(isomorphism)
    cfg.dcfr.alpha, cfg.dcfr.beta, cfg.dcfr.gamma = alpha, beta, gamma
    cfg.dcfr.beta_clip = int(beta_clip)
    cfg.dcfr.restart_average, cfg.dcfr.unweighted_average = int(restart_average), int(unweighted_average)
    cfg.precision = PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    if sampled is not None:
        cfg.chance = CHANCE_SAMPLED
        cfg.chance_turn, cfg.chance_river, cfg.chance_seed = sampled
    return cfg


def action(kind: int, amount: int = 0) -> tuple[int, int]:
    return (kind, amount)


def path_steps(path) -> tuple[C.Array, int]:
    """Steps from ("check"|"call"|"fold"|("raise", to)|card string or
    (kind, amount) tuples) (Step, crates/solver/src/lib.rs:212-217)."""
    steps = (Step * max(1, len(path)))()
    for i, s in enumerate(path):
        st = steps[i]
        if isinstance(s, str) and s.lower() in ("fold", "check", "call"):
            st.kind, st.action_kind = 0, {"fold": FOLD, "check": CHECK, "call": CALL}[s.lower()]
        elif isinstance(s, str):
            st.kind, st.card = 1, parse_card(s)
        elif isinstance(s, tuple) and isinstance(s[0], str):
            st.kind, st.action_kind, st.amount = 0, RAISE, int(s[1])
        else:
            st.kind, st.action_kind, st.amount = 0, int(s[0]), int(s[1])
    return steps, len(path)
