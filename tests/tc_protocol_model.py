"""Test infrastructure: a discrete-event model of the tensor-core kernel's
hand-off protocol (simu_rca_ab_b200/csrc/fused_tc_kernel.cuh), run on the CPU.

The kernel's roles -- the producer (records into a ring, in rounds), the
loader (window loads into a ring of stages), three builder groups (weights
into a ring of slots; the epilogue of an item's end record) and the MMA
issuer (MMAs and commits) -- are modelled as coroutines that wait on
mbarriers with the hardware's parity test and arrive on them exactly where
the kernel does.  Asynchronous completions (a TMA landing, the MMAs behind a
tcgen05.commit, which complete in issue order) fire at random later times,
and the scheduler interleaves every runnable role at random.

An mbarrier's parity tells only its current phase from the previous one,
so every wait must start when the barrier has completed the phase before the
awaited one and must end before the barrier completes the phase after it.
The model checks both on every wait (a wait that started too early would
return at once on the wrong phase; one that fell two phases behind would
wait for ever), and that every record reaches the MMAs and every item's
epilogue in order.  ``acc_seen_wait=False`` removes the epilogue's wait for
the previous item's accumulator phase, the kernel's guard for items of
fewer than two records.
"""
from __future__ import annotations

import random
from dataclasses import dataclass, field

# the kernel's constants (TC_GROUPS, TC_NSA, TC_NSB, TC_NSR, TC_NPUB)
GROUPS, NSA, NSB = 3, 3, 6
NSR = 2 * NSB
NPUB = NSR // 2
STEP, END, FINAL = 0, 1, 2


class ProtocolError(AssertionError):
    pass


@dataclass
class Bar:
    name: str
    count: int = 1
    pending: int = 0
    phase: int = 0          # completed phases (the current phase's index)

    def arrive(self):
        self.pending += 1
        if self.pending == self.count:
            self.pending = 0
            self.phase += 1

    def passes(self, target: int) -> bool:
        """mbarrier try_wait.parity for the completion of phase `target`."""
        return (self.phase & 1) != (target & 1)


@dataclass
class Wait:
    bar: Bar
    target: int             # the phase whose completion is awaited
    who: str


@dataclass
class Spin:
    pred: object
    who: str


@dataclass
class Model:
    items: list             # records per item (>= 0)
    seed: int = 0
    acc_seen_wait: bool = True
    groups: int = GROUPS    # ring sizes, the kernel's by default
    nsa: int = NSA
    nsb: int = NSB
    nsr: int = NSR
    npub: int = NPUB
    rng: random.Random = field(init=False)

    def __post_init__(self):
        self.rng = random.Random(self.seed)
        B = lambda n, c=1: Bar(n, c)
        self.rec_full = [B(f"rec_full{i}") for i in range(self.nsr)]
        self.rec_empty = [B(f"rec_empty{i}") for i in range(self.nsr)]
        self.full_b = [B(f"full_b{i}") for i in range(self.nsb)]
        self.empty_b = [B(f"empty_b{i}") for i in range(self.nsb)]
        self.full_a = [B(f"full_a{i}") for i in range(self.nsa)]
        self.acc_full, self.acc_empty = B("acc_full"), B("acc_empty")
        self.info = [None] * self.nsr
        self.acc_seen = -1
        self.events = []            # (time, seq, fn)
        self.commit_tail = 0.0      # commits complete in issue order
        self.now = 0.0
        self.seq = 0
        self.mma_log, self.epi_log = [], []
        # the record sequence the producer will publish
        recs = []
        for it, n in enumerate(self.items):
            recs += [(STEP, it)] * n + [(END, it)]
        self.records = recs + [(FINAL, len(self.items))] * self.groups

    # -- asynchronous completions -------------------------------------------
    def later(self, delay, fn):
        self.seq += 1
        self.events.append((self.now + delay, self.seq, fn))

    def commit(self, bar):
        """tcgen05.commit: arrives once every earlier MMA has completed."""
        t = max(self.commit_tail, self.now + self.rng.uniform(0.5, 3.0))
        self.commit_tail = t
        self.seq += 1
        self.events.append((t, self.seq, bar.arrive))

    # -- roles ----------------------------------------------------------------
    def emit(self, q, rec):
        rs = q % self.nsr
        yield Wait(self.rec_empty[rs], q // self.nsr - 1, f"producer emit {q}")
        self.info[rs] = rec
        self.rec_full[rs].arrive()

    def producer(self):
        q = 0
        n_items = len(self.items)
        for it in range(n_items + 1):
            if it < n_items:
                recs = [(STEP, it)] * self.items[it] + [(END, it)]
            else:
                recs = [(FINAL, it)] * self.groups
            # rounds of at most self.npub records, emitted by parallel lanes
            for r0 in range(0, len(recs), self.npub):
                lanes = [self.emit(q + r, recs[r]) for r in range(r0, min(r0 + self.npub, len(recs)))]
                yield from self.join(lanes, "producer round")
            q += len(recs)

    def join(self, gens, who):
        """The lanes of one producer round: each lane waits for its own slot;
        the round ends when every lane has written its record (lanes taken
        in a random order)."""
        order = list(gens)
        self.rng.shuffle(order)
        for g in order:
            yield from g

    def loader(self):
        q = 0
        while True:
            rs, st = q % self.nsr, q % self.nsb
            yield Wait(self.rec_full[rs], q // self.nsr, f"loader rec {q}")
            kind, it = self.info[rs]
            if kind == FINAL:
                return
            yield Wait(self.empty_b[st], q // self.nsb - 1, f"loader stage {q}")
            if kind == STEP:
                self.later(self.rng.uniform(0.2, 4.0), self.full_b[st].arrive)
            else:
                self.full_b[st].arrive()
            q += 1

    def builder(self, g):
        q = g
        while True:
            rs = q % self.nsr
            yield Wait(self.rec_full[rs], q // self.nsr, f"builder{g} rec {q}")
            kind, it = self.info[rs]
            if kind == FINAL:
                return
            ast = q % self.nsa
            if q >= self.nsa:                              # the slot's previous use has been consumed
                qp = q - self.nsa
                yield Wait(self.empty_b[qp % self.nsb], qp // self.nsb, f"builder{g} slot {q}")
            self.full_a[ast].arrive()
            if kind == END:
                if self.acc_seen_wait and it > 0:
                    yield Spin(lambda it=it: self.acc_seen >= it - 1, f"builder{g} seen {it}")
                yield Wait(self.acc_full, it, f"builder{g} acc_full item {it}")
                self.acc_seen = max(self.acc_seen, it)
                self.epi_log.append(it)
                self.acc_empty.arrive()
            q += self.groups

    def mma(self):
        q, first = 0, True
        while True:
            rs, bst, ast = q % self.nsr, q % self.nsb, q % self.nsa
            yield Wait(self.rec_full[rs], q // self.nsr, f"mma rec {q}")
            kind, it = self.info[rs]
            if kind == FINAL:
                return
            yield Wait(self.full_b[bst], q // self.nsb, f"mma stage {q}")
            yield Wait(self.full_a[ast], q // self.nsa, f"mma slot {q}")
            if first:
                yield Wait(self.acc_empty, it - 1, f"mma acc_empty item {it}")
                first = False
            self.mma_log.append((kind, it))
            if kind == END:
                self.commit(self.acc_full)
                self.commit(self.empty_b[bst])
                first = True
            else:
                self.commit(self.empty_b[bst])
            self.rec_empty[rs].arrive()
            q += 1

    # -- scheduler --------------------------------------------------------------
    def run(self, max_steps: int = 2_000_000):
        roles = {"producer": self.producer(), "loader": self.loader(), "mma": self.mma()}
        for g in range(self.groups):
            roles[f"builder{g}"] = self.builder(g)
        blocked = {}
        for name, gen in roles.items():
            blocked[name] = self._start(name, gen)
        for _ in range(max_steps):
            self._check(blocked)
            runnable = [n for n, w in blocked.items() if w is not False and self._ready(w)]
            if not runnable and not self.events:
                if all(w is False for w in blocked.values()):
                    return
                raise ProtocolError(f"deadlock: {[(n, w.who) for n, w in blocked.items() if w]}")
            if self.events and (not runnable or self.rng.random() < 0.3):
                self.events.sort()
                t, _, fn = self.events.pop(0)
                self.now = max(self.now, t)
                fn()
                continue
            name = self.rng.choice(runnable)
            self.now += 0.01
            blocked[name] = self._resume(name, roles[name])
        raise ProtocolError("no progress")

    def _start(self, name, gen):
        try:
            w = next(gen)
        except StopIteration:
            return False
        self._entry_check(w)
        return w

    def _resume(self, name, gen):
        try:
            w = gen.send(None)
        except StopIteration:
            return False
        self._entry_check(w)
        return w

    @staticmethod
    def _ready(w):
        if isinstance(w, Wait):
            return w.bar.passes(w.target)
        return bool(w.pred())

    @staticmethod
    def _entry_check(w):
        # a wait starts only once the phase before the awaited one completed
        if isinstance(w, Wait) and w.bar.phase < w.target:
            raise ProtocolError(f"{w.who}: waits for phase {w.target} of {w.bar.name} at phase {w.bar.phase}")

    @staticmethod
    def _check(blocked):
        # ...and ends before the barrier completes the phase after it
        for w in blocked.values():
            if isinstance(w, Wait) and w.bar.phase > w.target + 1:
                raise ProtocolError(f"{w.who}: {w.bar.name} passed phase {w.target + 1} before the wait ended")
