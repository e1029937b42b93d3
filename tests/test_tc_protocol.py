"""The tensor-core kernel's hand-off protocol (producer, loader, builder
groups, MMA issuer over rings of mbarriers; fused_tc_kernel.cuh) in a
discrete-event model on the CPU (tests/tc_protocol_model.py): random
interleavings and completion times never let a wait start before the phase
ahead of the awaited one completed, nor let a barrier run two phases past a
waiter; every record reaches the MMAs and every epilogue runs, in order.
Items of zero and one record are included; without the epilogue's wait for
the previous item's accumulator phase the model finds the early wait the
kernel guards against."""
import random

import pytest

from tests.tc_protocol_model import Model, ProtocolError, END, STEP


def _items(rng, n, short):
    """Records per item: long items (as the C2 ensemble's), with short ones
    (0, 1, 2 records) mixed in when `short`."""
    return [rng.choice([0, 1, 2]) if short and rng.random() < 0.5 else rng.randint(3, 30) for _ in range(n)]


@pytest.mark.parametrize("seed", range(12))
@pytest.mark.parametrize("short", [False, True])
def test_protocol_keeps_every_wait_within_one_phase(seed, short):
    rng = random.Random(seed)
    items = _items(rng, 40, short)
    m = Model(items, seed=seed)
    m.run()
    expect = []
    for it, n in enumerate(items):
        expect += [(STEP, it)] * n + [(END, it)]
    assert m.mma_log == expect
    assert m.epi_log == list(range(len(items)))


def test_items_of_zero_records_back_to_back():
    m = Model([5] + [0] * 12 + [7, 0, 1, 0, 2, 0], seed=3)
    m.run()
    assert m.epi_log == list(range(19))


def test_the_epilogue_guard_is_needed():
    """Without the wait for the previous item's accumulator phase, some
    schedule with runs of empty items lets an epilogue wait on the
    accumulator barrier before the phase ahead of its own has completed."""
    found = False
    for seed in range(200):
        m = Model([0] * 30, seed=seed, acc_seen_wait=False)
        try:
            m.run()
        except ProtocolError:
            found = True
            break
    assert found


def _finds_violation(**rings):
    rng = random.Random(5)
    for seed in range(60):
        items = _items(rng, 30, True)
        try:
            Model(items, seed=seed, **rings).run()
        except ProtocolError:
            return True
    return False


@pytest.mark.parametrize("rings,why", [
    (dict(nsa=6, nsb=3, nsr=6, npub=3), "more weight slots than window stages: a slot's previous use is "
                                        "signalled on a stage that has moved on"),
    (dict(nsr=6, npub=12), "producer rounds longer than the record ring: a lane waits on a slot whose "
                           "previous record is not written yet"),
])
def test_ring_sizes_the_kernel_asserts_are_needed(rings, why):
    """The kernel's static_asserts keep at least as many window stages as
    weight slots and producer rounds no longer than the record ring (it uses
    6 stages, 3 slots and rounds of half the ring): break either and the
    model finds a wait outside its phase or a deadlock."""
    assert _finds_violation(**rings), why
