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
