"""Arithmetic of the persistent kernel's grid barrier (GridExec::barrier_timed
in gcdt_b200/csrc/exec.cuh), checked on the host.

Each block adds to one 32-bit counter once per barrier: block 0 adds
2^31 - (blocks - 1), every other block 1.  A block waits until the counter's
top bit differs from the top bit of the value its own add returned, and the
block whose add itself flips the top bit is the last arrival.  The counter
starts at 0 and is never reset.  Here the arrivals come in random orders over
many barriers, with 32-bit wrap-around, and the test checks that the top bit
flips exactly once per barrier, at its last arrival, and that no block would
stop waiting before every block has arrived."""
import random

import pytest

M32 = (1 << 32) - 1
TOP = 1 << 31


def _add(blocks, b):
    return (TOP - (blocks - 1)) & M32 if b == 0 else 1


@pytest.mark.parametrize("blocks", [1, 2, 3, 148, 296, 1024])
def test_top_bit_flips_once_per_barrier_at_the_last_arrival(blocks):
    rng = random.Random(blocks)
    count = 0
    for _ in range(64):
        start_top = count & TOP
        order = list(range(blocks))
        rng.shuffle(order)
        olds = {}
        for k, b in enumerate(order):
            old = count
            add = _add(blocks, b)
            count = (count + add) & M32
            olds[b] = old
            last = (((old + add) & M32) ^ old) & TOP != 0
            assert last == (k == blocks - 1)
            if k < blocks - 1:
                # nobody released yet: every arrived block still sees its own top bit
                assert count & TOP == start_top
                for o in olds.values():
                    assert (o ^ count) & TOP == 0
        # all arrived: every block sees the flip, and the low bits are back at 0
        assert count & TOP != start_top
        assert count & (TOP - 1) == 0
        for o in olds.values():
            assert (o ^ count) & TOP != 0
