"""The node stacks of the bulge tracebacks have no bounds checks: they rely
on the pop width and the refill rule keeping them inside their capacity.
This CPU test restates that policy (traceback_slots_kernel and
traceback_warp_kernel in csrc/bulge.cu, constants read from the source) and
runs it on adversarial trees -- every node with three children (diagonal,
RNA and DNA step) down to the deepest level a window allows -- asserting
that no step ever needs more slots than the stack has.

Policy restated:
* a step pops k = min(32, size, room / 2) nodes when room = cap - margin -
  size >= 2, else one node (the top), and pushes up to three children per
  popped node, the children of lane 0's node first;
* the slot kernel's free slots each push one root while the stack holds
  fewer than refill_below nodes (refill_below + slots <= the spare slots);
* a node's children are one level deeper, and a window of W cells has at
  most W levels (each step consumes a pattern or a text cell)."""
import os
import random
import re

import pytest

SRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                   "cas-offinder-rust-old_b200", "csrc", "bulge.cu")


def _const(name):
    m = re.search(r"constexpr (?:uint32_t|int) %s = (\d+);" % name, open(SRC).read())
    assert m, name
    return int(m.group(1))


def _margin(wmax):
    # tb_margin: two slots per level, never below the 80 of a 40-cell window
    return 2 * max(wmax, 40)


def _simulate(rng, wmax, n_slots, refill_below, spare, n_trees, p_branch, max_steps):
    """Largest stack size the policy reaches; each tree is a root at depth 0
    whose nodes have 3 children with probability p_branch (else 0 or 1)
    while their depth is below wmax."""
    margin = _margin(wmax)
    cap = margin + spare
    stack = []  # depths
    roots_left = n_trees
    used = 0   # trees with nodes on the stack (slot occupancy, by count)
    live = {}  # tree id -> nodes on the stack
    next_id = 0
    peak = 0
    for _ in range(max_steps):
        # refill: free slots take roots while the stack is thin
        if n_slots and roots_left and len(stack) < refill_below:
            while used < n_slots and roots_left:
                stack.append((0, next_id))
                live[next_id] = 1
                next_id += 1
                used += 1
                roots_left -= 1
        elif not n_slots and not stack and roots_left:
            stack.append((0, next_id))  # one tree per warp
            live[next_id] = 1
            next_id += 1
            roots_left -= 1
        if not stack:
            if not roots_left:
                break
            continue
        room = cap - margin - len(stack)
        k = min(32, len(stack), room // 2) if room >= 2 else 1
        popped = [stack.pop() for _ in range(k)]  # lane 0 takes the top
        pushed = []
        for depth, tid in popped:
            live[tid] -= 1
            if depth + 1 < wmax:
                r = rng.random()
                n_kids = 3 if r < p_branch else (1 if r < p_branch + (1 - p_branch) / 2 else 0)
            else:
                n_kids = 0
            pushed.extend([(depth + 1, tid)] * n_kids)
            live[tid] += n_kids
        stack.extend(pushed)
        peak = max(peak, len(stack))
        assert len(stack) <= cap, (len(stack), cap)
        for tid in [t for t, n in live.items() if n == 0]:
            del live[tid]
            if n_slots:
                used -= 1
    return peak, cap


@pytest.mark.parametrize("wmax", [23, 40, 48, 72])
@pytest.mark.parametrize("n_slots", [0, 1, 3, 6, 8])
def test_stack_stays_inside_its_capacity(wmax, n_slots):
    slots_max = _const("kTbSlotsMax")
    slot_spare = _const("kTbSlotSpare")
    warp_spare = _const("kTbSpare")
    assert n_slots <= slots_max
    spare = slot_spare if n_slots else warp_spare
    rng = random.Random(1000 * wmax + n_slots)
    refills = [1, _const("kTbRefill"), slot_spare - slots_max] if n_slots else [0]
    worst = 0
    for refill_below in refills:
        for p_branch in (1.0, 0.9, 0.6):
            peak, cap = _simulate(rng, wmax, n_slots, refill_below, spare, n_trees=40,
                                  p_branch=p_branch, max_steps=4000)
            worst = max(worst, peak / cap)
    # the full-branching trees drive the stack close to its capacity: the
    # bound is tight, not just loose
    assert 0.5 < worst <= 1.0
