"""Model check of the block kernels' slab ring (csrc/sweep_kernels.cu).

A block kernel's producer warp copies the block's slabs, in item order, into
R slots shared by the CTA; consumer warps take the items of each level
round-robin, wait for each slab's slot, read it and release it; levels are
separated by a barrier among the consumers.  Each slot has two mbarriers
("full": the copy landed, "empty": the slab was read), waited on by phase
parity, and the producer posts the use number of each slot before the copy.

This test restates that protocol as a small state machine and explores it
under random interleavings (copies landing late, warps running at different
speeds) on level structures like a block's: every consumer must read the
slab it expects, and the ring must never stall with work left.  It also
shows why the posted use number is there: without it, a consumer that runs
two uses of a slot ahead of the copy in it passes its parity wait on an
earlier phase and reads another slab.

The model follows the mbarrier rule of the PTX ISA: a parity wait for parity
p succeeds when the phase with parity p has completed, i.e. when p differs
from the parity of the current (incomplete) phase.
"""
import random

import pytest


def parity_wait_ok(completed_phases, p):
    return p != (completed_phases & 1)


def run(levels, ncw, R, seed, gate=True, max_actions=200000):
    """levels: list of levels, each a list of items (slab counts).  Returns
    'ok', 'wrong-read' or 'stall'."""
    rng = random.Random(seed)
    items = [n for lev in levels for n in lev]
    first, q = [], 0
    for n in items:
        first.append(q)
        q += n
    total = q
    # per consumer warp, its items level by level (round-robin inside a level)
    work, k = [[] for _ in range(ncw)], 0
    for lev in levels:
        for w in range(ncw):
            work[w].append([k + p for p in range(len(lev)) if p % ncw == w])
        k += len(lev)
    full_c = [0] * R      # completed phases of each slot's full barrier
    empty_c = [0] * R     # completed phases of each slot's empty barrier
    posted = [-1] * R     # use number posted for each slot
    content = [None] * R  # slab the slot holds once its copy landed
    inflight = []         # (slot, slab) copies issued, not landed
    nxt = 0               # producer: next slab to issue
    cons = [[0, 0, 0] for _ in range(ncw)]  # consumer: level, item of the level, slab of the item
    at_barrier = [False] * ncw
    arrived = [0] * len(levels)  # consumers at each level's barrier
    reads = 0

    def settle(w):
        L, i, _ = cons[w]
        if L < len(levels) and i >= len(work[w][L]) and not at_barrier[w]:
            at_barrier[w] = True
            arrived[L] += 1

    for w in range(ncw):
        settle(w)
    for _ in range(max_actions):
        acts = []
        if nxt < total:
            slot, use = nxt % R, nxt // R
            if use == 0 or parity_wait_ok(empty_c[slot], (use - 1) & 1):
                acts.append(("issue",))
        if inflight:
            acts.append(("land",))
        for w in range(ncw):
            L, i, j = cons[w]
            if L >= len(levels):
                continue
            if at_barrier[w]:
                if arrived[L] == ncw:
                    acts.append(("advance", w))
                continue
            qq = first[work[w][L][i]] + j
            slot, use = qq % R, qq // R
            if gate and posted[slot] != use:
                continue
            if parity_wait_ok(full_c[slot], use & 1):
                acts.append(("read", w))
        if not acts:
            return "ok" if reads == total else "stall"
        a = rng.choice(acts)
        if a[0] == "issue":
            slot, use = nxt % R, nxt // R
            posted[slot] = use
            inflight.append((slot, nxt))
            nxt += 1
        elif a[0] == "land":
            slot, slab = inflight.pop(rng.randrange(len(inflight)))
            content[slot] = slab
            full_c[slot] += 1
        elif a[0] == "advance":
            w = a[1]
            cons[w] = [cons[w][0] + 1, 0, 0]
            at_barrier[w] = False
            settle(w)
        else:
            w = a[1]
            L, i, j = cons[w]
            it = work[w][L][i]
            qq = first[it] + j
            slot = qq % R
            if content[slot] != qq:
                return "wrong-read"
            reads += 1
            empty_c[slot] += 1
            j += 1
            if j == items[it]:
                i, j = i + 1, 0
            cons[w] = [L, i, j]
            settle(w)
    return "stall"


def block_like(rng):
    """A block's level structure: many short items at the leaves, fewer and
    longer ones towards the root (slab counts 1-8)."""
    nlev = rng.randint(2, 6)
    levels = []
    width = rng.randint(8, 40)
    for L in range(nlev):
        levels.append([rng.randint(1, 2 + 2 * L) for _ in range(max(1, width))])
        width = max(1, width // 2)
    return levels


@pytest.mark.parametrize("seed", range(40))
def test_ring_with_posted_use_numbers_reads_every_slab_and_never_stalls(seed):
    rng = random.Random(1000 + seed)
    levels = block_like(rng)
    ncw = rng.choice([4, 8])
    R = rng.choice([2, 3, 4, 8, 10, 24])
    assert run(levels, ncw, R, seed, gate=True) == "ok"


def test_parity_waits_alone_let_a_warp_read_another_slab():
    """Without the posted use number, some interleaving lets a consumer pass
    its parity wait on a slot two uses behind and read the wrong slab (the
    hazard the use number removes)."""
    outcomes = set()
    for seed in range(300):
        rng = random.Random(seed)
        levels = block_like(rng)
        outcomes.add(run(levels, 8, rng.choice([2, 3, 4]), seed, gate=False))
        if "wrong-read" in outcomes:
            break
    assert "wrong-read" in outcomes
