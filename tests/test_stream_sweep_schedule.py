"""The ring schedule of the fused streaming sweep launch (CPU model).

spin-glass_b200/csrc/stream_sweep.cu walks z with a ring of 4 slots per
colour: step z issues the copies of colour 0 at z+1 (up to L+1) and colour 1 at
z+2 (up to L), updates colour 0 in plane z, then colour 1 in plane z-1 (plane
index L standing for plane 0 at the end).  This model replays that schedule
for every even L the launch takes and checks what the kernel relies on:

* every plane a step reads sits in the ring slot it is read from, at the right
  version (colour 1 as it was before the sweep for colour 0's updates; colour 0
  already updated for colour 1's);
* no copy issued in a step overwrites a slot that step reads;
* no copy issued in a step reads a plane that step writes to global memory;
* every plane of both colours is updated exactly once.
"""
import pytest

SLOTS = 4


def _replay(L):
    glob = {(p, z): 0 for p in (0, 1) for z in range(L)}  # version in global memory
    ring = {}
    updates = {(p, z): 0 for p in (0, 1) for z in range(L)}

    def slot(u):
        return (u + SLOTS) % SLOTS

    def copy(p, u):
        ring[(p, slot(u))] = (u % L, glob[(p, u % L)])

    for p, u in [(0, 0), (1, -1), (1, 0), (1, 1)]:
        copy(p, u)
    for z in range(L + 2):
        pending = [(0, z + 1)] if z + 1 <= L + 1 else []
        pending += [(1, z + 2)] if z + 2 <= L else []
        halves = []
        if z < L:
            halves.append(([((0, z), 0), ((1, z - 1), 0), ((1, z), 0), ((1, z + 1), 0)], (0, z)))
        if 2 <= z <= L + 1:
            v = z - 1
            halves.append(([((1, v), 0), ((0, v - 1), 1), ((0, v), 1), ((0, v + 1), 1)], (1, v)))
        for reads, (wp, wu) in halves:
            for (p, u), version in reads:
                assert ring.get((p, slot(u))) == (u % L, version), (L, z, p, u)
                for pp, uu in pending:
                    assert not (pp == p and slot(uu) == slot(u)), (L, z, p, u, uu)
            for pp, uu in pending:
                assert not (pp == wp and uu % L == wu % L), (L, z, wp, wu, uu)
            glob[(wp, wu % L)] = 1
            updates[(wp, wu % L)] += 1
            if wp == 0:  # new colour-0 words also go to their ring slot
                ring[(0, slot(wu))] = (wu % L, 1)
        for pp, uu in pending:
            copy(pp, uu)
    assert all(n == 1 for n in updates.values())


@pytest.mark.parametrize("L", list(range(4, 60, 2)))
def test_ring_schedule(L):
    _replay(L)
