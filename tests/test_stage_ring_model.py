"""Model of the stage-ring protocol of the barrier-free contraction (k_contract_wl in csrc/contract.cu).

One producer lane streams units (tickets) into NSTAGE shared-memory stages; ticket it uses stage
it % NSTAGE in round it / NSTAGE. NG warp groups take tickets round-robin (group g: g, g + NG, ...).
Every warp of a group waits on the stage's full barrier, reads it and arrives on its empty barrier, which
completes when all warps of the group have arrived. mbarrier parity semantics: a wait for parity P
succeeds when the barrier's current phase parity differs from P.

The model explores random interleavings, with copies landing out of order, and checks two things:
* a warp never passes a wait while its stage holds another unit or a copy is in flight;
* the producer never issues into a stage that a warp is still reading.

Without the in-order ticket rule, a parity wait can pass on a stale phase as soon as two groups share a
ring that is not a multiple of their count. With the rule (a warp waits for ticket it only after ticket
it-1 has been passed), every shape is safe, including more groups than stages.
"""
import random

import pytest


def _run(NG, NSTAGE, W, n_units, in_order, seed):
    rng = random.Random(seed)
    full_ph = [0] * NSTAGE
    empty_ph = [0] * NSTAGE
    empty_cnt = [0] * NSTAGE
    content = [None] * NSTAGE
    inflight = {}
    readers = [set() for _ in range(NSTAGE)]
    prod = 0
    passed = 0
    warps = {(g, w): {"it": g, "state": "gate" if in_order else "wait"} for g in range(NG) for w in range(W)}
    for _ in range(400000):
        acts = []
        if prod < n_units:
            s, r = prod % NSTAGE, prod // NSTAGE
            if r == 0 or (empty_ph[s] & 1) != ((r - 1) & 1):
                acts.append(("issue",))
        acts += [("land", s) for s in inflight]
        acts += [("warp", k) for k, st in warps.items() if st["it"] < n_units]
        if not acts:
            done = prod >= n_units and not inflight and all(st["it"] >= n_units for st in warps.values())
            return "ok" if done else "deadlock"
        a = rng.choice(acts)
        if a[0] == "issue":
            s = prod % NSTAGE
            if readers[s] or s in inflight:
                return "issue into a busy stage"
            inflight[s] = prod
            prod += 1
        elif a[0] == "land":
            s = a[1]
            content[s] = inflight.pop(s)
            full_ph[s] += 1
        else:
            key = a[1]
            st = warps[key]
            it = st["it"]
            s, r = it % NSTAGE, it // NSTAGE
            if st["state"] == "gate":
                if passed >= it:
                    st["state"] = "wait"
            elif st["state"] == "wait":
                if (full_ph[s] & 1) != (r & 1):
                    if content[s] != it or s in inflight:
                        return "stale pass"
                    passed = max(passed, it + 1)
                    readers[s].add(key)
                    st["state"] = "read"
            else:
                readers[s].discard(key)
                empty_cnt[s] += 1
                if empty_cnt[s] == W:
                    empty_cnt[s] = 0
                    empty_ph[s] += 1
                st["it"] = it + NG
                st["state"] = "gate" if in_order else "wait"
    return "livelock"


# (groups, stages) of the shipped variants and a few others, more groups than stages included
SHAPES = [(1, 3), (2, 3), (3, 3), (4, 3), (2, 6), (3, 6), (4, 6), (6, 6), (8, 6), (2, 5), (4, 5), (5, 5), (3, 2)]


@pytest.mark.parametrize("ng,nstage", SHAPES)
def test_in_order_tickets_are_safe(ng, nstage):
    for seed in range(60):
        assert _run(ng, nstage, 2, 40, True, seed) == "ok", seed


def test_shared_ring_without_the_rule_passes_stale_phases():
    """The race the rule removes: two groups on three stages, four groups on three or six stages."""
    for ng, nstage in [(2, 3), (4, 3), (4, 6)]:
        results = {_run(ng, nstage, 2, 40, False, seed) for seed in range(200)}
        assert "stale pass" in results, (ng, nstage)
    # a ring whose stages are a multiple of the groups is safe even without it (each group owns stages)
    assert {_run(2, 4, 2, 40, False, seed) for seed in range(100)} == {"ok"}
