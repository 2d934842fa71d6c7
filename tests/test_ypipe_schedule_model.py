"""CPU model of the fused y-pass schedule (giem2g_b200/csrc/ypipe.cu), run under random interleavings.

Each CTA has a producer (grabs the next unit from a global counter after a free stage, issues the tensor copy,
waits for the forward transforms of the unit's batch, then issues the spectrum copy), consumer groups (stage
tickets taken in order, the stage released after the sums, the unit's completion counted) and FFT warps
(grab transform tasks in the kernel's order F(0), F(1), I(0), F(2), I(1), ..., I(nb-1); an inverse task waits
until its batch's units are all contracted).  The model checks that every schedule ends with every task and
unit done exactly once, that no spectrum copy is issued before its batch's forward transforms finished, that
no inverse transform starts before its batch's contractions finished, and that stage slots are never
overwritten while a group still reads them.  The task decode is the kernel's, restated.  (Without the release
of the stage at a group's end ticket, a configuration with more groups than stages never ends: the model found
that before the kernel ran.)
"""
import random

import pytest


def decode(t, fpb, nb, nblk, qb):
    seg, within = divmod(t, fpb)
    if seg == 0:
        fwd, b = True, 0
    elif seg == 2 * nb - 1:
        fwd, b = False, nb - 1
    elif seg & 1:
        fwd, b = True, (seg + 1) // 2
    else:
        fwd, b = False, seg // 2 - 1
    qi, rem = divmod(within, 2 * nblk)
    sx, lb = divmod(rem, nblk)
    return fwd, b, b * qb + qi, sx, lb


def test_task_decode_covers_every_transform_once():
    for nx, zl, nl, qb in ((4, 96, 8, 4), (8, 96, 8, 4), (128, 96, 8, 4), (32, 192, 8, 4), (16, 96, 4, 4)):
        nb, nblk = nx // qb, (zl + nl - 1) // nl
        fpb = qb * 2 * nblk
        seen, order = set(), []
        for t in range(2 * nb * fpb):
            fwd, b, q, sx, lb = decode(t, fpb, nb, nblk, qb)
            assert 0 <= q < nx and q // qb == b and sx in (0, 1) and 0 <= lb < nblk
            key = (fwd, q, sx, lb)
            assert key not in seen
            seen.add(key)
            order.append((fwd, b))
        assert len(seen) == 2 * nx * 2 * nblk
        # every inverse task of batch b comes after every forward task of batches b and b + 1
        last_f = {b: max(i for i, (f, bb) in enumerate(order) if f and bb == b) for b in range(nb)}
        for i, (f, b) in enumerate(order):
            if not f:
                assert i > last_f[b] and (b + 1 >= nb or i > last_f[b + 1])


class Sim:
    def __init__(self, rng, ncta, nx, ny, nblk, qb, ng, nstage):
        self.rng, self.ncta, self.nx, self.ny, self.qb = rng, ncta, nx, ny, qb
        self.nb, self.nblk, self.ng, self.nstage = nx // qb, nblk, ng, nstage
        self.fpb = qb * 2 * nblk
        self.total = nx * ny
        self.next_unit = 0
        self.next_task = 0
        self.f_done = [0] * self.nb
        self.c_done = [0] * self.nb          # finished units (one arrival per unit in the model)
        self.units_done = []
        self.tasks_done = []
        self.ctas = [self.new_cta() for _ in range(ncta)]

    def new_cta(self):
        return {"prod": {"it": 0, "state": "free", "u": None, "done": False},
                "stage": [None] * self.nstage,          # (ticket, unit, landed) in each slot
                "released": [True] * self.nstage,
                "passed": 0,
                "groups": [{"it": g, "done": False, "phase": "wait"} for g in range(self.ng)],
                "fft": {"task": None, "done": False}}

    # --- producer: one step at a time
    def step_producer(self, c):
        p = c["prod"]
        if p["done"]:
            return False
        slot = p["it"] % self.nstage
        if p["state"] == "free":
            if not c["released"][slot]:
                return False
            u = self.next_unit
            self.next_unit += 1
            if u >= self.total:
                p["state"] = "sentinel"
                p["sent"] = 0
                return True
            c["released"][slot] = False
            c["stage"][slot] = [p["it"], u, False]
            p["u"] = u
            p["state"] = "await_f"
            return True
        if p["state"] == "await_f":
            b = (p["u"] // self.ny) // self.qb
            if self.f_done[b] < self.fpb:
                return False
            c["stage"][slot][2] = True      # the spectrum copy may go; the stage lands
            p["it"] += 1
            p["state"] = "free"
            return True
        if p["state"] == "sentinel":
            if p["sent"] == self.ng:
                p["done"] = True
                return True
            if not c["released"][slot]:
                return False
            c["released"][slot] = False
            c["stage"][slot] = [p["it"], -1, True]
            p["it"] += 1
            p["sent"] += 1
            return True
        return False

    def step_group(self, c, g):
        gr = c["groups"][g]
        if gr["done"]:
            return False
        it = gr["it"]
        slot = it % self.nstage
        if gr["phase"] == "wait":
            if c["passed"] < it:
                return False
            st = c["stage"][slot]
            if st is None or st[0] != it or not st[2]:
                return False
            c["passed"] = max(c["passed"], it + 1)
            if st[1] < 0:
                c["released"][slot] = True   # end tickets release their stage too
                gr["done"] = True
                return True
            gr["unit"] = st[1]
            gr["phase"] = "sums"
            return True
        if gr["phase"] == "sums":
            assert c["stage"][slot][0] == it and c["stage"][slot][1] == gr["unit"]   # not overwritten
            c["released"][slot] = True
            gr["phase"] = "store"
            return True
        if gr["phase"] == "store":
            u = gr["unit"]
            self.units_done.append(u)
            self.c_done[(u // self.ny) // self.qb] += 1
            gr["it"] += self.ng
            gr["phase"] = "wait"
            return True
        return False

    def step_fft(self, c):
        f = c["fft"]
        if f["done"]:
            return False
        if f["task"] is None:
            t = self.next_task
            self.next_task += 1
            if t >= 2 * self.nb * self.fpb:
                f["done"] = True
                return True
            f["task"] = decode(t, self.fpb, self.nb, self.nblk, self.qb)
            return True
        fwd, b, q, sx, lb = f["task"]
        if not fwd:
            if self.c_done[b] < self.qb * self.ny:
                return False
            self.tasks_done.append(("I", q, sx, lb))
        else:
            self.tasks_done.append(("F", q, sx, lb))
            self.f_done[b] += 1
        f["task"] = None
        return True

    def run(self, max_steps=10_000_000):
        actors = []
        for c in self.ctas:
            actors.append(lambda c=c: self.step_producer(c))
            for g in range(self.ng):
                actors.append(lambda c=c, g=g: self.step_group(c, g))
            actors.append(lambda c=c: self.step_fft(c))
        for _ in range(max_steps):
            self.rng.shuffle(actors)
            if not any(a() for a in actors):
                break
        return self


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("cfg", [(3, 8, 4, 2, 2, 2), (5, 4, 8, 3, 6, 5), (2, 16, 4, 2, 4, 4), (7, 12, 8, 2, 2, 2)])
def test_schedule_terminates_in_order(seed, cfg):
    ncta, nx, ny, nblk, ng, nstage = cfg
    qb = 4
    sim = Sim(random.Random(seed), ncta, nx, ny, nblk, qb, ng, nstage).run()
    assert sorted(sim.units_done) == list(range(nx * ny))
    assert len(sim.tasks_done) == 2 * nx * 2 * nblk
    for c in sim.ctas:
        assert c["prod"]["done"] and c["fft"]["done"] and all(g["done"] for g in c["groups"])
