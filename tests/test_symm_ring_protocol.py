"""The handover protocol of the warp-specialised tensor-core SYMM (tile_symm_tc3_kernel), modelled on
the CPU with random interleavings of its roles.

The kernel's roles (two producer lanes taking the even and the odd blocks, four converter warps, one
MMA lane, four epilogue warps) pass NS shared-memory stages and two tensor-memory accumulators
through mbarriers that are waited on by phase parity.  A parity wait is only sound while the waiter
is at most one phase ahead of the barrier, so the model checks, over random unit lists and random
completion orders of the bulk copies and MMA commits:
  * no role waits forever (the simulation ends);
  * a producer refills a stage only after the MMAs of the stage's previous block have completed;
  * the converters and the MMA lane always see the block they expect in a stage;
  * an accumulator is reused only after the epilogue has read it.
A mutation test plants a fault in the model (a converter that skips a wait, as a converter without a
tile row once did in a variant with a separate low-part ring) and checks that the model catches it.
"""
import random

NS = 4          # stages of tile_symm_tc3_kernel
NS_LOW, NL = 6, 2   # stages and low-part buffers of the dropped variant with a separate low ring


class Bar:
    """mbarrier: arrival count, transaction bytes, phase; try_wait.parity(p) succeeds once the phase
    of parity p has completed, i.e. while the current phase parity differs from p."""

    def __init__(self, count):
        self.count, self.pending, self.phase, self.tx = count, count, 0, 0

    def arrive(self):
        self.pending -= 1
        self._check()

    def arrive_tx(self, nbytes):
        self.tx += nbytes
        self.arrive()

    def complete_tx(self, nbytes):
        self.tx -= nbytes
        self._check()

    def _check(self):
        if self.pending == 0 and self.tx == 0:
            self.phase += 1
            self.pending = self.count

    def done(self, parity):
        return (self.phase & 1) != parity


def simulate(units, seed, ns=NS, low_ring=False, skip_low_wait_without_tile=False):
    """units: list of (tn, nq) per unit of one CTA (tile rows of the subdomain, tile rows of the unit).
    low_ring: the variant with NL separate low-part buffers, freed by an MMA commit per block."""
    rnd = random.Random(seed)
    NS = ns
    full = [Bar(1) for _ in range(NS)]
    conv = [Bar(4) for _ in range(NS)]
    empty = [Bar(1) for _ in range(NS)]
    lofree = [Bar(1) for _ in range(NL)]
    accf = [Bar(1) for _ in range(2)]
    acce = [Bar(4) for _ in range(2)]
    inflight = []
    stage = {}      # stage -> (state, block)
    low = {}        # low buffer -> (state, block)

    def producer(par):
        t = 0
        for tn, nq in units:
            for _ in range(tn):
                if t % 2 == par:
                    s = t % NS
                    if t >= NS:
                        while not empty[s].done(((t // NS) - 1) & 1):
                            yield
                    assert stage.get(s, ("free", None))[0] == "free", ("stage refilled while in use", s, t)
                    stage[s] = ("copying", t)
                    full[s].arrive_tx(4096 * nq + 4096)
                    inflight.extend([("copy", s, 4096)] * (nq + 1))
                    yield
                t += 1

    def converter(q):
        t = 0
        for tn, nq in units:
            for _ in range(tn):
                s, l = t % NS, t % NL
                while not full[s].done((t // NS) & 1):
                    yield
                assert stage[s][1] == t and stage[s][0] in ("copying", "converting"), (stage[s], t)
                stage[s] = ("converting", t)
                if low_ring:
                    if t >= NL and not (skip_low_wait_without_tile and q >= nq):
                        while not lofree[l].done(((t // NL) - 1) & 1):
                            yield
                    if q < nq:
                        assert low.get(l, ("free", None))[0] in ("free", "converting"), ("low buffer in use", l, t)
                        low[l] = ("converting", t)
                conv[s].arrive()
                t += 1
                yield

    def mma():
        t = 0
        for k, (tn, _) in enumerate(units):
            a = k & 1
            if k >= 2:
                while not acce[a].done(((k >> 1) - 1) & 1):
                    yield
            for j in range(tn):
                s, l = t % NS, t % NL
                while not conv[s].done((t // NS) & 1):
                    yield
                assert stage[s] == ("converting", t), (stage[s], t)
                stage[s] = ("mma", t)
                inflight.append(("empty", s))
                if low_ring:
                    low[l] = ("mma", t)
                    inflight.append(("lofree", l))
                if j == tn - 1:
                    inflight.append(("accf", a))
                t += 1
                yield

    def epilogue():
        for k in range(len(units)):
            a = k & 1
            while not accf[a].done((k >> 1) & 1):
                yield
            acce[a].arrive()
            yield

    roles = [producer(0), producer(1)] + [converter(q) for q in range(4)] + [mma()] + [epilogue() for _ in range(4)]
    alive = list(roles)
    steps = 0
    while alive or inflight:
        steps += 1
        assert steps < 200000, "a role waits forever"
        if inflight and rnd.random() < 0.3:
            copies = [i for i, e in enumerate(inflight) if e[0] == "copy"]
            commits = [i for i, e in enumerate(inflight) if e[0] != "copy"]
            # copies land in any order; the commits of one thread complete in issue order
            i = rnd.choice(copies) if copies and (not commits or rnd.random() < 0.5) else commits[0]
            ev = inflight.pop(i)
            if ev[0] == "copy":
                full[ev[1]].complete_tx(ev[2])
            elif ev[0] == "empty":
                stage[ev[1]] = ("free", None)
                empty[ev[1]].arrive()
            elif ev[0] == "lofree":
                low[ev[1]] = ("free", None)
                lofree[ev[1]].arrive()
            else:
                accf[ev[1]].arrive()
            continue
        if alive:
            r = rnd.choice(alive)
            try:
                next(r)
            except StopIteration:
                alive.remove(r)


def random_units(rnd):
    units = []
    for _ in range(rnd.randint(1, 8)):
        tn = rnd.randint(1, 14)
        i0 = 4 * rnd.randint(0, (tn - 1) // 4)
        units.append((tn, min(4, tn - i0)))
    return units


def test_ring_protocol_holds():
    for seed in range(150):
        simulate(random_units(random.Random(seed)), seed)


def test_low_ring_variant_holds_when_every_warp_waits():
    for seed in range(150):
        simulate(random_units(random.Random(seed)), seed, ns=NS_LOW, low_ring=True)


def test_model_catches_a_skipped_wait():
    """Planted fault: converters without a tile row skip the low-buffer wait, so a later wait can be
    two phases ahead of the barrier and its parity test passes too early."""
    caught = 0
    for seed in range(300):
        try:
            simulate(random_units(random.Random(seed)), seed, ns=NS_LOW, low_ring=True,
                     skip_low_wait_without_tile=True)
        except AssertionError:
            caught += 1
    assert caught > 0
