"""The mbarrier hand-off schedule of the TMA-staged tcgen05 convolutions
(`conv_umma_tma` and `conv_umma_pair` in flursys_b200/csrc/fcgnet.cu),
restated in Python and run under random interleavings of the issuer, the
four epilogue warps and the asynchronous copies and MMA groups.

Each step of the kernels' schedule is mirrored: the plane ring (slot
(p - z0 + 1) % NS, phase parity ((p - z0 + 1) // NS) & 1), the prologue
copies, the waits on `full`, `done` and `empty` with their parities, and
the refills after the previous group's MMAs are seen complete. The checks:
every MMA group reads the planes it needs and nothing overwrites a slot
an in-flight group reads, no accumulator buffer is reissued before its
epilogue has read it, every parity wait refers to a phase that can still
come, and the schedule always terminates."""
import random

import pytest


class Bar:
    """An mbarrier: arrival count, transaction bytes, phase."""

    def __init__(self, count):
        self.count = count
        self.pending = count
        self.phase = 0
        self.tx = 0

    def arrive(self):
        self.pending -= 1
        self._advance()

    def expect_tx(self, nbytes):
        self.tx += nbytes
        self.arrive()

    def complete_tx(self, nbytes):
        self.tx -= nbytes
        self._advance()

    def _advance(self):
        if self.pending == 0 and self.tx == 0:
            self.phase += 1
            self.pending = self.count

    def passed(self, parity):
        """try_wait.parity: the phase of this parity has completed."""
        return (self.phase & 1) != parity


def run_schedule(z0, z1, ns, pairs, seed):
    rnd = random.Random(seed)
    full = [Bar(1) for _ in range(ns)]
    done = [Bar(1) for _ in range(2)]
    empty = [Bar(4) for _ in range(2)]
    slot_of = lambda p: (p - z0 + 1) % ns
    parity = lambda p: ((p - z0 + 1) // ns) & 1
    step = 2 if pairs else 1
    groups = (z1 - z0) // step
    span = (lambda z: range(z - 1, z + 3)) if pairs else (lambda z: range(z - 1, z + 2))
    content, inflight, owner, reads = {}, [], {0: None, 1: None}, []

    def copy(p):
        s = slot_of(p)
        old = content.get(s)
        for kind, g in inflight:
            assert not (kind == "mma" and old in span(z0 + step * g)), ("slot overwritten while read", p, old, g)
        full[s].expect_tx(1)
        content[s] = None
        inflight.append(("tma", p))

    def issuer():
        for p in range(z0 - 1, min(z1, z0 - 2 + ns) + 1):
            copy(p)
        yield
        waited = z0 - 2
        for g in range(groups):
            z, b = z0 + step * g, g & 1
            if g >= 2:
                while not empty[b].passed(((g - 2) >> 1) & 1):
                    yield
            last = z + 2 if pairs else z + 1
            while waited < last:
                while not full[slot_of(waited + 1)].passed(parity(waited + 1)):
                    yield
                waited += 1
            for q in span(z):
                assert content[slot_of(q)] == q, ("MMA group reads a wrong plane", g, q)
            assert owner[b] is None, ("accumulator reissued before its epilogue", g)
            owner[b] = g
            inflight.append(("mma", g))
            if g >= 1:
                while not done[(g - 1) & 1].passed(((g - 1) >> 1) & 1):
                    yield
                first = z - 3 + ns if pairs else z - 2 + ns
                last_refill = z - 2 + ns
                for p in range(first, min(last_refill, z1) + 1):
                    copy(p)
            yield

    def epilogue(w):
        for g in range(groups):
            b = g & 1
            while not done[b].passed((g >> 1) & 1):
                yield
            assert owner[b] == g and ("mma", g) not in inflight
            reads.append((w, g))
            yield
            empty[b].arrive()
            if sum(1 for _, gg in reads if gg == g) == 4:
                owner[b] = None
            yield

    threads = [issuer()] + [epilogue(w) for w in range(4)]
    steps = 0
    while threads or inflight:
        steps += 1
        assert steps < 400000, "the schedule does not terminate"
        if inflight and rnd.random() < 0.3:
            i = rnd.randrange(len(inflight))
            kind, v = inflight[i]
            if kind == "mma" and any(k == "mma" and vv < v for k, vv in inflight):
                continue  # MMA groups complete in issue order
            inflight.pop(i)
            if kind == "tma":
                content[slot_of(v)] = v
                full[slot_of(v)].complete_tx(1)
            else:
                done[v & 1].arrive()
            continue
        if not threads:
            continue
        t = rnd.choice(threads)
        try:
            next(t)
        except StopIteration:
            threads.remove(t)
    assert len(reads) == 4 * groups


@pytest.mark.parametrize("ns", [4, 5])
def test_one_plane_schedule(ns):
    for z0 in (0, 16):
        for kz in (1, 2, 3, 8, 64):
            for nz in (z0 + 1, z0 + kz, z0 + 100):
                z1 = min(z0 + kz, nz)
                for seed in range(6):
                    run_schedule(z0, z1, ns, False, seed)


def test_paired_plane_schedule():
    for z0 in (0, 16):
        for kz in (2, 4, 8, 64):
            for nz in (z0 + 2, z0 + kz, z0 + 100):
                z1 = min(z0 + kz, nz)
                if (z1 - z0) % 2:
                    continue
                for seed in range(6):
                    run_schedule(z0, z1, 6, True, seed)
