"""The search kernel's exact visited set (artea_b200/csrc/search.cuh: Visited,
table_walk, table_try, visited_test_and_set2) restated in Python and checked
against a plain set.

The reference marks visited vertices in a version-tagged table
(containers/version_tag_table.hpp:128-132 test_and_set, :142-148 clear): a
vertex is new exactly once between clears. The kernel keeps a shared-memory
table of 2^t buckets of four 16-bit slots (vid -> p = vid * 0x9E3779B1 mod 2^k,
bucket A = p >> (k - t), quotient Q = the low bits; a second bucket
B = A ^ h(Q) holds Q | 0x8000 once A is full) and spills ids whose two buckets
are full to a bitset. Lanes of a warp insert distinct ids at once: each reads
both buckets, and a CAS that lost its slot to another lane reads again.

Checked here: with lanes interleaved adversarially (snapshot reads, CAS in a
random lane order), every id is reported new exactly once and never again,
at loads from a quarter of the slots to three times their number; every
stored value decodes to the one id that was put there; visited_kbits rejects
tables whose quotients would not fit in 15 bits.
"""
import random

import pytest

MUL = 0x9E3779B1
ALT_MUL = 0x2545F491
FLAG = 0x8000
EMPTY = 0xFFFF
M32 = 0xFFFFFFFF


def visited_kbits(n, table_log):
    kb = 1
    while kb < 32 and (1 << kb) < n:
        kb += 1
    if table_log == 0:
        return kb
    tbits = table_log + 1
    kb = max(kb, tbits + 1)
    return 0 if kb - tbits > 15 else kb


class Table:
    def __init__(self, n, table_log):
        self.kbits = visited_kbits(n, table_log)
        assert self.kbits
        self.tbits = table_log + 1
        self.qbits = self.kbits - self.tbits
        self.slots = [[EMPTY] * 4 for _ in range(1 << self.tbits)]
        self.bits = set()

    def walk(self, vid):
        p = (vid * MUL) & ((1 << self.kbits) - 1)
        a, q = p >> self.qbits, p & ((1 << self.qbits) - 1)
        h = ((q * ALT_MUL) & M32) >> (32 - self.tbits)
        b = (a ^ h) if (self.qbits <= 14 and h != 0) else None
        return a, b, q

    def try_step(self, w, snap):
        """table_try on a snapshot of the two buckets: ('present',), ('full',)
        or ('cas', bucket, slot, value)."""
        a, b, q = w
        sa, sb = snap
        if q in sa or (b is not None and (q | FLAG) in sb):
            return ("present",)
        if EMPTY in sa:
            return ("cas", a, sa.index(EMPTY), q)
        if b is not None and EMPTY in sb:
            return ("cas", b, sb.index(EMPTY), q | FLAG)
        return ("full",)

    def warp_test_and_set(self, vids, rng):
        """One warp step over distinct ids; returns {vid: is_new}."""
        walks = {v: self.walk(v) for v in vids}
        pending, result = set(vids), {}
        for _ in range(24):
            if not pending:
                break
            snaps = {v: (list(self.slots[walks[v][0]]),
                         list(self.slots[walks[v][1]]) if walks[v][1] is not None else [0, 0, 0, 0])
                     for v in pending}
            order = list(pending)
            rng.shuffle(order)
            for v in order:
                act = self.try_step(walks[v], snaps[v])
                if act[0] == "present":
                    result[v] = False
                elif act[0] == "full":
                    result[v] = v not in self.bits   # atomicOr on the bitset
                    self.bits.add(v)
                else:
                    _, bucket, slot, value = act
                    snap = snaps[v][0] if bucket == walks[v][0] else snaps[v][1]
                    # CAS on the slot's word: it succeeds only if that word is unchanged.
                    word = slot // 2
                    if self.slots[bucket][2 * word:2 * word + 2] == snap[2 * word:2 * word + 2]:
                        self.slots[bucket][slot] = value
                        result[v] = True
                    else:
                        continue
                pending.discard(v)
        assert not pending, "a walk did not end"
        return result

    def decode(self):
        """Every stored value back to its vid."""
        inv = pow(MUL, -1, 1 << self.kbits)
        out = []
        for bucket, slots in enumerate(self.slots):
            for val in slots:
                if val == EMPTY:
                    continue
                q = val & ~FLAG & 0xFFFF if (val & FLAG and self.qbits <= 14) else val
                a = bucket
                if val & FLAG and self.qbits <= 14:
                    h = ((q * ALT_MUL) & M32) >> (32 - self.tbits)
                    a = bucket ^ h
                p = (a << self.qbits) | q
                out.append((p * inv) & ((1 << self.kbits) - 1))
        return out


@pytest.mark.parametrize("n,table_log,load", [(10_000_000, 9, 0.25), (10_000_000, 9, 0.7), (10_000_000, 9, 3.0),
                                              (1_000_000, 8, 1.0), (300, 6, 2.0), (1_000_000, 10, 0.9)])
def test_warp_inserts_report_each_id_new_exactly_once(n, table_log, load):
    rng = random.Random(n * 31 + table_log * 7 + int(load * 10))
    t = Table(n, table_log)
    capacity = 4 << t.tbits
    universe = rng.sample(range(n), min(n, int(capacity * load) + 64))
    seen = set()
    for _ in range(max(20, int(capacity * load * 3) // 64)):
        row = rng.sample(universe, 64)   # a level-0 row: 64 distinct ids, some already visited
        got = t.warp_test_and_set(row, rng)
        for v in row:
            assert got[v] == (v not in seen), v
            seen.add(v)
    stored = t.decode()
    assert len(stored) == len(set(stored))
    assert set(stored) | t.bits == seen and not (set(stored) & t.bits)


def test_kbits_rejects_quotients_past_15_bits():
    assert visited_kbits(10_000_000, 9) == 24          # 2^10 buckets, 14-bit quotients: two choices
    assert visited_kbits(10_000_000, 8) == 24          # 15-bit quotients: one choice
    assert visited_kbits(10_000_000, 7) == 0           # 16-bit quotients would reach 0xFFFF
    assert visited_kbits(100, 9) == 11                 # small graphs: one quotient bit at least
    assert visited_kbits(1 << 20, 0) == 20


def test_second_bucket_only_when_quotient_has_room_for_the_flag():
    t = Table(10_000_000, 8)                           # 15-bit quotients
    assert all(t.walk(v)[1] is None for v in range(1000))
    t = Table(10_000_000, 9)                           # 14-bit quotients
    assert sum(t.walk(v)[1] is not None for v in range(1000)) > 990
