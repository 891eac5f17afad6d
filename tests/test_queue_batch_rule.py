"""The batched exact candidate queue of the search kernel against the
reference's sequential StdCandidateQueue rules, on random tie-heavy inputs.

Reference (router/data_structures/std_candidate_queue.hpp):
  try_push (:358-388): reject when |T| >= L and d >= lb; else push into the
    unexplored heap U and the top-L heap T, pop T's maximum by (dist, vid)
    when |T| > L, and set lb = T.top().dist. Entries evicted from T stay in U.
  should_terminate (:503-513): U empty -> stop; |T| < L -> go on; else stop
    when U's minimum has dist > lb.
  pop_best_unexplored_entry (:398-406): pop U's minimum by (dist, vid).

Kernel (artea_b200/csrc/search.cuh, queue_push_batch / queue_pop_peek): one
sorted array A of (dist, vid, explored); a row's candidates are accepted at
once by the closed-form rule
    accept(j) <=> d_j < lim and #{e in T : e.dist <= d_j} + #{i < j : d_i <= d_j} < L
(T = A's first min(n, L) entries, lim = lb when A holds L entries), merged
into A, and A is trimmed to the entries with dist <= lb (ties with lb stay:
the reference's evicted-but-expandable entries). A pop takes A's first
unexplored entry; none left is should_terminate.

Both are restated here in Python and run side by side: after every row and
every pop, T, the set of expandable entries and the popped entry agree.
"""
import numpy as np
import pytest

INF = float("inf")


class Sequential:
    def __init__(self, L):
        self.L, self.T, self.U, self.lb = L, [], set(), INF

    def push_row(self, row):
        for d, v in row:
            if len(self.T) >= self.L and d >= self.lb:
                continue
            self.U.add((d, v))
            self.T.append((d, v))
            if len(self.T) > self.L:
                self.T.remove(max(self.T))
            self.lb = max(self.T)[0]

    def expandable(self):
        if len(self.T) < self.L:
            return set(self.U)
        return {e for e in self.U if e[0] <= self.lb}

    def pop(self):
        if not self.U or (len(self.T) >= self.L and min(self.U)[0] > self.lb):
            return None
        e = min(self.U)
        self.U.remove(e)
        return e


class Batched:
    def __init__(self, L):
        self.L, self.cap, self.A, self.lb = L, 2 * L, [], INF   # A: sorted [d, v, explored]

    def push_row(self, row):
        L, A = self.L, self.A
        tn = min(len(A), L)
        lim = self.lb if len(A) >= L else INF
        accepted = []
        for j, (d, v) in enumerate(row):
            if not d < lim:
                continue
            pre = sum(1 for i in range(j) if row[i][0] < lim and row[i][0] <= d)
            if pre < L and (L - pre - 1 >= tn or A[L - pre - 1][0] > d):
                accepted.append([d, v, False])
        if not accepted:
            return
        A.extend(accepted)
        A.sort(key=lambda e: (e[0], e[1]))
        assert len(A) <= self.cap + len(accepted)
        del A[self.cap:]
        if len(A) >= L:
            self.lb = A[L - 1][0]
            k = L
            while k < len(A) and A[k][0] <= self.lb:
                k += 1
            del A[k:]
        assert len(A) <= self.cap, "more than L entries tie lb"

    def top(self):
        return [(e[0], e[1]) for e in self.A[:min(len(self.A), self.L)]]

    def expandable(self):
        return {(e[0], e[1]) for e in self.A if not e[2]}

    def pop(self):
        for e in self.A:
            if not e[2]:
                e[2] = True
                return (e[0], e[1])
        return None


def run_case(rng, L, n_ops, dist_levels, vid_space):
    seq, bat = Sequential(L), Batched(L)
    used = set()
    for _ in range(n_ops):
        if rng.random() < 0.6:
            k = int(rng.integers(0, 70))
            row = []
            for _ in range(k):
                v = int(rng.integers(0, vid_space))
                if v in used:
                    continue          # the visited set hands each id over once
                used.add(v)
                row.append((float(rng.integers(0, dist_levels)), v))
            seq.push_row(row)
            bat.push_row(row)
        else:
            a, b = seq.pop(), bat.pop()
            assert a == b, f"pop: sequential {a}, batched {b}"
        assert sorted(seq.T) == bat.top(), "top-L differs"
        assert seq.expandable() == bat.expandable(), "expandable entries differ"
        if len(seq.T) >= L:
            assert seq.lb == bat.lb


@pytest.mark.parametrize("seed", range(6))
def test_batched_queue_equals_sequential_try_push(seed):
    rng = np.random.default_rng(1000 + seed)
    for _ in range(500):
        L = int(rng.integers(1, 12))
        run_case(rng, L, n_ops=int(rng.integers(5, 40)), dist_levels=int(rng.integers(2, 12)),
                 vid_space=int(rng.integers(50, 400)))


def test_rule_counts_earlier_candidates_of_the_same_row():
    # A full queue and a row whose later candidates tie earlier accepted ones:
    # two 1.0 entries fill T (lb = 1.0), so the third 1.0 is rejected
    # (d >= lb); 0.5 then evicts (1.0, 4), which stays expandable (d == lb).
    seq, bat = Sequential(2), Batched(2)
    for q in (seq, bat):
        q.push_row([(5.0, 1), (6.0, 2)])
        q.push_row([(1.0, 3), (1.0, 4), (1.0, 5), (0.5, 6)])
    assert sorted(seq.T) == bat.top() == [(0.5, 6), (1.0, 3)]
    assert seq.expandable() == bat.expandable()


def gather_merge(old, batch, cap):
    """queue_merge's move step as the kernel runs it: final batch positions
    (rank in the old array + rank in the batch), then output chunks of 32,
    tail first, each lane reading its source (batch entry, or old entry
    o - #{batch positions < o}) before any lane of the chunk writes, in place."""
    n, m = len(old), len(batch)
    a = list(old) + [None] * (cap - n)
    batch = sorted(batch)
    posb = [sum(1 for e in old if e < b) + r for r, b in enumerate(batch)]
    p0, end = posb[0], min(n + m, cap)
    cb = end - 32
    while cb + 32 > p0:
        mask = 0
        for p in posb:
            if 0 <= p - cb < 32:
                mask |= 1 << (p - cb)
        nb = sum(1 for p in posb if p < cb)
        reads = []
        for lane in range(32):
            o = cb + lane
            if o < p0:
                continue
            before = nb + bin(mask & ((1 << lane) - 1)).count("1")
            reads.append((o, batch[before] if (mask >> lane) & 1 else a[o - before]))
        for o, e in reads:
            a[o] = e
        cb -= 32
    return a[:end]


@pytest.mark.parametrize("seed", range(3))
def test_gather_merge_moves_equal_a_sorted_merge(seed):
    # The in-place chunked moves give the sorted union cut at the capacity,
    # for batches of 1..64 entries landing anywhere, with and without truncation.
    rng = np.random.default_rng(2000 + seed)
    for _ in range(400):
        n = int(rng.integers(0, 700))
        m = int(rng.integers(1, 65))
        cap = n + int(rng.integers(0, 80)) if rng.random() < 0.5 else 1100
        keys = [(float(d), int(v)) for d, v in zip(rng.integers(0, 40, n + m), rng.permutation(100000)[: n + m])]
        old, batch = sorted(keys[:n]), keys[n:]
        assert gather_merge(old, batch, cap) == sorted(keys)[: min(n + m, cap)]


class BatchedRecording(Batched):
    """Batched, keeping the row's accepted candidates for the next-pop rule."""

    def push_row(self, row):
        L, A = self.L, self.A
        tn = min(len(A), L)
        lim = self.lb if len(A) >= L else INF
        self.last_accepted = []
        for j, (d, v) in enumerate(row):
            if not d < lim:
                continue
            pre = sum(1 for i in range(j) if row[i][0] < lim and row[i][0] <= d)
            if pre < L and (L - pre - 1 >= tn or A[L - pre - 1][0] > d):
                self.last_accepted.append((d, v))
        super().push_row(row)


@pytest.mark.parametrize("seed", range(3))
def test_next_pop_is_min_of_p2_and_smallest_accepted(seed):
    # The pipelined level-0 loop (l0_search_pipelined) decides the next pop right
    # after acceptance, before the merge: min(p2, smallest accepted candidate),
    # p2 being the first unexplored entry once the current one is popped; with
    # neither, the search ends. Checked against the merged queue's actual pop on
    # beam-search sequences (pop, push its row, pop, ...).
    rng = np.random.default_rng(3000 + seed)
    for _ in range(300):
        L = int(rng.integers(1, 12))
        q, used = BatchedRecording(L), set()
        first = (float(rng.integers(0, 8)), int(rng.integers(0, 400)))
        used.add(first[1])
        q.A.append([first[0], first[1], False])
        for _ in range(int(rng.integers(3, 40))):
            cur = q.pop()
            if cur is None:
                break
            p2 = next(((e[0], e[1]) for e in q.A if not e[2]), None)
            row = []
            for _ in range(int(rng.integers(0, 70))):
                v = int(rng.integers(0, 400))
                if v not in used:
                    used.add(v)
                    row.append((float(rng.integers(0, int(rng.integers(2, 12)))), v))
            q.push_row(row)
            options = [e for e in ([p2] if p2 else []) + ([min(q.last_accepted)] if q.last_accepted else [])]
            predicted = min(options) if options else None
            actual = next(((e[0], e[1]) for e in q.A if not e[2]), None)
            assert predicted == actual, (L, cur, p2, q.last_accepted, actual)
