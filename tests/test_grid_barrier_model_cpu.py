"""The grid barrier of the persistent kernels (``grid_sync`` in
``csrc/fugu_internal.cuh``), modelled and checked exhaustively on the CPU.

Within a launch the arrival counter only grows (the host zeroes it before
every launch); a CTA at its barrier number g adds one to the counter and
waits until the counter reaches (g + 1) * nblocks.  The model runs n CTAs
through B barriers over every interleaving of their atomic steps (an arrival,
or a poll that passes or fails) and checks:

- safety: a CTA passes barrier g only after every CTA has arrived at it;
- progress: from every reachable state every CTA can still finish, so no
  interleaving deadlocks;
- the failure-detection arrangement (the barrier waits for nblocks + 1
  arrivals): no CTA ever passes the first barrier, so only the bounded wait
  ends the kernel, which then reports the timeout.

The GPU kernels are checked against the oracle in ``tests/test_gpu_routines.py``
and the timeout paths in ``tests/test_gpu_failures.py``.
"""
from collections import deque

import pytest

ARRIVE, WAIT = 0, 1


def explore(n, B, nblocks):
    """All reachable states (phases, modes, count) of n CTAs and B barriers;
    returns (states, edges, violations)."""
    start = (tuple([0] * n), tuple([ARRIVE] * n), 0)
    seen = {start}
    edges = {}
    violations = []
    q = deque([start])
    while q:
        st = q.popleft()
        ph, md, cnt = st
        nxt = []
        for i in range(n):
            if ph[i] == B:
                continue
            if md[i] == ARRIVE:
                m = list(md)
                m[i] = WAIT
                nxt.append((ph, tuple(m), cnt + 1))
            elif cnt >= (ph[i] + 1) * nblocks:
                g = ph[i]
                # safety: every CTA arrived at barrier g
                for j in range(n):
                    if not (ph[j] > g or (ph[j] == g and md[j] == WAIT)):
                        violations.append((st, i, j))
                p, m = list(ph), list(md)
                p[i] += 1
                m[i] = ARRIVE
                nxt.append((tuple(p), tuple(m), cnt))
            # a failed poll leaves the state as it is
        edges[st] = nxt
        for s2 in nxt:
            if s2 not in seen:
                seen.add(s2)
                q.append(s2)
    return seen, edges, violations


def can_finish(states, edges, B):
    """states from which the all-done state is reachable"""
    done = {s for s in states if all(p == B for p in s[0])}
    rev = {}
    for s, ns in edges.items():
        for t in ns:
            rev.setdefault(t, []).append(s)
    good, q = set(done), deque(done)
    while q:
        t = q.popleft()
        for s in rev.get(t, ()):
            if s not in good:
                good.add(s)
                q.append(s)
    return good


@pytest.mark.parametrize("n,B", [(2, 4), (3, 3), (4, 2)])
def test_barrier_is_safe_and_never_deadlocks(n, B):
    states, edges, violations = explore(n, B, n)
    assert not violations, violations[:3]
    good = can_finish(states, edges, B)
    assert good == states  # every interleaving can still complete
    assert any(all(p == B for p in s[0]) and s[2] == n * B for s in states)


@pytest.mark.parametrize("n", [2, 3])
def test_one_arrival_too_many_never_releases(n):
    """nblocks = n + 1, as the failure-detection test arms it: every CTA
    arrives and then only polls; nothing passes the first barrier."""
    states, edges, violations = explore(n, 2, n + 1)
    assert not violations
    assert all(all(p == 0 for p in s[0]) for s in states)
    stuck = (tuple([0] * n), tuple([WAIT] * n), n)
    assert stuck in states and edges[stuck] == []
