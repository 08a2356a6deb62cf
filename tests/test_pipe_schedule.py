"""The work order of the pipelined red-black line solve, replayed on the CPU.

The eight passes of a whole-domain red-black solve (2 colours x 4 sweeps) run
as one launch (sweep_rb_pipe_kernel, k_linesolve.cu): work item (pass q, plane
k, line j of colour q mod 2) is handed out by an atomic ticket, decoded from
the ticket by a closed form of the (key, pass, line) order with key
(k - k0) + D q; the item waits until its four neighbouring lines have finished
pass q - 1 and the line itself pass q - 2.  Here the decode is restated and
checked: every line of every pass appears exactly once; every item an item
waits for has a smaller ticket (so the smallest outstanding ticket is always
runnable and the launch cannot deadlock, whatever the residency); and a toy
line update run ticket by ticket, each item reading its neighbours as the flags
allow, gives the same result as the eight passes one after the other.
"""
import numpy as np
import pytest


def pairs_before(s, K, D):
    """(pass, plane) pairs with key below s: sum over q of clamp(s - D q, 0, K)."""
    return sum(min(max(s - D * q, 0), K) for q in range(8))


def decode(tk, J, K, D):
    """Ticket -> (pass, k, j) as the kernel decodes it (k0 = j0 = 1); j > J is
    the missing line of a colour with one line fewer in the plane."""
    half = (J + 1) // 2
    idx, r = divmod(tk, half)
    lo, hi = 0, K - 1 + 7 * D
    while lo < hi:
        mid = (lo + hi + 1) >> 1
        if pairs_before(mid, K, D) <= idx:
            lo = mid
        else:
            hi = mid - 1
    q = ((lo - K + D) // D if lo >= K else 0) + (idx - pairs_before(lo, K, D))
    k = 1 + lo - D * q
    jpar = (((q & 1) - k - 1) % 2 + 2) % 2
    return q, k, 1 + jpar + 2 * r


def deps(q, k, j, J, K):
    """The items (pass, k, j) that item (q, k, j) waits for."""
    out = []
    if q >= 2:
        out.append((q - 2, k, j))
    if q >= 1:
        for kk, jj in ((k, j - 1), (k, j + 1), (k - 1, j), (k + 1, j)):
            if 1 <= kk <= K and 1 <= jj <= J:
                out.append((q - 1, kk, jj))
    return out


@pytest.mark.parametrize("J,K", [(1, 1), (2, 3), (3, 2), (7, 5), (20, 9), (200, 12)])
@pytest.mark.parametrize("D", [2, 8, 16, 32])
def test_every_item_once_and_dependencies_earlier(J, K, D):
    half = (J + 1) // 2
    seen = {}
    for tk in range(half * 8 * K):
        q, k, j = decode(tk, J, K, D)
        assert 0 <= q < 8 and 1 <= k <= K, (tk, q, k)
        if j > J:
            continue
        assert (j + k) % 2 == q % 2, "the line is of the pass's colour"
        assert (q, k, j) not in seen
        seen[(q, k, j)] = tk
    assert len(seen) == 4 * J * K  # every line in each of the 4 passes of its colour
    for item, tk in seen.items():
        for d in deps(*item, J, K):
            assert seen[d] < tk, (d, item)


def test_ticket_order_reproduces_the_passes():
    """A line update that reads the four neighbouring lines (like the TDMA
    right-hand side), run item by item in ticket order where each item reads
    only what its flags guarantee, equals eight sequential colour passes."""
    rng = np.random.default_rng(7)
    J, K, N, D = 9, 6, 5, 8
    phi0 = rng.standard_normal((K + 2, J + 2, N))
    w = rng.uniform(0.1, 0.2, size=(4, K + 2, J + 2, N))

    def update(phi, k, j):
        return (w[0, k, j] * phi[k + 1, j] + w[1, k, j] * phi[k - 1, j] + w[2, k, j] * phi[k, j + 1]
                + w[3, k, j] * phi[k, j - 1] + np.sin(k + 3 * j))

    ref = phi0.copy()
    for q in range(8):
        for k in range(1, K + 1):
            for j in range(1, J + 1):
                if (j + k) % 2 == q % 2:
                    ref[k, j] = update(ref, k, j)
    # ticket order with the flag discipline: an item may run only once its
    # dependencies have run, and reads the current state
    pipe = phi0.copy()
    done = set()
    half = (J + 1) // 2
    for tk in range(half * 8 * K):
        q, k, j = decode(tk, J, K, D)
        if j > J:
            continue
        assert all(d in done for d in deps(q, k, j, J, K))
        pipe[k, j] = update(pipe, k, j)
        done.add((q, k, j))
    assert np.array_equal(pipe, ref)
