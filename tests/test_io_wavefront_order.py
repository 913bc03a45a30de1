"""The launch order of the overlapped time_step (Impl::time_step_io in
porturb_b200/csrc/impl.cuh), restated and checked on the CPU: every stage of
every chunk reads the versions of the state buffers that the serial order
(load_state, then the stages of advance one after the other) gives it, and
leaves the same final versions.

Model: chunk c of ZT_Z levels; op (0, c) brings chunk c in (writes s0[c]);
op (g, c), g = 1 .. 3 nsteps, is stage g on chunk c: stage m = (g-1) % 3
reads s0 / s1 / s2 at chunks c-1, c, c+1 (the z stencils reach 5 levels into
each neighbour; the x/y stencils stay in the level) and, for m = 1, 2, s0 at
chunk c (the step's initial state), and writes s1 / s2 / s0 at chunk c.  The
x/y tendency buffer is written and read inside one op.  The wavefront order:
diagonals w = g + c, each in increasing g.
"""
import pytest


def wavefront(nch, last):
    order = []
    for w in range(last + nch):
        for g in range(max(0, w - (nch - 1)), min(w, last) + 1):
            order.append((g, w - g))
    return order


def serial(nch, last):
    return [(0, c) for c in range(nch)] + [(g, c) for g in range(1, last + 1) for c in range(nch)]


def accesses(g, c, nch):
    if g == 0:
        return [], [("s0", c)]
    m = (g - 1) % 3
    reads = [(("s0", "s1", "s2")[m], cc) for cc in (c - 1, c, c + 1) if 0 <= cc < nch]
    if m in (1, 2):
        reads.append(("s0", c))
    return reads, [(("s1", "s2", "s0")[m], c)]


def versions(order, nch):
    ver, seen = {}, {}
    for g, c in order:
        reads, writes = accesses(g, c, nch)
        seen[(g, c)] = tuple(ver.get(x) for x in reads)
        for x in writes:
            ver[x] = (g, c)
    return seen, ver


@pytest.mark.parametrize("nsteps", [1, 2, 3, 4, 10])
@pytest.mark.parametrize("nch", [2, 3, 4, 8, 9])
def test_wavefront_reads_the_serial_versions(nch, nsteps):
    last = 3 * nsteps
    w, s = wavefront(nch, last), serial(nch, last)
    assert sorted(w) == sorted(s) and len(set(w)) == len(w)
    assert versions(w, nch) == versions(s, nch)


def test_a_wrong_order_is_caught():
    """Swapping the order inside a diagonal (decreasing g) breaks the check."""
    nch, last = 4, 6
    bad = []
    for w in range(last + nch):
        for g in reversed(range(max(0, w - (nch - 1)), min(w, last) + 1)):
            bad.append((g, w - g))
    assert versions(bad, nch) != versions(serial(nch, last), nch)
