"""The ghost index map the EMF kernel reads the CT flux arrays through
(bc_map in csrc/cell_ops.cuh) against the ghost fill it stands in for
(op_bound_column, the reference's in-place statement order,
src/bound.cpp:19-107): after the fill, A[s] == A[bc_map(s)] for every padded
index s in [1, n+4] on an axis of n >= 2 active cells, periodic or open.
The map is restated here from its definition; the GPU ensemble tests check
the kernels that use it bitwise against runs that fill the ghosts."""
import pytest


def bc_map(s, n, periodic):
    if s < 3:
        return s + n if periodic else 3
    if s > n + 2:
        return s - n if periodic else n + 2
    return s


def ghost_fill(a, n, periodic):
    """The fill in its statement order, ghosts holding stale values."""
    if periodic:
        a[0] = a[n]; a[1] = a[n + 1]; a[2] = a[n + 2]
        a[n + 3] = a[3]; a[n + 4] = a[4]; a[n + 5] = a[5]
    else:
        lo = a[3]
        a[0] = a[1] = a[2] = lo
        hi = a[n + 2]
        a[n + 3] = a[n + 4] = a[n + 5] = hi


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("n", [2, 3, 4, 5, 8, 31, 256])
def test_map_reads_what_the_fill_leaves(n, periodic):
    before = [1000 + s for s in range(n + 6)]   # distinct values; ghosts stale
    after = list(before)
    ghost_fill(after, n, periodic)
    for s in range(1, n + 5):
        m = bc_map(s, n, periodic)
        assert 3 <= m <= n + 2, (s, m)
        assert after[s] == before[m], (n, periodic, s)
