"""The device mesh generator's index logic, checked on the CPU.

``csrc/mesh_random.cu`` turns draw number g of a host thread's stream into
(system, row, array) without replaying the loop of ``include/util/mesh.hpp:
108-121``: a closed-form row lookup (rows of 4, 5, 6, ..., 6, 5, 4 draws for
n >= 4, a search of the prefix counts below), and per placing thread a cursor
(system, draw in the system, inner index, first element) that moves by a fixed
stride -- 624 C draws for a cluster of C CTAs -- with one wrap at most when the
system is longer than the stride, and a division otherwise.  This restates
those steps in Python and checks them against the reference's draw order,
enumerated row by row, for every system size up to 40 and every stride the
kernel uses; the bit-exact GPU tests check the kernel itself.
"""
import pytest


def draw_order(n):
    """(row, array) of each draw of one system, in the reference's order:
    ds (row > 1), dl (row > 0), d, du (row < n-1), dw (row < n-2, n unsigned), x."""
    out = []
    for r in range(n):
        has = [r > 1, r > 0, True, r < n - 1, (r < n - 2) if n >= 2 else True, True]
        out += [(r, a) for a in range(6) if has[a]]
    return out


def draws_before(r, n):
    ds = r - 2 if r > 2 else 0
    dl = r - 1 if r > 1 else 0
    du = r if r < n - 1 else n - 1
    dw = (r if r < n - 2 else n - 2) if n >= 2 else r
    return 2 * r + ds + dl + du + dw


def row_of(e, n):
    if n >= 4:
        if e < 4:
            return 0, e
        if e < 9:
            return 1, e - 4
        if e < 6 * n - 15:
            r = (e + 3) // 6
            return r, e + 3 - 6 * r
        if e < 6 * n - 10:
            return n - 2, e - (6 * n - 15)
        return n - 1, e - (6 * n - 10)
    a, b = 0, n
    while b - a > 1:
        mid = (a + b) >> 1
        if draws_before(mid, n) <= e:
            a = mid
        else:
            b = mid
    return a, e - draws_before(a, n)


def slot_of(r, k, n):
    has = [r > 1, r > 0, True, r < n - 1, (r < n - 2) if n >= 2 else True, True]
    seen = -1
    for slot in range(6):
        seen += 1 if has[slot] else 0
        if seen == k:
            return slot
    raise AssertionError("draw rank beyond the row")


@pytest.mark.parametrize("n", range(1, 41))
def test_row_lookup_matches_the_draw_order(n):
    order = draw_order(n)
    assert draws_before(n, n) == len(order)
    for e, (r, a) in enumerate(order):
        rr, k = row_of(e, n)
        assert (rr, slot_of(rr, k, n)) == (r, a), (n, e)


class Cursor:
    """The kernel's cursor: draw e of system sys (= i * inner + j) whose first
    element is start = i * inner * n + j."""

    def __init__(self, sys_, e, inner, n):
        self.inner, self.n = inner, n
        self.set(sys_, e)

    def set(self, sys_, e):
        i = sys_ // self.inner
        self.sys, self.e, self.j = sys_, e, sys_ - i * self.inner
        self.start = i * self.inner * self.n + self.j

    def advance(self, step, per):
        self.e += step
        if self.e < per:
            return
        if self.e - per < per:  # one system on, no division
            self.e -= per
            self.sys += 1
            self.start += 1
            self.j += 1
            if self.j == self.inner:
                self.j = 0
                self.start += self.inner * (self.n - 1)
            return
        w = self.e // per
        self.set(self.sys + w, self.e - w * per)


@pytest.mark.parametrize("n,inner,outer", [(1, 3, 2), (2, 5, 3), (3, 1, 7), (4, 6, 2),
                                           (5, 1, 40), (7, 4, 9), (40, 3, 5), (300, 2, 3),
                                           (1000, 1, 4)])
@pytest.mark.parametrize("stride", [624, 1248, 2496, 4992])
def test_cursor_walks_the_stream(n, inner, outer, stride):
    per = draws_before(n, n)
    count = inner * outer
    total = count * per
    order = draw_order(n)
    for lo in (0, 1, count // 2):
        chunk = (count - lo) * per
        for p in (0, 1, stride // 2, stride - 1):
            if p >= chunk:
                continue
            c = Cursor(lo + p // per, p % per, inner, n)
            g = p
            while g < min(chunk, p + 50 * stride):
                sys_ = lo + g // per
                e = g % per
                assert (c.sys, c.e) == (sys_, e)
                i, j = divmod(sys_, inner)
                r, a = order[e]
                rr, k = row_of(c.e, n)
                assert (rr, slot_of(rr, k, n)) == (r, a)
                assert c.start + rr * inner == i * inner * n + j + r * inner
                c.advance(stride, per)
                g += stride
    assert total == count * len(order)
