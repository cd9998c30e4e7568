"""Integer model of where the MSM combine writes each work item's result
(fb_part_index and fb_fill_unused_slots, csrc/zg_kernels.cuh).

The AMT tree kernel sums, per node, the part slots of that node's 1024-point
column chunks (R slots per coset and line). Wide items are 1024-bucket blocks
of units; a merged class (mlog = 1) has half as many items per line as slots
and fills the rest with the identity. This test restates the index arithmetic
and checks, for the classes of the 1024-column shapes, that every slot of a
class's lines is written exactly once, that item results land in the slots of
their own unit (so of their own node), and that the block weight the combine
applies (1024 blk) matches the bucket range of the item.
"""
import pytest

LC = 10


def part_index(lr_items, lines, l0, L, hi_last, bpu_log, mlog, v):
    l, g = v % lines, v // lines
    nch = 1 << lr_items
    line = L - 1 if (hi_last and l == lines - 1) else l0 + l
    b, bmask = g % nch, (1 << bpu_log) - 1
    slot = ((b >> bpu_log) << (bpu_log + mlog)) | (b & bmask)
    return ((g // nch) * L + line) * (nch << mlog) + slot


def classes(lr):
    """The wide classes plan_wide_classes builds at 1024 columns: (ulog, mlog,
    l0, nl, hi_last), largest unit first (unit log = min(16, log2 node))."""
    out, nxt = [], 0
    for u in range(16, 10, -1):
        ulog = min(u, 15)
        nq = 0
        while nxt + nq < lr and min(16, lr + 9 - (nxt + nq)) == u:
            nq += 1
        hi = min(16, lr + 10) == u
        if not nq and not hi:
            continue
        out.append((ulog, u - ulog, nxt, nq + (1 if hi else 0), 1 if hi else 0))
        nxt += nq
    return out


@pytest.mark.parametrize("lr", [5, 6, 7, 10])
def test_every_slot_written_once(lr):
    R, L = 1 << lr, lr + 2
    seen = {}
    for ulog, mlog, l0, nl, hi_last in classes(lr):
        bl = ulog - 10
        lr_items = lr - mlog
        for v in range(3 * (R >> mlog) * nl):
            idx = part_index(lr_items, nl, l0, L, hi_last, bl, mlog, v)
            writes = [idx] + [idx + (t << bl) for t in range(1, 1 << mlog)]
            for k, w in enumerate(writes):
                assert w not in seen, (lr, ulog, mlog, v)
                seen[w] = (ulog, mlog, v, k)
            # the item's slot lies in its unit's 2^(bl + mlog) slots, unit =
            # (v / lines mod items per line) >> bl
            g = v // nl
            b = g % (1 << lr_items)
            unit_slots = 1 << (bl + mlog)
            assert (idx % R) // unit_slots == b >> bl
            # block weight: the item's buckets are 1024 blk + 1 .. 1024 blk + 1024
            assert (g & ((1 << bl) - 1)) == b & ((1 << bl) - 1)
    wide_lines = sum(c[3] for c in classes(lr))
    assert len(seen) == 3 * wide_lines * R


def test_merged_class_at_production_shape():
    cls = classes(10)
    assert cls[0] == (15, 1, 0, 5, 1)  # quotient lines 0-3 and the high line, 2^16-point units
    assert [c[:2] for c in cls[1:]] == [(15, 0), (14, 0), (13, 0), (12, 0), (11, 0)]
    assert sum(c[3] for c in cls) == 10  # every line but quotient 9 and the basis
