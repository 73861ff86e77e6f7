"""The batched march's bulk-copy ring schedule, restated on the host and checked exhaustively.

The solve passes of `march_sum_impl.cuh` stream the rows of a tile in blocks
of kRB rows through a ring of kNB blocks (`ring_issue`, `solve_iters`,
`solve_blocks`, `sum_pass`).  This restates their arithmetic - the memory rows
each block's tensor copies cover, the row each iteration reads from a block,
the ring slot and mbarrier parity of each block, and the split of a pass into
checked iterations and unchecked whole blocks - and checks, for every column
height and shallowest ray up to a few hundred rows, that:

* every stream iteration reads exactly the row it processes (and its
  elimination row, two behind the stream; one in the residual pass);
* the checked ranges and the unchecked blocks cover the pass once, and every
  row of an unchecked block is interior to every ray of the warp and past
  every first back-substitution row;
* every block is issued once, before the iteration that first reads it, into
  a slot whose previous block has been consumed, and is waited on with the
  parity of its own use of the slot.
"""
import pytest

KRB, KNB, KU = 8, 2, 2
DOWN, UP = True, False


def row_of(down, span, k):
    return k if down else span - 1 - k


def block_rows(down, span, b, elim_shift=0):
    """First memory row of block b's copies (ring_issue: lo, or lm = lo + shift)."""
    lo = b * KRB if down else span - KRB - b * KRB
    return lo + elim_shift


def read_pos(down, k):
    """Row of its block that iteration k reads (load_row index)."""
    jk = k % KRB
    return jk if down else KRB - 1 - jk


def steady_blocks(down, span, nzmin):
    """sum_pass: unchecked whole blocks [b_lo, b_hi) and the iteration bounds around them."""
    lb = 3 if down else span + 1 - nzmin
    ub = nzmin + 1 - KU if down else span - KU - 1
    b_lo = (max(lb, 0) + KRB - 1) // KRB
    b_hi = max(b_lo, int((ub + KU) / KRB))  # C++ division truncates toward zero
    k_lo, k_hi = min(span, b_lo * KRB), min(span, b_hi * KRB)
    return k_lo, k_hi


def row_ok_unchecked(down, r, nz_list):
    """The conditions solve_row / refine_row drop when CHECK is false, for every ray."""
    for nz in nz_list:
        if not (1 <= r <= nz):
            return False
        if down and (r < 3 or r == 1):           # elimination row m = r - 2 >= 1; not the first row
            return False
        if not down and (r + 2 > nz or r == nz):  # m = r + 2 <= nz; not the first row (nz)
            return False
    return True


@pytest.mark.parametrize("down", [DOWN, UP])
def test_rows_read_match_rows_processed(down):
    for rows in range(2, 150):
        span = (rows + KU - 1) // KU * KU
        for k in range(span):
            b = k // KRB
            r = row_of(down, span, k)
            assert block_rows(down, span, b) + read_pos(down, k) == r
            shift = -2 if down else 2
            assert block_rows(down, span, b, shift) + read_pos(down, k) == r + shift
            # the refined form's residual pass (UP) eliminates one row behind
            if not down:
                assert block_rows(down, span, b, 1) + read_pos(down, k) == r + 1


@pytest.mark.parametrize("down", [DOWN, UP])
def test_unchecked_blocks_cover_only_safe_rows(down):
    for nzmax in range(1, 130):
        rows = nzmax + 2
        span = (rows + KU - 1) // KU * KU
        for nzmin in range(1, nzmax + 1):
            k_lo, k_hi = steady_blocks(down, span, nzmin)
            assert 0 <= k_lo <= k_hi <= span
            assert k_lo % KRB == 0 or k_lo == span
            assert k_hi % KRB == 0 or k_hi == span
            for k in range(k_lo, k_hi):
                r = row_of(down, span, k)
                assert row_ok_unchecked(down, r, [nzmin, nzmax]), (down, span, nzmin, k, r)


@pytest.mark.parametrize("down", [DOWN, UP])
def test_ring_issue_wait_order(down):
    for span in range(2, 120, 2):
        nblk = (span + KRB - 1) // KRB
        for seq0 in range(0, 5):
            issued = {}          # block -> (slot, time)
            consumed_upto = -1   # last block whose rows were all used
            slot_busy = {}       # slot -> block occupying it
            t = 0
            for b in range(min(KNB, nblk)):       # pass prologue
                s = (seq0 + b) % KNB
                assert s not in slot_busy
                slot_busy[s] = b
                issued[b] = (s, t)
                t += 1
            for k in range(0, span, KU):
                b, jk = k // KRB, k % KRB
                q = seq0 + b
                slot, parity = q % KNB, (q // KNB) & 1
                if jk == 0:  # wait: the block must have been issued into this slot
                    assert b in issued and issued[b][0] == slot and slot_busy[slot] == b
                    # its use of the slot is the (q // KNB)-th: parity alternates per use
                    assert parity == ((seq0 + b) // KNB) % 2
                t += 1
                if jk + KU == KRB or k + KU >= span:   # rows of block b used
                    consumed_upto = b
                if jk + KU == KRB and b + KNB < nblk:   # ring_refill after the last rows
                    assert consumed_upto == b and slot_busy[slot] == b
                    slot_busy[slot] = b + KNB
                    issued[b + KNB] = (slot, t)
                    t += 1
            assert sorted(issued) == list(range(nblk))  # every block issued once
