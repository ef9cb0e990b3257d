"""CPU model of the tensor-core kernel's operand-slot handoff (csrc/kernels_tc.cu,
tc_grm_kernel): the MMA warp waits on named barrier 1 + ab/hb once per batch of hb
sub-stages, and the two unpack groups take alternate batches, arriving on the same
barrier after filling the batch's slots.  A mismatch in the sequence of barriers, slots
or ring positions between the two sides would leave a bar.sync waiting forever on the
GPU, so both loops are restated here, step for step, and compared for every ring shape
the host accepts (launch_tc: hb in {1, 2}, sa a multiple of 2 hb, sl >= 2, sub in
{1, 2, 4})."""
import pytest


def mma_side(nk, sub, sl, sa, hb):
    t = s = ab = k = 0
    out = []
    while k < nk:
        bar, batch, j = 1 + (ab >> (hb - 1)), [], 0
        while j < hb and k < nk:
            batch.append((k, s, t, ab))
            t += 1
            if t == sub:
                t, s = 0, (s + 1) % sl
            ab = (ab + 1) % sa
            j, k = j + 1, k + 1
        out.append((bar, batch))
    return out


def unpack_side(nk, sub, sl, sa, hb, grp):
    st = dict(t=0, s=0, ab=0, ph_l=0, ph_a=0)

    def step():
        st["t"] += 1
        if st["t"] == sub:
            st["t"] = 0
            st["s"] += 1
            if st["s"] == sl:
                st["s"], st["ph_l"] = 0, st["ph_l"] ^ 1
        st["ab"] += 1
        if st["ab"] == sa:
            st["ab"], st["ph_a"] = 0, st["ph_a"] ^ 1

    for _ in range(grp * hb):
        step()
    out, kb = [], grp * hb
    while kb < nk:
        bar, batch = 1 + (st["ab"] >> (hb - 1)), []
        for j in range(hb):
            k = kb + j
            if k < nk:
                # the incrementally kept positions and mbarrier parities equal the
                # closed forms the waits rely on
                assert st["t"] == k % sub and st["s"] == (k // sub) % sl
                assert st["ph_l"] == ((k // sub) // sl) & 1
                assert st["ab"] == k % sa and st["ph_a"] == (k // sa) & 1
                batch.append((k, st["s"], st["t"], st["ab"]))
            step()
        out.append((bar, batch))
        for _ in range(hb):
            step()
        kb += 2 * hb
    return out


@pytest.mark.parametrize("sa,hb", [(2, 1), (4, 1), (6, 1), (4, 2)])
def test_both_sides_take_the_same_handoffs(sa, hb):
    for nk in list(range(1, 40)) + [141, 1164, 1172, 1564]:
        for sub in (1, 2, 4):
            for sl in (2, 3, 5, 8, 24):
                mma = mma_side(nk, sub, sl, sa, hb)
                g0 = unpack_side(nk, sub, sl, sa, hb, 0)
                g1 = unpack_side(nk, sub, sl, sa, hb, 1)
                merged = []
                for i in range(max(len(g0), len(g1))):
                    merged += g0[i:i + 1] + g1[i:i + 1]
                assert merged == mma, (nk, sub, sl, sa, hb)
                # barrier ids stay within the sa / hb the kernel initialises, and a
                # barrier is always reused by the same unpack group (one use ahead at
                # most, held by the slot-reuse wait)
                for i, (bar, _) in enumerate(mma):
                    assert 1 <= bar <= sa // hb
                    if i + 2 < len(mma) and sa // hb == 2:
                        assert mma[i + 2][0] == bar


def producer_side(nk, sub, sl, abort_at):
    """The producer's loop with the slot-reuse wait giving up at load stage abort_at
    (no abort when abort_at >= the stage count), then its drain: the (slot, parity)
    pairs of FULL it waits on before the CTA exits."""
    n_load = (nk + sub - 1) // sub
    S = ph = issued = 0
    for J in range(n_load):
        if J >= sl and J >= abort_at:
            break  # mbar_wait_sleep(LDONE) gave up
        assert S == J % sl and ph == (J // sl) & 1
        issued = J + 1
        S += 1
        if S == sl:
            S, ph = 0, ph ^ 1
    drain = [(J, J % sl, (J // sl) & 1) for J in range(max(0, issued - sl), issued)]
    return n_load, issued, drain


@pytest.mark.parametrize("sub", [1, 2, 4])
@pytest.mark.parametrize("sl", [2, 3, 5, 24])
def test_producer_drain_covers_every_copy_in_flight(sub, sl):
    for nk in list(range(1, 30)) + [141, 1564]:
        n_load = (nk + sub - 1) // sub
        for abort_at in sorted({0, 1, sl - 1, sl, sl + 1, 2 * sl, n_load - 1, n_load, 10 ** 9}):
            n, issued, drain = producer_side(nk, sub, sl, abort_at)
            if abort_at >= n:
                assert issued == n  # no abort: every stage issued
            # stage J was issued only after stage J - sl was consumed (its LDONE phase),
            # so the stages not in the drain list are complete; the drain waits on
            # distinct slots, each at the parity of its one outstanding phase
            consumed = set(range(0, max(0, issued - sl)))
            drained = {J for J, _, _ in drain}
            assert consumed | drained == set(range(issued))
            assert len({slot for _, slot, _ in drain}) == len(drain) <= sl
            for J, slot, par in drain:
                assert slot == J % sl and par == (J // sl) & 1


def merged_unpack_waits(nk, sl, grp):
    """The unpack loop of the merged mode (two sub-stages per batch and per load stage):
    at the start of each of the group's batches, the LDONE slot and parity it waits on
    for its operand slots (computed as the kernel does, from the current ring position)."""
    st = dict(t=0, s=0, ph_l=0)

    def step():
        st["t"] += 1
        if st["t"] == 2:
            st["t"] = 0
            st["s"] += 1
            if st["s"] == sl:
                st["s"], st["ph_l"] = 0, st["ph_l"] ^ 1

    for _ in range(grp * 2):
        step()
    out, kb = [], grp * 2
    while kb < nk:
        assert st["t"] == 0
        if kb >= 4:
            s, ph = st["s"], st["ph_l"]
            out.append((kb // 2, s - 2 if s >= 2 else s - 2 + sl, ph if s >= 2 else ph ^ 1))
        for _ in range(4):  # this batch and the other group's
            step()
        kb += 4
    return out


def merged_mma_commits(nk, sl):
    """The MMA warp's commits in the merged mode: (load stage, LDONE slot) in order."""
    t = s = 0
    out = []
    for k in range(nk):
        if t == 1 or k == nk - 1:
            out.append((k // 2, s))
        t += 1
        if t == 2:
            t, s = 0, (s + 1) % sl
    return out


@pytest.mark.parametrize("sl", [3, 4, 5, 24])
def test_merged_batches_wait_on_the_commit_of_their_previous_batch(sl):
    for nk in list(range(1, 40)) + [1164, 1565]:
        commits = merged_mma_commits(nk, sl)
        # one commit per batch (load stage), on LDONE(stage % sl)
        assert commits == [(b, b % sl) for b in range((nk + 1) // 2)]
        for grp in (0, 1):
            for b, slot, par in merged_unpack_waits(nk, sl, grp):
                # the group's previous batch b - 2, whose commit is phase (b-2)//sl of its slot
                assert slot == (b - 2) % sl and par == ((b - 2) // sl) & 1
                # that phase is still the barrier's latest when the wait runs: the next use
                # of the slot is load stage b - 2 + sl > b, whose MMAs follow batch b's
                assert b - 2 + sl > b
