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


def mma_commit_log(nk, sub, sl, sa, merged, abort_at):
    """The MMA warp's commits (barrier, slot, phase) in issue order, with no further MMA or
    commit from sub-stage abort_at on, and the (barrier, slot, parity) waits of its exit
    drain, computed as the kernel does from the last committed load and sub-stage."""
    log, phases = [], {}
    t = s = ab = 0
    j_done = k_done = -1
    for k in range(nk):
        if k < abort_at:
            if not merged:
                log.append(("ADONE", ab, phases.setdefault(("A", ab), [0])[0]))
                phases[("A", ab)][0] += 1
                k_done = k
            if t == sub - 1 or k == nk - 1:
                log.append(("LDONE", s, phases.setdefault(("L", s), [0])[0]))
                phases[("L", s)][0] += 1
                j_done = k // sub
        t += 1
        if t == sub:
            t, s = 0, (s + 1) % sl
        ab = (ab + 1) % sa
    drain = []
    for ls in range(sl):
        if j_done >= ls:
            j = j_done - (j_done - ls) % sl
            drain.append(("LDONE", ls, (j // sl) & 1))
    if not merged:
        for a_s in range(sa):
            if k_done >= a_s:
                kk2 = k_done - (k_done - a_s) % sa
                drain.append(("ADONE", a_s, (kk2 // sa) & 1))
    return log, drain


@pytest.mark.parametrize("shape", [(1, 2, 2, False), (2, 5, 4, False), (4, 3, 6, False),
                                   (1, 24, 2, False), (2, 3, 4, True), (2, 5, 4, True),
                                   (2, 24, 4, True)])
def test_exit_drain_waits_on_the_last_commit_of_every_barrier(shape):
    # a commit's mbarrier arrival lands when its MMAs complete, in no set order with the
    # final ACCF commit: the exit drain must wait on the newest phase of every barrier
    # that received a commit, so that no arrival is still in flight when the CTA exits
    sub, sl, sa, merged = shape
    for nk in list(range(1, 30)) + [141, 1164, 1565]:
        for abort_at in sorted({0, 1, 2, nk // 2, nk - 1, nk}):
            log, drain = mma_commit_log(nk, sub, sl, sa, merged, abort_at)
            last = {}
            for bar, slot, phase in log:
                last[(bar, slot)] = phase
            assert sorted((b, sl_, p) for b, sl_, p in drain) == \
                sorted((b, sl_, ph & 1) for (b, sl_), ph in last.items())


def full_waits(nk, sub, sl, sa, hb, merged, grp, slot_wait_first=True):
    """For each sub-stage k of unpack group grp: (k, load stage J, the load stages known
    to have landed when the group waits on FULL(J % sl)).  Known: the group's own earlier
    loads, and — once its slot-reuse wait returned — every load up to the last sub-stage
    the MMA warp has taken (it takes a sub-stage only after its group saw the codes
    land).  With slot_wait_first=False the wait on the codes comes first, as it did before
    (then only the previous batch's slot wait counts)."""
    out, own = [], set()
    kb = grp * hb
    last_taken = -1
    while kb < nk:
        for j in range(hb):
            k = kb + j
            if k >= nk:
                break
            if merged:
                taken = 2 * (kb // 2 - 2) + 1 if (j == 0 and kb >= 2 * hb) else None
            else:
                taken = k - sa if k >= sa else None
            if slot_wait_first and taken is not None:
                last_taken = max(last_taken, taken)
            known = own | {x // sub for x in range(last_taken + 1)}
            out.append((k, k // sub, known))
            own.add(k // sub)
            if not slot_wait_first and taken is not None:
                last_taken = max(last_taken, taken)
        kb += 2 * hb
    return out


def accepted_shapes():
    for sub in (1, 2, 4):
        for sl in (2, 3, 4, 5, 8, 24):
            for sa in (2, 4, 6):
                for hb in (1, 2):
                    if sa % (2 * hb) == 0 and (sl - 1) * sub + 1 >= sa:  # launch_tc's rule
                        yield sub, sl, sa, hb, False
    for sl in (3, 4, 5, 24):
        yield 2, sl, 4, 2, True


def test_codes_wait_never_reads_a_parity_a_phase_early():
    # A group waits on FULL(s) by parity; if the load slot's previous load (J - sl) were
    # still landing, the barrier's parity would already read as load J's and the group
    # would unpack codes that are still being written.  With the slot-reuse wait first,
    # that previous load is always known to have landed, for every accepted shape.
    for sub, sl, sa, hb, merged in accepted_shapes():
        for nk in list(range(1, 48)) + [141, 1165, 1564]:
            for grp in (0, 1):
                for k, J, known in full_waits(nk, sub, sl, sa, hb, merged, grp):
                    assert J - sl < 0 or (J - sl) in known, (sub, sl, sa, hb, merged, nk, k)


def test_the_earlier_wait_order_could_read_a_phase_early():
    # the merged batches with a three-stage ring (pass B at 42 columns): waiting on the
    # codes before the slot left load stage b - 3 unknown at batch b
    bad = [(k, J) for k, J, known in full_waits(64, 2, 3, 4, 2, True, 1, slot_wait_first=False)
           if J - 3 >= 0 and (J - 3) not in known]
    assert bad
