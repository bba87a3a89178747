"""The multigrid cycles' event order (fb_multigrid_cycle_events, host only) against a restatement of
the reference's cycle drivers: MultiGrid::_apply_cycle_v/_f/_w with _apply_rest, _apply_prol and
_apply_smooth_peak (kernel/solver/multigrid.hpp:1335-1440, 1632-1700, 1713-1990), for every cycle,
both kinds of coarse-grid correction and 2..10 levels.  The GPU tests check the results of the same
sequences bitwise against the reference binary at levels 5 and 6; this pins the order for deeper
hierarchies (the W cycle's 2^(levels-1) coarse solves)."""
import pytest


def reference_cycle(cycle, nl, cgc):
    ev = []
    last = nl - 1

    def rest(cur, smooth):
        # _apply_rest(cur_lvl, cur_smooth): smooth (and form the defect) unless this is the level the
        # restriction starts from without smoothing, then restrict
        for i in range(cur, last):
            if smooth or i > cur:
                ev.extend([("pre", i), ("def", i)])
            ev.append(("res", i))

    def prol(cur, smooth, top=False):
        # _apply_prol(cur_lvl, cur_smooth): prolongate, then post-smooth unless this is the peak level
        for i in range(last - 1, cur - 1, -1):
            ev.append(("proc" if cgc else "pro", i))
            if smooth or i > cur:
                name = ("postc" if cgc else "post") + ("_top" if top and i == 0 else "")
                ev.append((name, i))

    def peak(lvl):
        # _apply_smooth_peak: defect, peak smoother as a correction, new defect
        ev.extend([("post", lvl), ("def", lvl)])

    def coarse():
        ev.append(("crs", last))

    if cycle == "V":
        rest(0, True)
        coarse()
        prol(0, True, top=True)
    elif cycle == "F":
        rest(0, True)
        for pk in range(last - 1, 0, -1):
            coarse()
            prol(pk, False)
            peak(pk)
            rest(pk, False)
        coarse()
        prol(0, True, top=True)
    else:
        rest(0, True)
        coarse()
        counters = [0] * (last + 1)
        for _ in range(1, 1 << last):
            pk = last
            while pk > 0:
                pk -= 1
                if counters[pk] == 0:
                    break
            for i in range(last - 1, pk, -1):
                counters[i] = 0
            counters[pk] += 1
            prol(pk, False)
            peak(pk)
            rest(pk, False)
            coarse()
        assert all(c == 1 for c in counters[:last])
        prol(0, True, top=True)
    return ev


@pytest.mark.parametrize("cycle", ["V", "F", "W"])
@pytest.mark.parametrize("cgc", ["Fixed", "MinEnergy", "MinDefect"])
def test_cycle_events_match_reference_order(featlib, cycle, cgc):
    fb = featlib
    for nl in range(2, 11):
        got = fb.cycle_events(cycle, nl, cgc)
        assert got == reference_cycle(cycle, nl, cgc != "Fixed"), (cycle, cgc, nl)


def test_cycle_event_counts(featlib):
    fb = featlib
    # V(2,2) over L levels: (L-1) x (pre, def, res) + coarse + (L-1) x (pro, post)
    assert len(fb.cycle_events("V", 10)) == 9 * 3 + 1 + 9 * 2
    # W: 2^(L-1) coarse solves
    assert sum(1 for e in fb.cycle_events("W", 10) if e[0] == "crs") == 2 ** 9
    # F: L-1 coarse solves
    assert sum(1 for e in fb.cycle_events("F", 10) if e[0] == "crs") == 9
    with pytest.raises(fb.FeatB200Error):
        fb.cycle_events("V", 1)
