"""The device schedule built with a symbolic analysis, checked on the CPU through the read-only schedule fields of
amp_plan_array: every supernode's work is listed exactly once, and every task waits only for tasks listed before it.

The solve sweeps are persistent kernels whose CTAs take tasks in list order and wait (bounded) for the tasks they
depend on: a forward task for its supernode's children (their pass-up vectors) and for its own supernode's earlier
pivot blocks, a backward task for its parent's pivot blocks and its own supernode's later blocks. The order checked
here is what keeps them free of deadlock. The small-front factor's warp classes need each level's m <= 32 fronts
sorted by m, split at m = 16."""
import numpy as np
import pytest

import ampsolve as amp
import workloads as wl

B = 64  # solve block rows
TINY, TINY_MID, WHOLE = 32, 16, 512


class _Pat:
    """A pattern alone (no coordinates): what analyze needs for AMD."""

    def __init__(self, rows):
        n = len(rows)
        self.pat = wl.CsrPattern(n, np.cumsum([0] + [len(r) for r in rows]).astype(np.int32),
                                 np.concatenate([np.asarray(sorted(r), np.int32) for r in rows]) if n else
                                 np.zeros(0, np.int32))
        self.x = self.y = self.z = None


def _dense(n):
    return _Pat([list(range(n)) for _ in range(n)])


def _diagonal(n):
    return _Pat([[i] for i in range(n)])


def _arrow(n):  # every row coupled to the last: a star whose hub is eliminated last
    return _Pat([[i, n - 1] for i in range(n - 1)] + [list(range(n))])


def _cases():
    return [
        ("elastic3d-14-nd3", lambda: wl.elastic3d(14), "nd3"),
        ("poisson2d-40-amd", lambda: wl.poisson2d(40), "amd"),
        ("grid27-11-amd", lambda: wl.grid27(11, 11, 11, sym=True), "amd"),
        ("heat2d-48-nd", lambda: wl.heat2d_lognormal(48, 7, 1), "nd"),
        # edge cases: one supernode of several pivot blocks, only 1 x 1 supernodes, a chain, a hub, one entry
        ("dense-200", lambda: _dense(200), "amd"),
        ("diagonal-100", lambda: _diagonal(100), "amd"),
        ("chain-300", lambda: wl.chain(300), "amd"),
        ("arrow-150", lambda: _arrow(150), "amd"),
        ("one", lambda: _diagonal(1), "amd"),
        # a forest of uneven trees: 12 problems of the batched heat set, block-diagonal, per-matrix AMD orders
        ("heat2d-batch-12", _batch12, "perm"),
    ]


class _Batch:
    def __init__(self, ws):
        import batch

        self.pat, offs, _ = batch.block_diagonal([w.pat for w in ws])
        self.perm = np.concatenate([amp.amdOrder(w.pat) + offs[i] for i, w in enumerate(ws)]).astype(np.int32)
        self.x = self.y = self.z = None


def _batch12():
    return _Batch(wl.heat2d_batch(12))


@pytest.fixture(scope="module", params=_cases(), ids=lambda c: c[0])
def plan(request):
    _, make, ordering = request.param
    w = make()
    kw = {"perm": w.perm} if ordering == "perm" else {"ordering": ordering}
    if ordering in ("nd", "nd3") and w.x is not None:
        kw.update(x=w.x, y=w.y, z=w.z)
    sym = amp.analyze(w.pat, **kw)
    ss = np.asarray(sym.superStart, np.int64)
    ns = len(ss) - 1
    nc = np.diff(ss)
    m = np.diff(np.asarray(sym.Sp, np.int64))[:ns]
    par = np.asarray(sym.superParent)[:ns]
    lp, ls = np.asarray(sym.levelPtr), np.asarray(sym.levelSupernodes)
    level = np.full(ns, -1)
    for L in range(len(lp) - 1):
        level[ls[lp[L]:lp[L + 1]]] = L
    return sym, ns, nc, m, par, level


def test_levels_cover_every_supernode_below_its_parent(plan):
    sym, ns, nc, m, par, level = plan
    assert np.all(level >= 0)
    assert len(sym.levelSupernodes) == ns
    has = par >= 0
    assert np.all(level[has] < level[par[has]])
    assert np.all((m - nc)[~has] == 0) and np.all((m - nc)[has] > 0)


def _walk(tasks, small):
    """(first, last) task index of each supernode, and the work items listed: ('d', s, b), ('b', s, j), ('w', s),
    ('s', s)."""
    first, last, items = {}, {}, []
    for i, (x, y, k, _) in enumerate(tasks.reshape(-1, 4)):
        if k == 2:
            assert 1 <= y <= 4
            sns = [int(v) for v in small[x:x + y]]
            items += [("s", s) for s in sns]
        else:
            sns = [int(x)]
            items.append({0: ("d", x, y), 1: ("b", x, y), 3: ("w", x)}[int(k)])
        for s in sns:
            first.setdefault(s, i)
            last[s] = i
    return first, last, items


def _expected(ns, nc, m, whole):
    out = []
    for s in range(ns):
        if m[s] <= TINY:
            out.append(("s", s))
        elif whole and nc[s] <= B and m[s] <= WHOLE:
            out.append(("w", s))
        else:
            out += [("d", s, b) for b in range((nc[s] + B - 1) // B)]
            out += [("b", s, j) for j in range((m[s] - nc[s] + B - 1) // B)]
    return out


def _key(t):
    return tuple(int(v) for v in t[1:]) + (t[0],)


def _forward_violations(tasks, small, nc, m, par):
    """Tasks that wait for a task listed after them (forward sweep)."""
    ns = len(nc)
    first, last, _ = _walk(tasks, small)
    bad = [("child after parent", s) for s in range(ns) if par[s] >= 0 and not last[s] < first[int(par[s])]]
    pos = {}
    for i, (x, y, k, _) in enumerate(tasks.reshape(-1, 4)):
        if k in (0, 1):
            pos[(int(x), int(k), int(y))] = i
    for s in range(ns):
        d = [pos[(s, 0, b)] for b in range((nc[s] + B - 1) // B) if (s, 0, b) in pos]
        below = [pos[(s, 1, j)] for j in range((m[s] - nc[s] + B - 1) // B) if (s, 1, j) in pos]
        if d != sorted(d) or (d and below and max(d) > min(below)):
            bad.append(("blocks out of order", s))
    return bad


def _backward_violations(tasks, small, nc, par):
    ns = len(nc)
    first, last, _ = _walk(tasks, small)
    bad = [("parent after child", s) for s in range(ns) if par[s] >= 0 and not last[int(par[s])] < first[s]]
    blks = {}
    for (x, y, k, _) in tasks.reshape(-1, 4):
        if k == 0:
            blks.setdefault(int(x), []).append(int(y))
    for s in sorted(blks):
        if blks[s] != sorted(blks[s], reverse=True):
            bad.append(("blocks out of order", s))
    return bad


@pytest.mark.parametrize("field,whole", [("fwdTasks", True), ("fwdTasksMulti", False)])
def test_forward_schedule_covers_and_orders(plan, field, whole):
    sym, ns, nc, m, par, level = plan
    tasks = np.asarray(getattr(sym, field))
    small = np.asarray(sym.solveSmall)
    _, _, items = _walk(tasks, small)
    assert sorted(map(_key, items)) == sorted(map(_key, _expected(ns, nc, m, whole)))  # every piece exactly once
    assert _forward_violations(tasks, small, nc, m, par) == []


def test_backward_schedule_covers_and_orders(plan):
    sym, ns, nc, m, par, level = plan
    tasks = np.asarray(sym.bwdTasks)
    small = np.asarray(sym.solveSmall)
    _, _, items = _walk(tasks, small)
    exp = []
    for s in range(ns):
        exp += [("s", s)] if m[s] <= TINY else [("d", s, b) for b in range((nc[s] + B - 1) // B)]
    assert sorted(map(_key, items)) == sorted(map(_key, exp))
    assert _backward_violations(tasks, small, nc, par) == []


def test_order_checks_catch_a_reordered_schedule(plan):
    # the checks above are not vacuous: the last forward task (a root's) moved to the front, and the first backward
    # task (a root's) moved to the end, are both reported
    sym, ns, nc, m, par, level = plan
    if not (np.any(par >= 0) or (ns and nc.max() > B)):
        pytest.skip("no task waits for another (no supernode has a parent or a second pivot block)")
    small = np.asarray(sym.solveSmall)
    f = np.asarray(sym.fwdTasks).reshape(-1, 4)
    if len(f) > 1 and not (f[-1, 2] == 2 and f[0, 2] == 2):
        moved = np.concatenate([f[-1:], f[:-1]]).reshape(-1)
        assert _forward_violations(moved, small, nc, m, par)
    b = np.asarray(sym.bwdTasks).reshape(-1, 4)
    if len(b) > 1 and ns > 1:
        moved = np.concatenate([b[1:], b[:1]]).reshape(-1)
        assert _backward_violations(moved, small, nc, par)


def test_tiny_front_classes(plan):
    sym, ns, nc, m, par, level = plan
    tiny = np.asarray(sym.tinyFronts)
    tp, tm = np.asarray(sym.tinyPtr), np.asarray(sym.tinyMid)
    assert len(tp) == len(tm) + 1 == len(sym.levelPtr)
    assert sorted(tiny.tolist()) == [s for s in range(ns) if m[s] <= TINY]
    for L in range(len(tm)):
        sl = tiny[tp[L]:tp[L + 1]]
        assert np.all(level[sl] == L)
        ms = m[sl]
        assert np.all(np.diff(ms) >= 0)
        k = tm[L] - tp[L]
        assert 0 <= k <= len(sl)
        assert np.all(ms[:k] <= TINY_MID) and np.all(ms[k:] > TINY_MID)


# ---- schedule parameters (the autotuner's search space) -------------------------------------------------------------
@pytest.mark.parametrize("gb,sf", [(1, 32), (2, 64), (8, 128), (16, 96)])
def test_schedule_parameters_leave_the_symbolic_analysis_unchanged(gb, sf):
    w = wl.elastic3d(8)
    base = amp.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z)
    tuned = amp.analyze(w.pat, ordering="nd3", x=w.x, y=w.y, z=w.z, groupBlocks=gb, smallFront=sf)
    for f in ("perm", "parent", "superStart", "Sp", "Si", "Lxp", "fwdTasks", "bwdTasks"):
        assert np.array_equal(getattr(base, f), getattr(tuned, f)), f
    # fronts factored whole by one warp (m <= 32) do not depend on the whole-front CTA cut-off either
    assert np.array_equal(base.tinyFronts, tuned.tinyFronts)


@pytest.mark.parametrize("gb,sf,dfr", [(17, 128, 0), (4, 129, 0), (4, 20, 0), (4, 128, 9)])
def test_schedule_parameters_out_of_range_are_rejected(gb, sf, dfr):
    w = wl.poisson2d(8)
    with pytest.raises(amp.AmpError, match="schedule parameters out of range"):
        amp.analyze(w.pat, groupBlocks=gb, smallFront=sf, deferUpdates=dfr)
