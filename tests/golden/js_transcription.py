"""A line-by-line Python transcription of the reference's symbolic phase, used only to derive the ordering goldens.

The reference is JavaScript and no JS engine exists here, so this file restates, statement by statement and with the
JS names, the functions that decide the orderings and the supernode partition:

  amdOrder   packages/core/src/la/sparse.mjs:297-592
  ndOrder    packages/core/src/la/sparse.mjs:231-283
  nd3Order   packages/core/src/la/order3d.mjs:11-77 (subPattern, leafOrder, rec)
  postorder, etreeOf, analyze (perm, parent, colCount, amalgamation, row structures)
             packages/core/src/la/sparse.mjs:597-902

It is written separately from the C oracle (oracle/amp_oracle.c) and from the product (csrc/host/symbolic.cpp), from
the JS text alone, so a disagreement points at a transcription error in one of the three. JS semantics that matter
are emulated explicitly: Int32Array reads out of range (including negative indices) give undefined and writes out of
range are ignored (amdOrder's postorder reads head[Cp[n]] with Cp[n] = -1); stores convert with ToInt32 (undefined
and NaN become 0); Array.prototype.sort is stable; typed-array sort is numeric; numbers are IEEE doubles.

Test infrastructure only: tests/golden/make_ordering_golden.py runs it to write the committed fixtures.
"""
from __future__ import annotations

import math


def to_int32(v) -> int:
    if v is None or (isinstance(v, float) and (math.isnan(v) or math.isinf(v))):
        return 0
    v = int(v)  # truncation toward zero, as ToInt32
    v &= 0xFFFFFFFF
    return v - (1 << 32) if v >= (1 << 31) else v


class I32:
    """Int32Array: reads outside [0, length) are undefined (None), writes there are ignored."""

    def __init__(self, n, fill=0):
        self.a = [to_int32(fill)] * int(n)

    @staticmethod
    def of(vals):
        r = I32(0)
        r.a = [to_int32(v) for v in vals]
        return r

    def __len__(self):
        return len(self.a)

    def __getitem__(self, i):
        return self.a[i] if isinstance(i, int) and 0 <= i < len(self.a) else None

    def __setitem__(self, i, v):
        if isinstance(i, int) and 0 <= i < len(self.a):
            self.a[i] = to_int32(v)

    def tolist(self):
        return list(self.a)


def FLIP(i):
    return -i - 2


# ---- amdOrder (sparse.mjs:297-592) ----------------------------------------------------------------------------------
def amdOrder(pat, denseFactor=10):
    n = pat["n"]
    rowptr, colidx = pat["rowptr"], pat["colidx"]
    if n == 0:
        return []
    cnz = 0
    for i in range(n):
        for p in range(rowptr[i], rowptr[i + 1]):
            if colidx[p] != i:
                cnz += 1
    nzmax = cnz + math.floor(cnz / 5) + 2 * n
    Cp = I32(n + 1)
    Ci = I32(nzmax)
    q0 = 0
    for i in range(n):
        Cp[i] = q0
        for p in range(rowptr[i], rowptr[i + 1]):
            if colidx[p] != i:
                Ci[q0] = colidx[p]
                q0 += 1
    Cp[n] = q0
    len_ = I32(n + 1)
    nv = I32(n + 1)
    next_ = I32(n + 1)
    head = I32(n + 1)
    elen = I32(n + 1)
    degree = I32(n + 1)
    w = I32(n + 1)
    hhead = I32(n + 1)
    last = I32(n + 1)
    for k in range(n):
        len_[k] = Cp[k + 1] - Cp[k]
    dense = min(n - 2, max(16, denseFactor * math.sqrt(n)))
    for i in range(n + 1):
        head[i] = -1
        last[i] = -1
        next_[i] = -1
        hhead[i] = -1
        nv[i] = 1
        w[i] = 1
        elen[i] = 0
        degree[i] = len_[i]

    def wclear(mark, lemax):
        if mark < 2 or mark + lemax > 2e9:
            for k in range(n):
                if w[k] != 0:
                    w[k] = 1
            return 2
        return mark

    mark = wclear(0, 0)
    elen[n] = -2
    Cp[n] = -1
    w[n] = 0
    nv[n] = 0
    nel = 0
    for i in range(n):
        d = degree[i]
        if d == 0:
            elen[i] = -2
            nel += 1
            Cp[i] = -1
            w[i] = 0
        elif d > dense:
            nv[i] = 0
            elen[i] = -1
            nel += 1
            Cp[i] = FLIP(n)
            nv[n] = nv[n] + 1
        else:
            if head[d] != -1:
                last[head[d]] = i
            next_[i] = head[d]
            head[d] = i
    mindeg = 0
    lemax = 0
    while nel < n:
        k = -1
        while mindeg < n:
            k = head[mindeg]
            if k != -1:
                break
            mindeg += 1
        if next_[k] != -1:
            last[next_[k]] = -1
        head[mindeg] = next_[k]
        elenk = elen[k]
        nvk = nv[k]
        nel += nvk
        if elenk > 0 and cnz + mindeg >= nzmax:  # garbage collection
            for j in range(n):
                p = Cp[j]
                if p >= 0:
                    Cp[j] = Ci[p]
                    Ci[p] = FLIP(j)
            q = 0
            p = 0
            while p < cnz:
                j = FLIP(Ci[p])
                p += 1
                if j >= 0:
                    Ci[q] = Cp[j]
                    Cp[j] = q
                    q += 1
                    for _k3 in range(len_[j] - 1):
                        Ci[q] = Ci[p]
                        q += 1
                        p += 1
            cnz = q
        # new element Lk
        dk = 0
        nv[k] = -nvk
        p = Cp[k]
        pk1 = p if elenk == 0 else cnz
        pk2 = pk1
        for k1 in range(1, elenk + 2):
            if k1 > elenk:
                e = k
                pj = p
                ln = len_[k] - elenk
            else:
                e = Ci[p]
                p += 1
                pj = Cp[e]
                ln = len_[e]
            for _k2 in range(1, ln + 1):
                i = Ci[pj]
                pj += 1
                nvi = nv[i]
                if nvi <= 0:
                    continue
                dk += nvi
                nv[i] = -nvi
                Ci[pk2] = i
                pk2 += 1
                if next_[i] != -1:
                    last[next_[i]] = last[i]
                if last[i] != -1:
                    next_[last[i]] = next_[i]
                else:
                    head[degree[i]] = next_[i]
            if e != k:
                Cp[e] = FLIP(k)
                w[e] = 0
        if elenk != 0:
            cnz = pk2
        degree[k] = dk
        Cp[k] = pk1
        len_[k] = pk2 - pk1
        elen[k] = -2
        # set differences |Le \ Lk|
        mark = wclear(mark, lemax)
        for pk in range(pk1, pk2):
            i = Ci[pk]
            eln = elen[i]
            if eln <= 0:
                continue
            nvi = -nv[i]
            wnvi = mark - nvi
            q = Cp[i]
            while q <= Cp[i] + eln - 1:
                e = Ci[q]
                if w[e] >= mark:
                    w[e] = w[e] - nvi
                elif w[e] != 0:
                    w[e] = degree[e] + wnvi
                q += 1
        # approximate degree update, element absorption, hashing
        for pk in range(pk1, pk2):
            i = Ci[pk]
            p1 = Cp[i]
            p2 = p1 + elen[i] - 1
            pn = p1
            h = 0
            d = 0
            for q in range(p1, p2 + 1):
                e = Ci[q]
                if w[e] != 0:
                    dext = w[e] - mark
                    if dext > 0:
                        d += dext
                        Ci[pn] = e
                        pn += 1
                        h += e
                    else:
                        Cp[e] = FLIP(k)  # aggressive absorption
                        w[e] = 0
            elen[i] = pn - p1 + 1
            p3 = pn
            p4 = p1 + len_[i]
            for q in range(p2 + 1, p4):
                j = Ci[q]
                nvj = nv[j]
                if nvj <= 0:
                    continue
                d += nvj
                Ci[pn] = j
                pn += 1
                h += j
            if d == 0:  # mass elimination
                Cp[i] = FLIP(k)
                nvi = -nv[i]
                dk -= nvi
                nvk += nvi
                nel += nvi
                nv[i] = 0
                elen[i] = -1
            else:
                degree[i] = min(degree[i], d)
                Ci[pn] = Ci[p3]
                Ci[p3] = Ci[p1]
                Ci[p1] = k
                len_[i] = pn - p1 + 1
                h = math.fmod(-h if h < 0 else h, n)  # JS %: sign of the dividend (non-negative here)
                h = int(h)
                next_[i] = hhead[h]
                hhead[h] = i
                last[i] = h
        degree[k] = dk
        lemax = max(lemax, dk)
        mark = wclear(mark + lemax, lemax)
        # supervariable detection
        for pk in range(pk1, pk2):
            i = Ci[pk]
            if nv[i] >= 0:
                continue
            h = last[i]
            i = hhead[h]
            hhead[h] = -1
            while i != -1 and next_[i] != -1:
                ln = len_[i]
                eln = elen[i]
                for q in range(Cp[i] + 1, Cp[i] + ln):
                    w[Ci[q]] = mark
                jlast = i
                j = next_[i]
                while j != -1:
                    ok = len_[j] == ln and elen[j] == eln
                    q = Cp[j] + 1
                    while ok and q <= Cp[j] + ln - 1:
                        if w[Ci[q]] != mark:
                            ok = False
                        q += 1
                    if ok:
                        Cp[j] = FLIP(i)
                        nv[i] = nv[i] + nv[j]
                        nv[j] = 0
                        elen[j] = -1
                        j = next_[j]
                        next_[jlast] = j
                    else:
                        jlast = j
                        j = next_[j]
                i = next_[i]
                mark += 1
        # finalize Lk
        q = pk1
        for pk in range(pk1, pk2):
            i = Ci[pk]
            nvi = -nv[i]
            if nvi <= 0:
                continue
            nv[i] = nvi
            d = degree[i] + dk - nvi
            d = min(d, n - nel - nvi)
            if head[d] != -1:
                last[head[d]] = i
            next_[i] = head[d]
            last[i] = -1
            head[d] = i
            mindeg = min(mindeg, d)
            degree[i] = d
            Ci[q] = i
            q += 1
        nv[k] = nvk
        len_[k] = q - pk1
        if len_[k] == 0:
            Cp[k] = -1
            w[k] = 0
        if elenk != 0:
            cnz = q
    # postorder of the assembly tree
    for i in range(n):
        Cp[i] = FLIP(Cp[i])
    for j in range(n + 1):
        head[j] = -1
    for j in range(n, -1, -1):
        if nv[j] > 0:
            continue
        next_[j] = head[Cp[j]]  # head[-1] is undefined for j = n (Cp[n] = -1): stored as 0
        head[Cp[j]] = j         # ignored when Cp[j] is out of range
    for e in range(n, -1, -1):
        if nv[e] <= 0:
            continue
        if Cp[e] != -1:
            next_[e] = head[Cp[e]]
            head[Cp[e]] = e
    out = [0] * n
    o = 0
    for i in range(n + 1):
        if Cp[i] != -1:
            continue
        top = 0
        w[0] = i
        while top >= 0:
            pp = w[top]
            ii = head[pp]
            if ii == -1:
                top -= 1
                if pp < n:
                    out[o] = pp
                    o += 1
            else:
                head[pp] = next_[ii]
                top += 1
                w[top] = ii
    if o != n:
        raise RuntimeError(f"amdOrder: internal error (ordered {o} of {n})")
    return out


# ---- ndOrder (sparse.mjs:231-283) -------------------------------------------------------------------------------
def ndOrder(pat, x, y, leaf=48):
    n = pat["n"]
    rowptr, colidx = pat["rowptr"], pat["colidx"]
    side = [0] * n
    order = []

    def rec(nodes):
        if len(nodes) <= leaf:
            order.extend(nodes)
            return
        x0, x1, y0, y1 = math.inf, -math.inf, math.inf, -math.inf
        for v in nodes:
            if x[v] < x0:
                x0 = x[v]
            if x[v] > x1:
                x1 = x[v]
            if y[v] < y0:
                y0 = y[v]
            if y[v] > y1:
                y1 = y[v]
        key = x if x1 - x0 >= y1 - y0 else y
        srt = sorted(nodes, key=lambda v: key[v])  # stable, as Array.prototype.sort
        half = len(srt) >> 1
        for i in range(len(srt)):
            side[srt[i]] = 1 if i < half else 2
        A, S, Bn = [], [], []
        for i in range(len(srt)):
            v = srt[i]
            if i < half:
                sep = False
                for p in range(rowptr[v], rowptr[v + 1]):
                    w = colidx[p]
                    if w != v and side[w] == 2:
                        sep = True
                        break
                (S if sep else A).append(v)
            else:
                Bn.append(v)
        for v in srt:
            side[v] = 0
        rec(A)
        rec(Bn)
        order.extend(S)

    rec(list(range(n)))
    return order


# ---- nd3Order (order3d.mjs:11-77) -----------------------------------------------------------------------------------
def subPattern(pat, nodes, loc):
    m = len(nodes)
    rowptr = [0] * (m + 1)
    cols = []
    for i in range(m):
        v = nodes[i]
        for p in range(pat["rowptr"][v], pat["rowptr"][v + 1]):
            w = loc[pat["colidx"][p]]
            if w >= 0:
                cols.append(w)
        rowptr[i + 1] = len(cols)
    return {"n": m, "rowptr": rowptr, "colidx": cols}


def nd3Order(pat, x, y, z, leaf=2000):
    n = pat["n"]
    side = [0] * n
    loc = [-1] * n
    order = []

    def leafOrder(nodes):
        for i, v in enumerate(nodes):
            loc[v] = i
        sp = subPattern(pat, nodes, loc)
        for i in amdOrder(sp):
            order.append(nodes[i])
        for v in nodes:
            loc[v] = -1

    def rec(nodes):
        if len(nodes) <= leaf:
            leafOrder(nodes)
            return
        lo = [math.inf] * 3
        hi = [-math.inf] * 3
        Cs = [x, y, z]
        for v in nodes:
            for d in range(3):
                if Cs[d][v] < lo[d]:
                    lo[d] = Cs[d][v]
                if Cs[d][v] > hi[d]:
                    hi[d] = Cs[d][v]
        ax = 0
        for d in range(1, 3):
            if hi[d] - lo[d] > hi[ax] - lo[ax]:
                ax = d
        key = Cs[ax]
        srt = sorted(nodes, key=lambda v: key[v])
        half = len(srt) >> 1
        for i in range(len(srt)):
            side[srt[i]] = 1 if i < half else 2
        A, S, B = [], [], []
        for i in range(len(srt)):
            v = srt[i]
            if i < half:
                sep = False
                for p in range(pat["rowptr"][v], pat["rowptr"][v + 1]):
                    if side[pat["colidx"][p]] == 2:
                        sep = True
                        break
                (S if sep else A).append(v)
            else:
                B.append(v)
        for v in srt:
            side[v] = 0
        rec(A)
        rec(B)
        leafOrder(S)

    rec(list(range(n)))
    return order


# ---- postorder, etreeOf, analyze (sparse.mjs:597-902) --------------------------------------------------------------
def postorder(parent, n):
    head = I32(n, -1)
    next_ = I32(n)
    stack = I32(n)
    post = I32(n)
    for j in range(n - 1, -1, -1):
        if parent[j] == -1:
            continue
        next_[j] = head[parent[j]]
        head[parent[j]] = j
    k = 0
    for j in range(n):
        if parent[j] != -1:
            continue
        top = 0
        stack[0] = j
        while top >= 0:
            p = stack[top]
            i = head[p]
            if i == -1:
                top -= 1
                post[k] = p
                k += 1
            else:
                head[p] = next_[i]
                top += 1
                stack[top] = i
    return post


def etreeOf(pat, perm, pinv):
    n = pat["n"]
    parent = I32(n, -1)
    anc = I32(n, -1)
    for k in range(n):
        v = perm[k]
        for p in range(pat["rowptr"][v], pat["rowptr"][v + 1]):
            i = pinv[pat["colidx"][p]]
            while i != -1 and i < k:
                inext = anc[i]
                anc[i] = k
                if inext == -1:
                    parent[i] = k
                i = inext
    return parent


def analyze(pat, perm=None, ordering="amd", x=None, y=None, relax=True):
    """The structural fields of analyze(pat, opts): perm, parent, colCount, nnzL, flops, superStart, superParent, Sp,
    Si, Lxp, maxFront."""
    n = pat["n"]
    rowptr, colidx = pat["rowptr"], pat["colidx"]
    perm0 = perm
    if perm0 is None:
        perm0 = ndOrder(pat, x, y) if ordering == "nd" else amdOrder(pat)
    pinv = I32(n)
    for i in range(n):
        pinv[perm0[i]] = i
    parent0 = etreeOf(pat, perm0, pinv)
    post = postorder(parent0, n)
    permv = I32(n)
    for k in range(n):
        permv[k] = perm0[post[k]]
    postInv = I32(n)
    for k in range(n):
        postInv[post[k]] = k
    parent = I32(n)
    for k in range(n):
        p = parent0[post[k]]
        parent[k] = -1 if p == -1 else postInv[p]
    pinv = I32(n)
    for i in range(n):
        pinv[permv[i]] = i
    lowerP = I32(n + 1)
    for v in range(n):
        pv = pinv[v]
        for p in range(rowptr[v], rowptr[v + 1]):
            if pinv[colidx[p]] >= pv:
                lowerP[pv + 1] = lowerP[pv + 1] + 1
    for j in range(n):
        lowerP[j + 1] = lowerP[j + 1] + lowerP[j]
    nnzA = lowerP[n]
    lowerI = I32(nnzA)
    nxt = I32.of(lowerP.tolist()[:n])
    for v in range(n):
        pv = pinv[v]
        for p in range(rowptr[v], rowptr[v + 1]):
            pi = pinv[colidx[p]]
            if pi >= pv:
                q = nxt[pv]
                nxt[pv] = q + 1
                lowerI[q] = pi
    colCount = I32(n)
    first = I32(n, -1)
    maxfirst = I32(n, -1)
    prevleaf = I32(n, -1)
    ancestor = I32(n)
    for k in range(n):
        colCount[k] = 1 if first[k] == -1 else 0
        j = k
        while j != -1 and first[j] == -1:
            first[j] = k
            j = parent[j]
    for i in range(n):
        ancestor[i] = i
    for j in range(n):
        if parent[j] != -1:
            colCount[parent[j]] = colCount[parent[j]] - 1
        for p in range(lowerP[j], lowerP[j + 1]):
            i = lowerI[p]
            if i <= j or first[j] <= maxfirst[i]:
                continue
            maxfirst[i] = first[j]
            jprev = prevleaf[i]
            prevleaf[i] = j
            colCount[j] = colCount[j] + 1
            if jprev == -1:
                continue
            q = jprev
            while q != ancestor[q]:
                q = ancestor[q]
            s = jprev
            while s != q:
                sp = ancestor[s]
                ancestor[s] = q
                s = sp
            colCount[q] = colCount[q] - 1
        if parent[j] != -1:
            ancestor[j] = parent[j]
    for j in range(n):
        if parent[j] != -1:
            colCount[parent[j]] = colCount[parent[j]] + colCount[j]
    nnzL = 0
    flops = 0.0
    for j in range(n):
        nnzL += colCount[j]
        flops += float(colCount[j]) * float(colCount[j])
    nchild = I32(n)
    for j in range(n):
        if parent[j] != -1:
            nchild[parent[j]] = nchild[parent[j]] + 1
    fStart = [0]
    for j in range(1, n):
        if not (parent[j - 1] == j and colCount[j - 1] == colCount[j] + 1 and nchild[j] == 1):
            fStart.append(j)
    fStart.append(n)
    nsf = len(fStart) - 1
    colSuperF = I32(n)
    for s in range(nsf):
        for j in range(fStart[s], fStart[s + 1]):
            colSuperF[j] = s
    if relax and nsf > 1:
        sf = I32(nsf)
        sl = I32(nsf)
        sm = [0.0] * nsf  # Float64Array
        sz = [0.0] * nsf
        snnz = [0.0] * nsf
        alive = [1] * nsf
        sparent = I32(nsf)
        for s in range(nsf):
            sf[s] = fStart[s]
            sl[s] = fStart[s + 1] - 1
            sm[s] = float(colCount[fStart[s]])
            nc = fStart[s + 1] - fStart[s]
            snnz[s] = nc * sm[s] - (nc * (nc - 1)) / 2
            pl = parent[sl[s]]
            sparent[s] = -1 if pl == -1 else colSuperF[pl]
        for s in range(nsf):
            P = sparent[s]
            if P == -1 or sf[P] != sl[s] + 1:
                continue
            ncC = sl[s] - sf[s] + 1
            ncP = sl[P] - sf[P] + 1
            nc = ncC + ncP
            m = ncC + sm[P]
            stored = nc * m - (nc * (nc - 1)) / 2
            zeros = stored - snnz[s] - snnz[P] + sz[s] + sz[P]
            zf = zeros / stored
            merge = nc <= 4 or (nc <= 16 and zf < 0.8) or (nc <= 48 and zf < 0.1) or zf < 0.05
            if not merge:
                continue
            sf[P] = sf[s]
            sm[P] = m
            sz[P] = zeros
            snnz[P] = snnz[P] + snnz[s]
            alive[s] = 0
        superStart = [sf[s] for s in range(nsf) if alive[s]] + [n]
    else:
        superStart = list(fStart)
    nsuper = len(superStart) - 1
    colSuper = I32(n)
    for s in range(nsuper):
        for j in range(superStart[s], superStart[s + 1]):
            colSuper[j] = s
    superParent = I32(nsuper)
    for s in range(nsuper):
        pl = parent[superStart[s + 1] - 1]
        superParent[s] = -1 if pl == -1 else colSuper[pl]
    childHead = I32(nsuper, -1)
    childNext = I32(nsuper, -1)
    for s in range(nsuper):
        P = superParent[s]
        if P == -1:
            continue
        childNext[s] = childHead[P]
        childHead[P] = s
    Sp = [0] * (nsuper + 1)
    rowsOf = [None] * nsuper
    marker = I32(n, -1)
    maxFront = 0
    for s in range(nsuper):
        f, l = superStart[s], superStart[s + 1] - 1
        below = []
        for j in range(f, l + 1):
            for p in range(lowerP[j], lowerP[j + 1]):
                i = lowerI[p]
                if i > l and marker[i] != s:
                    marker[i] = s
                    below.append(i)
        c = childHead[s]
        while c != -1:
            rc = rowsOf[c]
            ncc = superStart[c + 1] - superStart[c]
            for r in range(ncc, len(rc)):
                i = rc[r]
                if i > l and marker[i] != s:
                    marker[i] = s
                    below.append(i)
            c = childNext[c]
        rows = list(range(f, l + 1)) + sorted(below)  # typed-array sort is numeric
        rowsOf[s] = rows
        Sp[s + 1] = Sp[s] + len(rows)
        maxFront = max(maxFront, len(rows))
    Si = [i for s in range(nsuper) for i in rowsOf[s]]
    Lxp = [0.0] * (nsuper + 1)
    for s in range(nsuper):
        Lxp[s + 1] = Lxp[s] + len(rowsOf[s]) * (superStart[s + 1] - superStart[s])
    return {"perm": permv.tolist(), "parent": parent.tolist(), "colCount": colCount.tolist(), "nnzL": nnzL,
            "flops": flops, "superStart": superStart, "superParent": superParent.tolist(), "Sp": Sp, "Si": Si,
            "Lxp": [int(v) for v in Lxp], "maxFront": maxFront}
