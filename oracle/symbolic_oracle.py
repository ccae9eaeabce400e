"""ORACLE — test infrastructure only; never imported by the product.

Pure-Python restatement of symPACK's symbolic analysis at one rank, written
independently of the product's C++ module so that the two can be compared bit
for bit.  Each function cites the reference routine it follows (symPACK v2.0):

  expand_symmetric   src/DistSparseMatrixGraph.cpp:929-1084 (ExpandSymmetric)
  set_keep_diag      src/DistSparseMatrixGraph.cpp:39-97
  genmmd             src/genmmd.F, mmdint.F, mmdelm.F, mmdupd.F, mmdnum.F
                     (ordmmd.F:70-79: delta = 0, maxint = 2,000,000,000)
  genrcm             src/genrcm.F, fnroot.F, rootls.F, degree.F, rcm.F
                     (called from src/Ordering.cpp:221-300, Ordering::RCM)
  amdbar             src/amdbar.F (called from src/Ordering.cpp:411-520, Ordering::AMD)
  construct_etree    src/ETree.cpp:317-397
  postorder_tree     src/ETree.cpp:24-119
  lcol_row_count     include/sympack/impl/symPACKMatrixBase_impl.hpp:310-470
  sort_children      src/ETree.cpp:122-225
  find_supernodes    symPACKMatrixBase_impl.hpp:42-80
  relax_supernodes   symPACKMatrixBase_impl.hpp:473-609 (+ DisjointSet, ETree.hpp:12-99)
  symbolic_factor    symPACKMatrixBase_impl.hpp:613-935
  build_cells        include/sympack/symPACKMatrix2D.hpp:3317-3396
  symbolic_chain     symPACKMatrix2D.hpp:2699-3081 (MMD, RCM, AMD and NATURAL branches)

Arrays are Python lists, 1-based values; index 0 of the work arrays of the
MMD routines is a dummy so that the Fortran subscripts carry over.
"""
from __future__ import annotations

import numpy as np

MAXINT = 2000000000


# ----------------------------------------------------------------- graphs --
def expand_symmetric(n, colptr, rowind):
    """Full symmetric graph in ExpandSymmetric's entry order: per column, the
    mirrored (upper) rows in descending order, then the original lower rows."""
    cols = [[] for _ in range(n + 1)]
    lower = [None] * (n + 1)
    for c in range(1, n + 1):
        lower[c] = [int(rowind[p - 1]) for p in range(int(colptr[c - 1]), int(colptr[c]))]
    mirrored = [[] for _ in range(n + 1)]
    for c in range(1, n + 1):          # unpack order: source column ascending
        for r in lower[c]:
            if r > c:
                mirrored[r].append(c)
    xadj = [1]
    adj = []
    for c in range(1, n + 1):
        # entries received later are written further to the left
        adj.extend(reversed(mirrored[c]))
        adj.extend(lower[c])
        xadj.append(len(adj) + 1)
    return xadj, adj


def set_keep_diag(n, xadj, adj, keep):
    nx, na = [1], []
    for c in range(1, n + 1):
        ent = adj[xadj[c - 1] - 1:xadj[c] - 1]
        if not keep:
            na.extend(r for r in ent if r != c)
        else:
            added = False
            for r in ent:
                if r < c:
                    na.append(r)
                if r > c:
                    if not added:
                        na.append(c)
                        added = True
                    na.append(r)
            if not added:
                na.append(c)
        nx.append(len(na) + 1)
    return nx, na


# -------------------------------------------------------------------- MMD --
def genmmd(neqns, xadj_in, adj_in):
    """Liu's multiple minimum external degree.  Returns invp (old -> new), 1-based."""
    xadj = [0] + list(xadj_in)           # xadj[1..n+1]
    adjncy = [0] + list(adj_in)          # adjncy[1..nadj]
    dhead = [0] * (neqns + 2)
    invp = [0] * (neqns + 2)             # DFORW during elimination
    perm = [0] * (neqns + 2)             # DBAKW during elimination
    qsize = [0] * (neqns + 2)
    llist = [0] * (neqns + 2)
    marker = [0] * (neqns + 2)
    delta = 0
    st = {"tag": 0}

    # mmdint
    for node in range(1, neqns + 1):
        dhead[node] = 0
        qsize[node] = 1
        marker[node] = 0
        llist[node] = 0
    for node in range(1, neqns + 1):
        ndeg = xadj[node + 1] - xadj[node] + 1
        fnode = dhead[ndeg]
        invp[node] = fnode
        dhead[ndeg] = node
        if fnode > 0:
            perm[fnode] = node
        perm[node] = -ndeg

    def reset_marker():
        for i in range(1, neqns + 1):
            if marker[i] < MAXINT:
                marker[i] = 0

    def mmdelm(mdnode):
        tag = st["tag"]
        dforw, dbakw = invp, perm
        marker[mdnode] = tag
        istrt = xadj[mdnode]
        istop = xadj[mdnode + 1] - 1
        elmnt = 0
        rloc = istrt
        rlmt = istop
        i = istrt
        while i <= istop:                             # do 200
            nabor = adjncy[i]
            if nabor == 0:
                break                                 # go to 300
            if marker[nabor] < tag:
                marker[nabor] = tag
                if dforw[nabor] < 0:                  # 100
                    llist[nabor] = elmnt
                    elmnt = nabor
                else:
                    adjncy[rloc] = nabor
                    rloc += 1
            i += 1
        while elmnt > 0:                              # 300
            adjncy[rlmt] = -elmnt
            link = elmnt
            restart = True
            while restart:                            # 400
                restart = False
                jstrt = xadj[link]
                jstop = xadj[link + 1] - 1
                j = jstrt
                while j <= jstop:
                    node = adjncy[j]
                    link = -node
                    if node < 0:
                        restart = True
                        break
                    if node == 0:
                        break                         # go to 900
                    if not (marker[node] >= tag or dforw[node] < 0):
                        marker[node] = tag
                        while rloc >= rlmt:           # 600
                            link2 = -adjncy[rlmt]
                            rloc = xadj[link2]
                            rlmt = xadj[link2 + 1] - 1
                        adjncy[rloc] = node           # 700
                        rloc += 1
                    j += 1
            elmnt = llist[elmnt]                      # 900
        if rloc <= rlmt:                              # 1000
            adjncy[rloc] = 0
        link = mdnode
        while True:                                   # 1100
            istrt = xadj[link]
            istop = xadj[link + 1] - 1
            jumped = False
            i = istrt
            while i <= istop:
                rnode = adjncy[i]
                link = -rnode
                if rnode < 0:
                    jumped = True
                    break
                if rnode == 0:
                    return                            # 1800
                pvnode = dbakw[rnode]                 # 1200
                if pvnode != 0 and pvnode != -MAXINT:
                    nxnode = dforw[rnode]
                    if nxnode > 0:
                        dbakw[nxnode] = pvnode
                    if pvnode > 0:
                        dforw[pvnode] = nxnode
                    npv = -pvnode
                    if pvnode < 0:
                        dhead[npv] = nxnode
                jstrt = xadj[rnode]                   # 1300
                jstop = xadj[rnode + 1] - 1
                xqnbr = jstrt
                j = jstrt
                while j <= jstop:
                    nabor = adjncy[j]
                    if nabor == 0:
                        break
                    if marker[nabor] < tag:
                        adjncy[xqnbr] = nabor
                        xqnbr += 1
                    j += 1
                nqnbrs = xqnbr - jstrt                # 1500
                if nqnbrs <= 0:
                    qsize[mdnode] += qsize[rnode]
                    qsize[rnode] = 0
                    marker[rnode] = MAXINT
                    dforw[rnode] = -mdnode
                    dbakw[rnode] = -MAXINT
                else:                                 # 1600
                    dforw[rnode] = nqnbrs + 1
                    dbakw[rnode] = 0
                    adjncy[xqnbr] = mdnode
                    xqnbr += 1
                    if xqnbr <= jstop:
                        adjncy[xqnbr] = 0
                i += 1                                # 1700
            if not jumped:
                return

    def place(enode, deg, mdeg):
        deg = deg - qsize[enode] + 1                  # 2100
        fnode = dhead[deg]
        invp[enode] = fnode
        perm[enode] = -deg
        if fnode > 0:
            perm[fnode] = enode
        dhead[deg] = enode
        return min(mdeg, deg)

    def mmdupd(ehead, mdeg):
        dforw, dbakw = invp, perm
        mdeg0 = mdeg + delta
        elmnt = ehead
        while elmnt > 0:                              # 100
            mtag = st["tag"] + mdeg0
            if mtag >= MAXINT:
                st["tag"] = 1
                reset_marker()
                mtag = st["tag"] + mdeg0
            q2head = qxhead = deg0 = 0                # 300
            link = elmnt
            again = True
            while again:                              # 400
                again = False
                istrt = xadj[link]
                istop = xadj[link + 1] - 1
                i = istrt
                while i <= istop:
                    enode = adjncy[i]
                    link = -enode
                    if enode < 0:
                        again = True
                        break
                    if enode == 0:
                        break
                    if qsize[enode] != 0:
                        deg0 += qsize[enode]
                        marker[enode] = mtag
                        if dbakw[enode] == 0:
                            if dforw[enode] != 2:
                                llist[enode] = qxhead
                                qxhead = enode
                            else:
                                llist[enode] = q2head
                                q2head = enode
                    i += 1
            enode = q2head                            # 800 / 900
            while enode > 0:
                if dbakw[enode] == 0:
                    st["tag"] += 1
                    tag = st["tag"]
                    deg = deg0
                    istrt = xadj[enode]
                    nabor = adjncy[istrt]
                    if nabor == elmnt:
                        nabor = adjncy[istrt + 1]
                    link = nabor
                    if dforw[nabor] >= 0:
                        deg += qsize[nabor]
                    else:
                        again = True
                        while again:                  # 1000
                            again = False
                            istrt = xadj[link]
                            istop = xadj[link + 1] - 1
                            i = istrt
                            while i <= istop:
                                node = adjncy[i]
                                link = -node
                                if node != enode:
                                    if node < 0:
                                        again = True
                                        break
                                    if node == 0:
                                        break
                                    if qsize[node] != 0:
                                        if marker[node] < tag:
                                            marker[node] = tag
                                            deg += qsize[node]
                                        elif dbakw[node] == 0:
                                            if dforw[node] == 2:
                                                qsize[enode] += qsize[node]
                                                qsize[node] = 0
                                                marker[node] = MAXINT
                                                dforw[node] = -enode
                                                dbakw[node] = -MAXINT
                                            elif dbakw[node] == 0:
                                                dbakw[node] = -MAXINT
                                i += 1
                    mdeg = place(enode, deg, mdeg)
                enode = llist[enode]                  # 2200
            enode = qxhead                            # 1500 / 1600
            while enode > 0:
                if dbakw[enode] == 0:
                    st["tag"] += 1
                    tag = st["tag"]
                    deg = deg0
                    istrt = xadj[enode]
                    istop = xadj[enode + 1] - 1
                    i = istrt
                    while i <= istop:
                        nabor = adjncy[i]
                        if nabor == 0:
                            break
                        if marker[nabor] < tag:
                            marker[nabor] = tag
                            link = nabor
                            if dforw[nabor] >= 0:
                                deg += qsize[nabor]
                            else:
                                again = True
                                while again:          # 1700
                                    again = False
                                    jstrt = xadj[link]
                                    jstop = xadj[link + 1] - 1
                                    j = jstrt
                                    while j <= jstop:
                                        node = adjncy[j]
                                        link = -node
                                        if node < 0:
                                            again = True
                                            break
                                        if node == 0:
                                            break
                                        if marker[node] < tag:
                                            marker[node] = tag
                                            deg += qsize[node]
                                        j += 1
                        i += 1
                    mdeg = place(enode, deg, mdeg)
                enode = llist[enode]
            st["tag"] = mtag                          # 2300
            elmnt = llist[elmnt]
        return mdeg

    # genmmd
    num = 1
    nextmd = dhead[1]
    while nextmd > 0:                                 # 100
        mdnode = nextmd
        nextmd = invp[mdnode]
        marker[mdnode] = MAXINT
        invp[mdnode] = -num
        num += 1
    if num <= neqns:
        st["tag"] = 1
        dhead[1] = 0
        mdeg = 2
        done = False
        while not done:                               # 300
            while dhead[mdeg] <= 0:
                mdeg += 1
            mdlmt = mdeg + delta
            ehead = 0
            while True:                               # 500
                mdnode = dhead[mdeg]
                if mdnode <= 0:
                    mdeg += 1
                    if mdeg > mdlmt:
                        break                         # 900
                    continue
                nextmd = invp[mdnode]                 # 600
                dhead[mdeg] = nextmd
                if nextmd > 0:
                    perm[nextmd] = -mdeg
                invp[mdnode] = -num
                if num + qsize[mdnode] > neqns:
                    done = True
                    break
                st["tag"] += 1
                if st["tag"] >= MAXINT:
                    st["tag"] = 1
                    reset_marker()
                mmdelm(mdnode)
                num += qsize[mdnode]
                llist[mdnode] = ehead
                ehead = mdnode
            if done or num > neqns:
                break
            mdeg = mmdupd(ehead, mdeg)
    # mmdnum
    for node in range(1, neqns + 1):
        perm[node] = invp[node] if qsize[node] <= 0 else -invp[node]
    for node in range(1, neqns + 1):
        if perm[node] > 0:
            continue
        father = node
        while perm[father] <= 0:
            father = -perm[father]
        root = father
        num = perm[root] + 1
        invp[node] = -num
        perm[root] = num
        father = node
        while True:
            nextf = -perm[father]
            if nextf <= 0:
                break
            perm[father] = -root
            father = nextf
    return [-invp[node] for node in range(1, neqns + 1)]


# ------------------------------------------------------ etree and counts --
def _rootls(root, xadj, adj, mask, xls, ls):
    """ROOTLS (rootls.F): level structure of root's component among mask != 0;
    fills ls[1..ccsize], xls[1..nlvl+1]; returns nlvl."""
    mask[root] = 0
    ls[1] = root
    nlvl = lvlend = 0
    ccsize = 1
    while True:
        lbegin = lvlend + 1
        lvlend = ccsize
        nlvl += 1
        xls[nlvl] = lbegin
        for i in range(lbegin, lvlend + 1):
            node = ls[i]
            for j in range(xadj[node], xadj[node + 1]):
                nbr = adj[j]
                if mask[nbr] != 0:
                    ccsize += 1
                    ls[ccsize] = nbr
                    mask[nbr] = 0
        if ccsize - lvlend <= 0:
            break
    xls[nlvl + 1] = lvlend + 1
    for i in range(1, ccsize + 1):
        mask[ls[i]] = 1
    return nlvl


def _fnroot(root, xadj, adj, mask, xls, ls):
    """FNROOT (fnroot.F): pseudo-peripheral node of root's component."""
    nlvl = _rootls(root, xadj, adj, mask, xls, ls)
    ccsize = xls[nlvl + 1] - 1
    if nlvl == 1 or nlvl == ccsize:
        return root
    while True:
        jstrt = xls[nlvl]
        mindeg = ccsize
        root = ls[jstrt]
        if ccsize != jstrt:
            for j in range(jstrt, ccsize + 1):
                node = ls[j]
                ndeg = sum(1 for k in range(xadj[node], xadj[node + 1]) if mask[adj[k]] > 0)
                if ndeg < mindeg:
                    root, mindeg = node, ndeg
        nunlvl = _rootls(root, xadj, adj, mask, xls, ls)
        if nunlvl <= nlvl:
            return root
        nlvl = nunlvl
        if nlvl >= ccsize:
            return root


def _rcm_component(root, xadj, adj, mask, perm, off, deg):
    """DEGREE + RCM (degree.F, rcm.F): reverse Cuthill-McKee numbering of root's
    component into perm[off .. off+ccsize-1]; returns ccsize."""
    # DEGREE: breadth first over the component, counting unmasked neighbours
    seen = {root}
    order = [root]
    lvlend = 0
    while True:
        lbegin, lvlend = lvlend, len(order)
        for i in range(lbegin, lvlend):
            node = order[i]
            ideg = 0
            for j in range(xadj[node], xadj[node + 1]):
                nbr = adj[j]
                if mask[nbr] == 0:
                    continue
                ideg += 1
                if nbr not in seen:
                    seen.add(nbr)
                    order.append(nbr)
            deg[node] = ideg
        if len(order) == lvlend:
            break
    ccsize = len(order)
    mask[root] = 0
    out = [root]
    if ccsize > 1:
        lvlend = 0
        while True:
            lbegin, lvlend = lvlend, len(out)
            for i in range(lbegin, lvlend):
                node = out[i]
                fnbr = len(out)
                for j in range(xadj[node], xadj[node + 1]):
                    nbr = adj[j]
                    if mask[nbr] != 0:
                        mask[nbr] = 0
                        out.append(nbr)
                # stable insertion sort of the new neighbours by increasing degree
                for k in range(fnbr + 1, len(out)):
                    v = out[k]
                    l = k - 1
                    while l >= fnbr and deg[out[l]] > deg[v]:
                        out[l + 1] = out[l]
                        l -= 1
                    out[l + 1] = v
            if len(out) <= lvlend:
                break
        out.reverse()
    perm[off:off + ccsize] = out
    return ccsize


def genrcm(neqns, xadj_in, adj_in):
    """GENRCM (genrcm.F) on a 1-based expanded graph without diagonal; returns
    invp (1-based) as Ordering::RCM forms it (Ordering.cpp:283-286)."""
    xadj = [0] + list(xadj_in)
    adj = [0] + list(adj_in)
    mask = [0] + [1] * neqns
    xls = [0] * (neqns + 2)
    ls = [0] * (neqns + 2)
    deg = [0] * (neqns + 1)
    perm = [0] * neqns
    num = 0
    for i in range(1, neqns + 1):
        if mask[i] == 0:
            continue
        root = _fnroot(i, xadj, adj, mask, xls, ls)
        num += _rcm_component(root, xadj, adj, mask, perm, num, deg)
        if num >= neqns:
            break
    invp = [0] * neqns
    for k, node in enumerate(perm):
        invp[node - 1] = k + 1
    return invp


def amdbar(n, xadj_in, adj_in):
    """AMDBAR (amdbar.F) as Ordering::AMD calls it (Ordering.cpp:466-490): IW holds
    the adjacency plus n free entries (IWLEN = nnz + n, PFREE = nnz + 1), IOVFLO =
    2**31 - 1; returns ELEN, the inverse permutation (1-based).  Index 0 of every
    array is a dummy so that the Fortran subscripts carry over."""
    nnz = len(adj_in)
    iwlen = nnz + n
    iw = [0] * (iwlen + 1)
    iw[1:nnz + 1] = list(adj_in)
    pe = [0] + [int(x) for x in xadj_in[:n]]
    ln_ = [0] + [int(xadj_in[i + 1] - xadj_in[i]) for i in range(n)]
    pfree = nnz + 1
    nv = [0] * (n + 1)
    nxt = [0] * (n + 1)
    last = [0] * (n + 1)
    head = [0] * (n + 1)
    elen = [0] * (n + 1)
    degree = [0] * (n + 1)
    w = [0] * (n + 1)
    wflg, mindeg, nel, hmod, dmax = 2, 1, 0, max(1, n - 1), 0
    wbig = 2 ** 31 - 1 - n
    for i in range(1, n + 1):
        nv[i], w[i], degree[i] = 1, 1, ln_[i]
    for i in range(1, n + 1):
        deg = degree[i]
        if deg > 0:
            inext = head[deg]
            if inext:
                last[inext] = i
            nxt[i] = inext
            head[deg] = i
        else:
            nel += 1
            elen[i], pe[i], w[i] = -nel, 0, 0

    def remove(i):
        ilast, inext = last[i], nxt[i]
        if inext:
            last[inext] = ilast
        if ilast:
            nxt[ilast] = inext
        else:
            head[degree[i]] = inext

    def reset_w():
        for x in range(1, n + 1):
            if w[x]:
                w[x] = 1

    while nel < n:
        deg = mindeg
        while head[deg] <= 0:
            deg += 1
        me = head[deg]
        mindeg = deg
        inext = nxt[me]
        if inext:
            last[inext] = 0
        head[deg] = inext
        elenme = elen[me]
        elen[me] = -(nel + 1)
        nvpiv = nv[me]
        nel += nvpiv
        nv[me] = -nvpiv
        degme = 0
        if elenme == 0:
            pme1 = pe[me]
            pme2 = pme1 - 1
            for p in range(pme1, pme1 + ln_[me]):
                i = iw[p]
                if nv[i] > 0:
                    degme += nv[i]
                    nv[i] = -nv[i]
                    pme2 += 1
                    iw[pme2] = i
                    remove(i)
            newmem = 0
        else:
            p = pe[me]
            pme1 = pfree
            slenme = ln_[me] - elenme
            for knt1 in range(1, elenme + 2):
                if knt1 > elenme:
                    e, pj, ln = me, p, slenme
                else:
                    e = iw[p]
                    p += 1
                    pj, ln = pe[e], ln_[e]
                for knt2 in range(1, ln + 1):
                    i = iw[pj]
                    pj += 1
                    nvi = nv[i]
                    if nvi <= 0:
                        continue
                    if pfree > iwlen:  # garbage collection
                        pe[me] = p
                        ln_[me] -= knt1
                        if ln_[me] == 0:
                            pe[me] = 0
                        pe[e] = pj
                        ln_[e] = ln - knt2
                        if ln_[e] == 0:
                            pe[e] = 0
                        for j in range(1, n + 1):
                            pn = pe[j]
                            if pn > 0:
                                pe[j] = iw[pn]
                                iw[pn] = -j
                        pdst = psrc = 1
                        pend = pme1 - 1
                        while psrc <= pend:
                            j = -iw[psrc]
                            psrc += 1
                            if j > 0:
                                iw[pdst] = pe[j]
                                pe[j] = pdst
                                pdst += 1
                                lenj = ln_[j]
                                iw[pdst:pdst + lenj - 1] = iw[psrc:psrc + lenj - 1] if lenj > 1 else []
                                pdst += lenj - 1
                                psrc += lenj - 1
                        p1 = pdst
                        for ps in range(pme1, pfree):
                            iw[pdst] = iw[ps]
                            pdst += 1
                        pme1, pfree = p1, pdst
                        pj, p = pe[e], pe[me]
                    degme += nvi
                    nv[i] = -nvi
                    iw[pfree] = i
                    pfree += 1
                    remove(i)
                if e != me:
                    pe[e], w[e] = -me, 0
            pme2 = pfree - 1
            newmem = pfree - pme1
        degree[me] = degme
        pe[me] = pme1
        ln_[me] = pme2 - pme1 + 1
        if wflg >= wbig:
            reset_w()
            wflg = 2
        for pme in range(pme1, pme2 + 1):
            i = iw[pme]
            eln = elen[i]
            if eln > 0:
                nvi = -nv[i]
                wnvi = wflg - nvi
                for p in range(pe[i], pe[i] + eln):
                    e = iw[p]
                    we = w[e]
                    if we >= wflg:
                        we -= nvi
                    elif we != 0:
                        we = degree[e] + wnvi
                    w[e] = we
        for pme in range(pme1, pme2 + 1):
            i = iw[pme]
            p1 = pe[i]
            p2 = p1 + elen[i] - 1
            pn = p1
            h = deg = 0
            for p in range(p1, p2 + 1):
                e = iw[p]
                if w[e] != 0:
                    deg += w[e] - wflg
                    iw[pn] = e
                    pn += 1
                    h += e
            elen[i] = pn - p1 + 1
            p3 = pn
            for p in range(p2 + 1, p1 + ln_[i]):
                j = iw[p]
                if nv[j] > 0:
                    deg += nv[j]
                    iw[pn] = j
                    pn += 1
                    h += j
            if elen[i] == 1 and p3 == pn:  # mass elimination
                pe[i] = -me
                nvi = -nv[i]
                degme -= nvi
                nvpiv += nvi
                nel += nvi
                nv[i] = elen[i] = 0
            else:
                degree[i] = min(degree[i], deg)
                iw[pn] = iw[p3]
                iw[p3] = iw[p1]
                iw[p1] = me
                ln_[i] = pn - p1 + 1
                h = h % hmod + 1
                j = head[h]
                if j <= 0:
                    nxt[i] = -j
                    head[h] = -i
                else:
                    nxt[i] = last[j]
                    last[j] = i
                last[i] = h
        degree[me] = degme
        dmax = max(dmax, degme)
        wflg += dmax
        if wflg >= wbig:
            reset_w()
            wflg = 2
        for pme in range(pme1, pme2 + 1):
            i = iw[pme]
            if nv[i] >= 0:
                continue
            h = last[i]
            j = head[h]
            if j == 0:
                continue
            if j < 0:
                i = -j
                head[h] = 0
            else:
                i = last[j]
                last[j] = 0
            while i != 0 and nxt[i] != 0:
                ln, eln = ln_[i], elen[i]
                for p in range(pe[i] + 1, pe[i] + ln):
                    w[iw[p]] = wflg
                jlast, j = i, nxt[i]
                while j != 0:
                    if ln_[j] == ln and elen[j] == eln and all(w[iw[p]] == wflg for p in range(pe[j] + 1, pe[j] + ln)):
                        pe[j] = -i
                        nv[i] += nv[j]
                        nv[j] = elen[j] = 0
                        j = nxt[j]
                        nxt[jlast] = j
                    else:
                        jlast, j = j, nxt[j]
                wflg += 1
                i = nxt[i]
        p = pme1
        nleft = n - nel
        for pme in range(pme1, pme2 + 1):
            i = iw[pme]
            nvi = -nv[i]
            if nvi > 0:
                nv[i] = nvi
                deg = max(1, min(degree[i] + degme - nvi, nleft - nvi))
                inext = head[deg]
                if inext:
                    last[inext] = i
                nxt[i] = inext
                last[i] = 0
                head[deg] = i
                mindeg = min(mindeg, deg)
                degree[i] = deg
                iw[p] = i
                p += 1
        nv[me] = nvpiv + degme
        ln_[me] = p - pme1
        if ln_[me] == 0:
            pe[me] = w[me] = 0
        if newmem:
            pfree = p
    for i in range(1, n + 1):
        if elen[i] == 0:
            j = -pe[i]
            while elen[j] >= 0:
                j = -pe[j]
            e = j
            k = -elen[e]
            j = i
            while elen[j] >= 0:
                jnext = -pe[j]
                pe[j] = -e
                if elen[j] == 0:
                    elen[j] = k
                    k += 1
                j = jnext
            elen[e] = -k
    return [abs(elen[i]) for i in range(1, n + 1)]


def construct_etree(n, xadj, adj, perm, invp):
    parent = [0] * n
    ancstr = [0] * n
    for i in range(1, n + 1):
        node = perm[i - 1]
        jstrt, jstop = xadj[node - 1], xadj[node] - 1
        if jstrt < jstop:
            for j in range(jstrt, jstop + 1):
                nbr = invp[adj[j - 1] - 1]
                if nbr < i:
                    if ancstr[nbr - 1] == i:
                        continue
                    brk = False
                    while ancstr[nbr - 1] > 0:
                        if ancstr[nbr - 1] == i:
                            brk = True
                            break
                        nxt = ancstr[nbr - 1]
                        ancstr[nbr - 1] = i
                        nbr = nxt
                    if not brk:
                        parent[nbr - 1] = i
                        ancstr[nbr - 1] = i
    return parent


def _btree_to_po(n, fson, brother):
    stack = []
    invpos = [0] * n
    vertex, m = n, 0
    while m < n:
        while True:
            stack.append(vertex)
            vertex = fson[vertex - 1]
            if vertex <= 0:
                break
        stop = False
        while vertex == 0:
            if not stack:
                stop = True
                break
            vertex = stack.pop()
            m += 1
            invpos[vertex - 1] = m
            vertex = brother[vertex - 1]
        if stop:
            break
    return invpos


def _compose(perm, invp, invp2):
    n = len(invp)
    for i in range(n):
        invp[i] = invp2[invp[i] - 1]
    for i in range(1, n + 1):
        perm[invp[i - 1] - 1] = i


def postorder_tree(parent, perm, invp):
    n = len(parent)
    fson = [0] * n
    brother = [0] * n
    lroot = n
    for v in range(n - 1, 0, -1):
        p = parent[v - 1]
        if p == 0 or p == v:
            brother[lroot - 1] = v
            lroot = v
        else:
            brother[v - 1] = fson[p - 1]
            fson[p - 1] = v
    invpos = _btree_to_po(n, fson, brother)
    po = [0] * n
    for i in range(1, n + 1):
        nd = parent[i - 1]
        po[invpos[i - 1] - 1] = invpos[nd - 1] if nd > 0 else nd
    _compose(perm, invp, invpos)
    return po


def lcol_row_count(n, xadj, adj, perm, invp, poparent):
    mask = 0xFFFFFFFF
    cc = [0] * n
    rc = [0] * n
    level = [0] * (n + 1)
    weight = [0] * (n + 1)
    fdesc = [0] * (n + 1)
    nchild = [0] * (n + 1)
    sset = [0] * n
    prvlf = [0] * n
    prvnbr = [0] * n
    xsup = 1
    for k in range(n, 0, -1):
        rc[k - 1] = 1
        sset[k - 1] = k
        level[k] = (level[poparent[k - 1]] + 1) & mask
        weight[k] = 1
        fdesc[k] = k
    for k in range(1, n):
        p = poparent[k - 1]
        weight[p] = 0
        nchild[p] += 1
        if fdesc[k] < fdesc[p]:
            fdesc[p] = fdesc[k]
    for low in range(1, n + 1):
        lflag = 0
        ifdesc = fdesc[low]
        old = perm[low - 1]
        for j in range(xadj[old - 1], xadj[old]):
            hi = invp[adj[j - 1] - 1]
            if hi > low:
                if ifdesc > prvnbr[hi - 1]:
                    weight[low] += 1
                    pleaf = prvlf[hi - 1]
                    if pleaf == 0:
                        rc[hi - 1] = (rc[hi - 1] + (level[low] - level[hi])) & mask
                    else:
                        last1 = pleaf
                        last2 = sset[last1 - 1]
                        lca = sset[last2 - 1]
                        while lca != last2:
                            sset[last1 - 1] = lca
                            last1 = lca
                            last2 = sset[last1 - 1]
                            lca = sset[last2 - 1]
                        rc[hi - 1] = (rc[hi - 1] + (level[low] - level[lca])) & mask
                        weight[lca] -= 1
                    prvlf[hi - 1] = low
                    lflag = 1
                prvnbr[hi - 1] = low
        p = poparent[low - 1]
        weight[p] -= 1
        if lflag == 1 or nchild[low] >= 2:
            xsup = low
        sset[xsup - 1] = p
    for k in range(1, n + 1):
        t = cc[k - 1] + weight[k]
        cc[k - 1] = t
        p = poparent[k - 1]
        if p != 0:
            cc[p - 1] += t
    return cc


def sort_children(poparent, cc, perm, invp):
    n = len(poparent)
    fson = [0] * n
    brother = [0] * n
    lson = [0] * n
    lroot = n
    for v in range(n - 1, 0, -1):
        p = poparent[v - 1]
        if p == 0 or p == v:
            brother[lroot - 1] = v
            lroot = v
        else:
            ls = lson[p - 1]
            if ls > 0:
                if cc[v - 1] >= cc[ls - 1]:
                    brother[v - 1] = fson[p - 1]
                    fson[p - 1] = v
                else:
                    brother[ls - 1] = v
                    lson[p - 1] = v
            else:
                fson[p - 1] = v
                lson[p - 1] = v
    brother[lroot - 1] = 0
    invpos = _btree_to_po(n, fson, brother)
    newpar = [0] * n
    for i in range(1, n + 1):
        nd = poparent[i - 1]
        newpar[invpos[i - 1] - 1] = invpos[nd - 1] if nd > 0 else nd
    newcc = [0] * n
    for node in range(1, n + 1):
        newcc[invpos[node - 1] - 1] = cc[node - 1]
    _compose(perm, invp, invpos)
    return newpar, newcc


# ------------------------------------------------------------- supernodes --
def find_supernodes(poparent, cc, max_size=0):
    n = len(cc)
    sup = [0] * n
    nsuper, supsize = 1, 1
    sup[0] = 1
    for i in range(2, n + 1):
        if poparent[i - 2] == i and cc[i - 2] == cc[i - 1] + 1 and (supsize < max_size or max_size == 0):
            supsize += 1
            sup[i - 1] = nsuper
            continue
        nsuper += 1
        supsize = 1
        sup[i - 1] = nsuper
    xsuper = [0] * (nsuper + 1)
    lst = nsuper + 1
    for i in range(n, 0, -1):
        k = sup[i - 1]
        if k != lst:
            xsuper[lst - 1] = i + 1
        lst = k
    xsuper[0] = 1
    return sup, xsuper


class _DisjointSet:
    def __init__(self, n):
        self.pp = [0] * n
        self.root = [0] * n

    def make(self, i):
        self.pp[i - 1] = i
        return i

    def find(self, i):
        p = self.pp[i - 1]
        gp = self.pp[p - 1]
        while gp != p:
            i = self.make(gp)
            p = self.pp[i - 1]
            gp = self.pp[p - 1]
        return p

    def union(self, s, t, r=-1):
        ts = self.find(t)
        ss = self.find(s)
        self.pp[ss - 1] = ts
        ss = ts
        self.root[ss - 1] = t if r == -1 else r


def relax_supernodes(poparent, cc, sup, xsuper, nrelax0=8, nrelax1=32, nrelax2=64, max_size=0,
                     zrelax0=0.8, zrelax1=0.1, zrelax2=0.05):
    nsuper = len(xsuper) - 1
    ds = _DisjointSet(nsuper)
    ncols = [0] * nsuper
    zeros = [0] * nsuper
    newcc = [0] * nsuper
    for k in range(nsuper, 0, -1):
        cs = ds.make(k)
        ds.root[cs - 1] = k
        fc, lc = xsuper[k - 1], xsuper[k] - 1
        ncols[k - 1] = lc - fc + 1
        newcc[k - 1] = cc[fc - 1]
    for k in range(nsuper, 0, -1):
        fc, lc = xsuper[k - 1], xsuper[k] - 1
        width = ncols[k - 1]
        pfc = poparent[lc - 1]
        if pfc == 0:
            continue
        ps = sup[pfc - 1]
        ps = ds.root[ds.find(ps) - 1]
        if ps != k + 1:
            continue
        pwidth = ncols[ps - 1]
        pfirst = xsuper[ps - 1]
        totzeros = zeros[ps - 1]
        merged = width + pwidth
        merge = False
        if (merged <= max_size or max_size == 0) and nrelax0 > 0:
            if merged <= nrelax0:
                merge = True
            elif merged <= max_size or max_size == 0:
                nnzchild = float(cc[fc - 1])
                nnzparent = float(cc[pfirst - 1])
                xnewzeros = width * (nnzparent + width - nnzchild)
                if xnewzeros == 0:
                    merge = True
                else:
                    xtotzeros = float(totzeros) + xnewzeros
                    xm = float(merged)
                    xtotsize = (xm * (xm + 1) / 2) + xm * (nnzparent - pwidth)
                    with np.errstate(divide="ignore", invalid="ignore"):
                        z = float(np.float64(xtotzeros) / np.float64(xtotsize))  # IEEE, as in C++
                    totzeros += int(xnewzeros)
                    if xtotsize * 8 < float(2 ** 64 - 1):
                        if merged <= nrelax1 and z < zrelax0:
                            merge = True
                        elif merged <= nrelax2 and z < zrelax1:
                            merge = True
                        elif z < zrelax2:
                            merge = True
        if merge:
            ncols[k - 1] += ncols[ps - 1]
            zeros[k - 1] = totzeros
            newcc[k - 1] = width + newcc[ps - 1]
            ds.union(k, ps, k)
    rx = []
    ncc = []
    for k in range(1, nsuper + 1):
        if k == ds.root[ds.find(k) - 1]:
            rx.append(xsuper[k - 1])
            ncc.append(newcc[k - 1])
    rx.append(xsuper[nsuper])
    cc = list(cc)
    sup = list(sup)
    for k in range(1, len(rx)):
        fc, lc = rx[k - 1], rx[k] - 1
        for c in range(fc, lc + 1):
            sup[c - 1] = k
            cc[c - 1] = ncc[k - 1] - (c - fc)
    return cc, sup, rx


def symbolic_factor(n, xadj, adj, invp, poparent, cc, xsuper, sup):
    """Row structure of each supernode: the union of its children's structures
    below their own columns and the permuted columns of A it contains (the
    reference merges these as a sorted linked list; a sorted set is the same)."""
    nsuper = len(xsuper) - 1
    pcols = [[] for _ in range(n + 1)]
    for c in range(1, n + 1):
        pc = invp[c - 1]
        pcols[pc] = [invp[adj[j - 1] - 1] for j in range(xadj[c - 1], xadj[c])]
    children = [[] for _ in range(nsuper + 1)]
    xlindx = [1]
    lindx = []
    struct = [None] * (nsuper + 1)
    for k in range(1, nsuper + 1):
        fc, lc = xsuper[k - 1], xsuper[k] - 1
        w = lc - fc + 1
        rows = set(range(fc, lc + 1))
        for ch in children[k]:
            cw = xsuper[ch] - xsuper[ch - 1]
            rows.update(struct[ch][cw:])
        for col in range(fc, lc + 1):
            rows.update(r for r in pcols[col] if r > fc)
        srt = sorted(rows)
        if len(srt) != cc[fc - 1]:
            raise AssertionError(f"supernode {k}: {len(srt)} rows, column count {cc[fc - 1]}")
        struct[k] = srt
        lindx.extend(srt)
        xlindx.append(len(lindx) + 1)
        if len(srt) > w:
            pcol = poparent[lc - 1]
            children[sup[pcol - 1]].append(k)
    return xlindx, lindx


def build_cells(xsuper, xlindx, lindx, sup):
    """Reference cell / block construction order: I descending, K ascending."""
    nsuper = len(xsuper) - 1
    cells = []   # (I, K, nrows, [(first_row, nrows), ...])
    for I in range(nsuper, 0, -1):
        rows = lindx[xlindx[I - 1] - 1:xlindx[I] - 1]
        cur = None
        for r in rows:
            K = sup[r - 1]
            if cur is None or cur[1] != K:
                cur = [I, K, 0, []]
                cells.append(cur)
            if cur[3] and cur[3][-1][0] + cur[3][-1][1] == r:
                cur[3][-1][1] += 1
            else:
                cur[3].append([r, 1])
            cur[2] += 1
    return cells


def symbolic_chain(n, colptr, rowind, ordering="MMD", relax=None, order_fn=None):
    """SymbolicFactorization (symPACKMatrix2D.hpp:2699-3081) on a 1-based lower CSC.

    order_fn(n, xadj, adj) -> invp replaces the ordering routine of `ordering`
    (used to run the reference's own compiled ordering in place of the Python one)."""
    relax = relax or {}
    xadj, adj = expand_symmetric(n, colptr, rowind)
    if ordering in ("MMD", "RCM", "AMD"):
        sx, sa = set_keep_diag(n, xadj, adj, False)
        fn = order_fn or {"MMD": genmmd, "RCM": genrcm, "AMD": amdbar}[ordering]
        invp = [int(i) for i in fn(n, sx, sa)]
        gx, ga = set_keep_diag(n, sx, sa, True)
    elif ordering == "NATURAL":
        invp = list(range(1, n + 1))
        gx, ga = xadj, adj
    else:
        raise ValueError(ordering)
    mmd_invp = list(invp)
    perm = [0] * n
    for i in range(1, n + 1):
        perm[invp[i - 1] - 1] = i
    parent = construct_etree(n, gx, ga, perm, invp)
    po = postorder_tree(parent, perm, invp)
    cc = lcol_row_count(n, gx, ga, perm, invp, po)
    if ordering != "NATURAL":
        po, cc = sort_children(po, cc, perm, invp)
    cc_fund = list(cc)
    sup, xsuper = find_supernodes(po, cc, relax.get("maxSize", 0))
    if relax.get("nrelax0", 8) > 0:
        cc, sup, xsuper = relax_supernodes(po, cc, sup, xsuper,
                                           nrelax0=relax.get("nrelax0", 8), nrelax1=relax.get("nrelax1", 32),
                                           nrelax2=relax.get("nrelax2", 64), max_size=relax.get("maxSize", 0))
    xlindx, lindx = symbolic_factor(n, xadj, adj, invp, po, cc, xsuper, sup)
    return dict(perm=np.array(perm, np.int32), invp=np.array(invp, np.int32),
                mmd_invp=np.array(mmd_invp, np.int32), parent=np.array(po, np.int32),
                cc_fund=np.array(cc_fund, np.int32), cc=np.array(cc, np.int32),
                xsuper=np.array(xsuper, np.int32), supmember=np.array(sup, np.int32),
                xlindx=np.array(xlindx, np.int64), lindx=np.array(lindx, np.int32),
                flops_stat=float(sum(float(c) * c for c in cc_fund)), nnzL_stat=int(sum(cc_fund)))


def reference_symbolic(n, colptr, rowind):
    """MMD symbolic analysis computed by the oracle alone: the executed reference
    MMD (oracle/_ref/libmmd_ref.so, built from src/ordmmd.F and friends) when that
    library exists, else the Python restatement, then the Python chain above.
    Returns the arrays the numeric oracle takes plus the reference's statistics
    (flops = sum of squared fundamental column counts, symPACKMatrix2D.hpp:3009-3016)."""
    from . import mmd_reference
    order_fn = None
    if mmd_reference.OUT_SO.exists():
        order_fn = lambda nn, x, a: mmd_reference.ordmmd(nn, np.asarray(x, np.int32), np.asarray(a, np.int32))
    d = symbolic_chain(n, colptr, rowind, "MMD", order_fn=order_fn)
    sym = dict(xsuper=d["xsuper"], xlindx=d["xlindx"], lindx=d["lindx"], supmember=d["supmember"], invp=d["invp"])
    return sym, d["flops_stat"], d["nnzL_stat"]
