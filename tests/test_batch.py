"""Batching form, host side: the merged symbolic analysis of a block-diagonal
batch equals each system's own analysis, shifted by the system's offset."""
import numpy as np
import pytest

from sympack_b200 import DistSparseMatrix, generators as G, symPACKMatrix2D, symPACKOptions


def analysis(M):
    perm, invp = M.GetOrdering()
    fund, rel = M.GetColCounts()
    xl, li = M.GetStructure()
    return dict(mmd_invp=M.GetMMDInvp(), perm=perm, invp=invp, parent=M.GetETree(), cc_fund=fund, cc=rel,
                xsuper=M.GetSupernodalPartition(), supmember=M.GetSupMembership(), xlindx=xl, lindx=li)


def single(n, cp, ri, **opt):
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=-1, **opt))
    M.SymbolicFactorization(DistSparseMatrix.from_lower_csc(n, cp, ri, np.zeros(len(ri))))
    return analysis(M), M.info()


def batched(systems, **opt):
    n, cp, ri, v, offs = G.block_diagonal(systems)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=-1, **opt))
    M.SymbolicFactorizationBatch(DistSparseMatrix.from_lower_csc(n, cp, ri, v), offs)
    return analysis(M), M.info(), offs


@pytest.mark.parametrize("ordering", ["MMD", "NATURAL"])
def test_batch_symbolic_is_concatenation_of_singles(ordering):
    systems = G.batch_systems(12, 40, 900, seed=3)
    b, binfo, offs = batched(systems, orderingStr=ordering)
    shift = {"mmd_invp": "row", "perm": "row", "invp": "row", "parent": "parent", "cc_fund": None, "cc": None,
             "supmember": "sn", "lindx": "row"}
    acc = {k: [] for k in shift}
    xs, xl = [np.array([1])], [np.array([1], np.int64)]
    nsn, nl, flops, nnzl = 0, 0, 0.0, 0
    for k, s in enumerate(systems):
        a, info = single(*s[:3], orderingStr=ordering)
        o = int(offs[k])
        for key, how in shift.items():
            x = np.asarray(a[key]).astype(np.int64)
            if how == "row":
                x = x + o
            elif how == "parent":
                x = np.where(x > 0, x + o, 0)
            elif how == "sn":
                x = x + nsn
            acc[key].append(x)
        xs.append(np.asarray(a["xsuper"][1:]) + o)
        xl.append(np.asarray(a["xlindx"][1:]) + nl)
        nsn += len(a["xsuper"]) - 1
        nl += len(a["lindx"])
        flops += info.flops_stat
        nnzl += info.nnz_l
    for key in shift:
        assert np.array_equal(np.asarray(b[key]), np.concatenate(acc[key])), key
    assert np.array_equal(b["xsuper"], np.concatenate(xs))
    assert np.array_equal(b["xlindx"], np.concatenate(xl))
    assert binfo.nsuper == nsn and binfo.nnz_l == nnzl
    assert binfo.flops_stat == pytest.approx(flops, rel=1e-15)


def test_batch_height_is_tallest_system():
    systems = G.batch_systems(8, 50, 2000, seed=4)
    _, binfo, _ = batched(systems)
    assert binfo.nlevels == max(single(*s[:3])[1].nlevels for s in systems)


def test_batch_of_one_equals_single():
    s = G.laplacian_2d(30, 17)
    a, _ = single(*s[:3])
    b, _, _ = batched([s])
    for k in a:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


def test_batch_rejects_coupled_systems():
    systems = [G.laplacian_2d(5, 5), G.laplacian_2d(4, 6)]
    n, cp, ri, v, offs = G.block_diagonal(systems)
    ri = ri.copy()
    # last entry of system 0's first column -> a row of system 1
    ri[cp[1] - 2] = offs[1] + 2
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=-1))
    with pytest.raises(ValueError, match="couples"):
        M.SymbolicFactorizationBatch(DistSparseMatrix.from_lower_csc(n, cp, ri, v), offs)


@pytest.mark.parametrize("offs", [[0, 25, 40], [1, 25, 49], [0, 25, 25, 49], [0, 49]])
def test_batch_rejects_bad_offsets(offs):
    systems = [G.laplacian_2d(5, 5), G.laplacian_2d(4, 6)]
    n, cp, ri, v, good = G.block_diagonal(systems)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=-1))
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    if offs == [0, 49]:  # one system covering both blocks is valid (a forest of two trees)
        M.SymbolicFactorizationBatch(A, offs)
        return
    with pytest.raises(ValueError):
        M.SymbolicFactorizationBatch(A, offs)


def test_batch_user_ordering_rejected():
    systems = [G.laplacian_2d(5, 5)]
    n, cp, ri, v, offs = G.block_diagonal(systems)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=-1, orderingStr="USER", perm=np.arange(1, n + 1)))
    with pytest.raises(ValueError):
        M.SymbolicFactorizationBatch(DistSparseMatrix.from_lower_csc(n, cp, ri, v), offs)
