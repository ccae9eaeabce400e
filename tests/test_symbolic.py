"""Symbolic analysis: bit-exact against the reference MMD, RCM and AMD orderings (golden
fixtures made by executing the reference's Fortran), against the independent
Python oracle, and against mathematical definitions (structure of the dense
Cholesky factor)."""
import hashlib
import os

import numpy as np
import pytest

from oracle import symbolic_oracle as so
from sympack_b200 import DistSparseMatrix, RelaxationParameters, generators as G, symPACKMatrix2D, symPACKOptions

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mmd_golden.npz")
GOLDEN_RCM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rcm_golden.npz")
GOLDEN_AMD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "amd_golden.npz")


def analyze(n, cp, ri, **opt):
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, np.zeros(len(ri)))
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=-1, **opt))
    M.SymbolicFactorization(A)
    perm, invp = M.GetOrdering()
    fund, rel = M.GetColCounts()
    xl, li = M.GetStructure()
    return dict(M=M, mmd_invp=M.GetMMDInvp(), perm=perm, invp=invp, parent=M.GetETree(), cc_fund=fund, cc=rel,
                xsuper=M.GetSupernodalPartition(), supmember=M.GetSupMembership(), xlindx=xl, lindx=li)


def golden_cases(path=GOLDEN):
    g = np.load(path)
    names = sorted({k.split("/")[0] for k in g.files if k.endswith("/invp")})
    return [(nm, g[f"{nm}/colptr"], g[f"{nm}/rowind"], g[f"{nm}/invp"]) for nm in names]


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c[0])
def test_mmd_matches_reference_fortran(case):
    name, cp, ri, invp = case
    n = len(cp) - 1
    assert np.array_equal(analyze(n, cp, ri)["mmd_invp"], invp)


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c[0])
def test_oracle_mmd_matches_reference_fortran(case):
    name, cp, ri, invp = case
    n = len(cp) - 1
    xadj, adj = so.expand_symmetric(n, cp, ri)
    sx, sa = so.set_keep_diag(n, xadj, adj, False)
    assert np.array_equal(np.array(so.genmmd(n, sx, sa)), invp)


@pytest.mark.parametrize("name,gen", [("lap3d_60", lambda: G.laplacian_3d(60, 60, 60, 1e-3)),
                                      ("st27_80", lambda: G.stencil27(80, 80, 80, 1e-2))])
def test_mmd_full_size_matches_reference_hash(name, gen):
    g = np.load(GOLDEN)
    n, cp, ri, _ = gen()
    inv = analyze(n, cp, ri)["mmd_invp"]
    assert np.array_equal(inv[:64], g[f"{name}/invp_head"])
    assert hashlib.sha256(inv.astype("<i4").tobytes()).digest() == g[f"{name}/invp_sha256"].tobytes()


@pytest.mark.parametrize("case", golden_cases(GOLDEN_RCM), ids=lambda c: c[0])
def test_rcm_matches_reference_fortran(case):
    name, cp, ri, invp = case
    n = len(cp) - 1
    assert np.array_equal(analyze(n, cp, ri, orderingStr="RCM")["mmd_invp"], invp)


@pytest.mark.parametrize("case", golden_cases(GOLDEN_RCM), ids=lambda c: c[0])
def test_oracle_rcm_matches_reference_fortran(case):
    name, cp, ri, invp = case
    n = len(cp) - 1
    xadj, adj = so.expand_symmetric(n, cp, ri)
    sx, sa = so.set_keep_diag(n, xadj, adj, False)
    assert np.array_equal(np.array(so.genrcm(n, sx, sa)), invp)


@pytest.mark.parametrize("name,gen", [("lap3d_60", lambda: G.laplacian_3d(60, 60, 60, 1e-3)),
                                      ("st27_80", lambda: G.stencil27(80, 80, 80, 1e-2))])
def test_rcm_full_size_matches_reference_hash(name, gen):
    g = np.load(GOLDEN_RCM)
    n, cp, ri, _ = gen()
    inv = analyze(n, cp, ri, orderingStr="RCM")["mmd_invp"]
    assert np.array_equal(inv[:64], g[f"{name}/invp_head"])
    assert hashlib.sha256(inv.astype("<i4").tobytes()).digest() == g[f"{name}/invp_sha256"].tobytes()


@pytest.mark.parametrize("case", golden_cases(GOLDEN_AMD), ids=lambda c: c[0])
def test_amd_matches_reference_fortran(case):
    name, cp, ri, invp = case
    n = len(cp) - 1
    assert np.array_equal(analyze(n, cp, ri, orderingStr="AMD")["mmd_invp"], invp)


@pytest.mark.parametrize("case", golden_cases(GOLDEN_AMD), ids=lambda c: c[0])
def test_oracle_amd_matches_reference_fortran(case):
    name, cp, ri, invp = case
    n = len(cp) - 1
    xadj, adj = so.expand_symmetric(n, cp, ri)
    sx, sa = so.set_keep_diag(n, xadj, adj, False)
    assert np.array_equal(np.array(so.amdbar(n, sx, sa)), invp)


@pytest.mark.parametrize("name,gen", [("lap3d_60", lambda: G.laplacian_3d(60, 60, 60, 1e-3)),
                                      ("st27_80", lambda: G.stencil27(80, 80, 80, 1e-2))])
def test_amd_full_size_matches_reference_hash(name, gen):
    """Full-size graphs: the workspace of nnz + n entries is compacted several times."""
    g = np.load(GOLDEN_AMD)
    n, cp, ri, _ = gen()
    inv = analyze(n, cp, ri, orderingStr="AMD")["mmd_invp"]
    assert np.array_equal(inv[:64], g[f"{name}/invp_head"])
    assert hashlib.sha256(inv.astype("<i4").tobytes()).digest() == g[f"{name}/invp_sha256"].tobytes()


def test_amd_fill_close_to_mmd():
    """Both are minimum-degree heuristics: the factor sizes agree within 15% on a 3D grid."""
    n, cp, ri, _ = G.laplacian_3d(16, 16, 16, 1e-3)
    nnz = {o: int(analyze(n, cp, ri, orderingStr=o)["cc_fund"].sum()) for o in ("MMD", "AMD")}
    assert abs(nnz["AMD"] - nnz["MMD"]) <= 0.15 * nnz["MMD"], nnz


def test_rcm_is_a_bandwidth_ordering():
    """On a 2D grid RCM numbers by level sets: the permuted bandwidth stays within
    one grid line (plus one), far below MMD's."""
    n, cp, ri, _ = G.laplacian_2d(40, 40)
    inv = analyze(n, cp, ri, orderingStr="RCM")["mmd_invp"]
    cols = np.repeat(np.arange(n), np.diff(cp))
    assert np.abs(inv[ri - 1] - inv[cols]).max() <= 41
    assert sorted(inv) == list(range(1, n + 1))


KEYS = ["mmd_invp", "perm", "invp", "parent", "cc_fund", "cc", "xsuper", "supmember", "xlindx", "lindx"]
GRAPHS = [
    ("lap2d_64", lambda: G.laplacian_2d(64, 64)),
    ("lap2d_1x50", lambda: G.laplacian_2d(1, 50)),
    ("lap3d_12", lambda: G.laplacian_3d(12, 12, 12, 1e-3)),
    ("st27_9", lambda: G.stencil27(9, 9, 9, 1e-2)),
    ("rand_1500", lambda: G.random_graph_spd(1500, 10, 1.05, seed=2)),
    ("rand_400_forest", lambda: G.random_graph_spd(400, 1.2, 1.05, seed=5)),
]


@pytest.mark.parametrize("name,gen", GRAPHS)
@pytest.mark.parametrize("ordering", ["MMD", "NATURAL", "RCM", "AMD"])
def test_symbolic_chain_matches_oracle(name, gen, ordering):
    n, cp, ri, _ = gen()
    p = analyze(n, cp, ri, orderingStr=ordering)
    o = so.symbolic_chain(n, cp, ri, ordering=ordering)
    for k in KEYS:
        assert np.array_equal(np.asarray(p[k]), np.asarray(o[k])), k
    cells = so.build_cells(list(o["xsuper"]), list(o["xlindx"]), list(o["lindx"]), list(o["supmember"]))
    pc = p["M"].GetCells()
    assert len(cells) == len(pc["I"])
    bf = []
    for i, (I, K, nr, blocks) in enumerate(cells):
        assert (I, K, nr, len(blocks)) == (pc["I"][i], pc["K"][i], pc["nrows"][i], pc["nblocks"][i])
        bf.extend(blocks)
    assert np.array_equal(np.array(bf)[:, 0], pc["block_first_row"])
    assert np.array_equal(np.array(bf)[:, 1], pc["block_nrows"])


@pytest.mark.parametrize("relax", [dict(maxSize=4), dict(nrelax0=0), dict(nrelax0=16, nrelax1=48, nrelax2=96)])
def test_relaxation_options_match_oracle(relax):
    n, cp, ri, _ = G.laplacian_3d(11, 11, 11, 1e-3)
    rp = RelaxationParameters(**{k: v for k, v in relax.items()})
    if rp.maxSize > 0:  # SetMaxSize caps the relaxation sizes (Types.hpp:63-70)
        rp.nrelax0, rp.nrelax1, rp.nrelax2 = (min(x, rp.maxSize) for x in (rp.nrelax0, rp.nrelax1, rp.nrelax2))
    p = analyze(n, cp, ri, relax=rp)
    o = so.symbolic_chain(n, cp, ri, relax=dict(nrelax0=rp.nrelax0, nrelax1=rp.nrelax1, nrelax2=rp.nrelax2,
                                                maxSize=rp.maxSize))
    for k in KEYS:
        assert np.array_equal(np.asarray(p[k]), np.asarray(o[k])), k
    w = np.diff(p["xsuper"])
    if rp.maxSize:
        fund_w = np.diff(so.find_supernodes(list(p["parent"]), list(p["cc_fund"]), rp.maxSize)[1])
        assert fund_w.max() <= rp.maxSize
    assert w.sum() == n


def dense_factor_structure(n, cp, ri, invp):
    """Nonzero pattern of the Cholesky factor of P A P^T, from numpy (values random SPD)."""
    rng = np.random.default_rng(0)
    D = np.zeros((n, n))
    cols = np.repeat(np.arange(n), np.diff(cp))
    rows = ri - 1
    off = rows != cols
    vals = np.where(off, -rng.uniform(0.1, 1.0, len(rows)), 0.0)
    D[invp[rows] - 1, invp[cols] - 1] = vals
    D = D + D.T
    D[np.diag_indices(n)] = np.abs(D).sum(1) + 1.0
    L = np.linalg.cholesky(D)
    return np.abs(L) > 1e-300


@pytest.mark.parametrize("name,gen", GRAPHS[:5])
@pytest.mark.parametrize("ordering", ["MMD", "RCM", "AMD"])
def test_etree_counts_structure_match_factor_pattern(name, gen, ordering):
    n, cp, ri, _ = gen()
    p = analyze(n, cp, ri, orderingStr=ordering)
    S = dense_factor_structure(n, cp, ri, p["invp"])
    # elimination tree: parent(j) = first off-diagonal nonzero row of column j
    for j in range(n):
        nz = np.nonzero(S[j + 1:, j])[0]
        assert p["parent"][j] == (j + 2 + nz[0] if len(nz) else 0)
    # column counts (fundamental) = nonzeros per column
    assert np.array_equal(p["cc_fund"], S.sum(0))
    # row structure of each (relaxed) supernode = union of its columns' patterns
    xs, xl, li = p["xsuper"], p["xlindx"], p["lindx"]
    for s in range(len(xs) - 1):
        fc, lc = xs[s] - 1, xs[s + 1] - 1
        union = np.nonzero(S[:, fc:lc].any(1))[0]
        union = np.union1d(union, np.arange(fc, lc))
        assert np.array_equal(li[xl[s] - 1:xl[s + 1] - 1] - 1, union[union >= fc])


def test_permutation_is_postorder_of_etree():
    n, cp, ri, _ = G.laplacian_3d(10, 10, 10, 1e-3)
    p = analyze(n, cp, ri)
    par = p["parent"]
    assert np.array_equal(np.sort(p["perm"]), np.arange(1, n + 1))
    assert np.array_equal(p["perm"][p["invp"] - 1], np.arange(1, n + 1))
    nz = par > 0
    assert np.all(par[nz] > np.arange(1, n + 1)[nz])  # parents numbered after children
    # subtrees are contiguous: descendants of j occupy [j - size(j) + 1, j]
    size = np.ones(n + 1, np.int64)
    for j in range(1, n + 1):
        if par[j - 1]:
            size[par[j - 1]] += size[j]
    first = np.arange(1, n + 1) - size[1:] + 1
    for j in range(1, n + 1):
        if par[j - 1]:
            assert first[par[j - 1] - 1] <= first[j - 1]


@pytest.mark.parametrize("bad", ["upper", "unsorted", "zero_based", "duplicate"])
def test_invalid_structure_rejected(bad):
    n, cp, ri, v = G.laplacian_2d(5, 5)
    ri = ri.copy()
    cp = cp.copy()
    if bad == "upper":
        ri[cp[3] - 1] = 1
    elif bad == "unsorted":
        a, b = cp[2] - 1, cp[2]
        ri[a], ri[b] = ri[b], ri[a]
    elif bad == "zero_based":
        cp = cp - 1
    elif bad == "duplicate":
        ri[cp[2]] = ri[cp[2] - 1]
    with pytest.raises(ValueError):
        analyze(n, cp, ri)


def test_statistics_match_reference_formula():
    n, cp, ri, _ = G.laplacian_2d(64, 64)
    p = analyze(n, cp, ri)
    inf = p["M"].info()
    assert inf.flops_stat == float(np.sum(p["cc_fund"].astype(np.float64) ** 2))
    assert inf.nnz_l == int(p["cc_fund"].sum())
    assert inf.nsuper == len(p["xsuper"]) - 1


TINY = {
    "n1": (1, [1, 2], [1]),
    "diag5": (5, [1, 2, 3, 4, 5, 6], [1, 2, 3, 4, 5]),
    "path2": (2, [1, 3, 4], [1, 2, 2]),
}
# invp the reference Fortran (ordmmd / amdbar / genrcm) returns for these graphs
TINY_INVP = {
    ("n1", "MMD"): [1], ("n1", "AMD"): [1], ("n1", "RCM"): [1],
    ("diag5", "MMD"): [5, 4, 3, 2, 1], ("diag5", "AMD"): [1, 2, 3, 4, 5], ("diag5", "RCM"): [1, 2, 3, 4, 5],
    ("path2", "MMD"): [2, 1], ("path2", "AMD"): [1, 2], ("path2", "RCM"): [2, 1],
}


@pytest.mark.parametrize("case,ordering", sorted(TINY_INVP), ids=lambda x: x if isinstance(x, str) else None)
def test_tiny_and_edgeless_graphs(case, ordering):
    """One vertex, vertices without edges, a single edge: the orderings' degenerate paths."""
    n, cp, ri = TINY[case]
    p = analyze(n, np.array(cp, np.int64), np.array(ri, np.int32), orderingStr=ordering)
    assert list(p["mmd_invp"]) == TINY_INVP[(case, ordering)]
    assert sorted(p["perm"]) == list(range(1, n + 1))
