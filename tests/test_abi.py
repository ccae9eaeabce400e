"""The C-ABI library loads and exports every entry point include/*.h declares;
host-only handles give the documented status codes (no GPU needed)."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from sympack_b200 import DistSparseMatrix, StateError, generators as G, symPACKMatrix2D, symPACKOptions
from sympack_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names.update(re.findall(r"\b(spb_\w+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = N.load()
    decl = declared_symbols()
    assert len(decl) >= 20
    for name in decl:
        assert hasattr(lib, name), name
    assert set(N.exported_symbols()) >= set(decl)


def test_host_only_handle_rejects_numeric_calls():
    n, cp, ri, v = G.laplacian_2d(8, 8)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=-1))
    M.SymbolicFactorization(A)
    for call in (lambda: M.DistributeMatrix(A), M.Factorize, lambda: M.Solve(np.ones(n)),
                 M.ReorderFactorFromTrace, lambda: M.SetFactorTrace(True)):
        with pytest.raises(StateError):
            call()


def test_calls_out_of_order():
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=-1))
    with pytest.raises(StateError):
        M.info()


def test_bad_options():
    with pytest.raises(ValueError):
        symPACKMatrix2D().Init(symPACKOptions(orderingStr="METIS"))
    with pytest.raises(ValueError):
        symPACKMatrix2D().Init(symPACKOptions(orderingStr="USER"))


def test_fp32_engine_option_is_validated():
    from sympack_b200 import symPACKMatrix2D, symPACKOptions
    for eng in ("tcgen05", "mma.sync", "tcgen05-persistent", "tcgen05-tma"):
        M = symPACKMatrix2D()
        M.Init(symPACKOptions(device=-1, fp32_engine=eng))
        M.close()
    with pytest.raises(ValueError):
        symPACKMatrix2D().Init(symPACKOptions(device=-1, fp32_engine="wmma"))


def test_factor_schedule_option_is_validated():
    for sched in ("auto", "persistent", "steps"):
        for prec in ("FP64", "FP32_IR"):
            M = symPACKMatrix2D()
            M.Init(symPACKOptions(device=-1, factor_schedule=sched, precision=prec))
            M.close()
    with pytest.raises(ValueError):
        symPACKMatrix2D().Init(symPACKOptions(device=-1, factor_schedule="eager"))
    o = N.spb_options()
    N.load().spb_default_options(C.byref(o))
    assert o.factor_schedule == 0 and o.fp32_engine == 3  # auto schedule, TMA-fed FP32 tiles
    o.factor_schedule = 3
    h = C.c_void_p()
    assert N.load().spb_create(C.byref(o), C.byref(h)) == -1  # SPB_ERR_INVALID


def test_decomposition_option_is_validated():
    from sympack_b200 import symPACKMatrix2D, symPACKOptions
    for dec in ("LL", "LDL"):
        M = symPACKMatrix2D()
        M.Init(symPACKOptions(device=-1, decomposition=dec))
        M.close()
    with pytest.raises(ValueError):
        symPACKMatrix2D().Init(symPACKOptions(device=-1, decomposition="LU"))
    with pytest.raises(ValueError):  # LDL^T runs in FP64 only
        symPACKMatrix2D().Init(symPACKOptions(device=-1, decomposition="LDL", precision="FP32_IR"))


def test_ldl_footprint_adds_the_scaled_copy():
    import numpy as np
    from sympack_b200 import DistSparseMatrix, generators as G, symPACKMatrix2D, symPACKOptions
    n, cp, ri, v = G.laplacian_3d(10, 10, 10, 1e-3)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    got = {}
    for dec in ("LL", "LDL"):
        M = symPACKMatrix2D()
        M.Init(symPACKOptions(device=-1, decomposition=dec))
        M.SymbolicFactorization(A)
        got[dec] = (M.PredictDeviceBytes(nrhs=1), M.info().arena_bytes, M.info().inverse_bytes)
        M.close()
    # one more FP64 arena (L D) and the inverses of its diagonal super-blocks
    assert got["LDL"][0] - got["LL"][0] == got["LL"][1] + got["LL"][2]


def test_host_only_analysis_predicts_footprint_and_is_reusable():
    import numpy as np
    from sympack_b200 import DistSparseMatrix, generators as G, symPACKMatrix2D, symPACKOptions
    n, cp, ri, v = G.laplacian_2d(20, 20)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    T = symPACKMatrix2D()
    T.Init(symPACKOptions(device=-1))
    T.SymbolicFactorization(A)
    b64, b32 = T.PredictDeviceBytes("FP64", 1), T.PredictDeviceBytes("FP32_IR", 1)
    assert b64 > T.info().arena_bytes > 0 and b32 > 0
    assert T.PredictDeviceBytes("FP64", 64) > b64  # right-hand-side buffers grow with nrhs
    M = symPACKMatrix2D()
    M.Init(symPACKOptions(device=-1))
    M.SymbolicFactorizationFrom(T)
    assert np.array_equal(M.GetSupernodalPartition(), T.GetSupernodalPartition())
    assert np.array_equal(M.GetOrdering()[0], T.GetOrdering()[0])
    with pytest.raises(ValueError):  # different relaxation: the analysis is not reusable
        R = symPACKMatrix2D()
        from sympack_b200 import RelaxationParameters
        R.Init(symPACKOptions(device=-1, relax=RelaxationParameters(nrelax0=4)))
        R.SymbolicFactorizationFrom(T)


def test_footprint_prediction_follows_the_target_precision_and_engine():
    """The plan depends on the precision (tile shapes, task graph), so a host-only analysis
    predicts the same footprint for a precision whatever precision it was made in; the
    TMA-fed FP32 tiles add split copies of the panels (at most two more FP32 arenas)."""
    n, cp, ri, v = G.stencil27(14, 14, 14, 1e-2)
    A = DistSparseMatrix.from_lower_csc(n, cp, ri, v)
    got = {}
    for prec in ("FP64", "FP32_IR"):
        for eng in ("tcgen05-tma", "tcgen05"):
            T = symPACKMatrix2D()
            T.Init(symPACKOptions(device=-1, precision=prec, fp32_engine=eng))
            T.SymbolicFactorization(A)
            got[(prec, eng)] = (T.PredictDeviceBytes("FP64", 1), T.PredictDeviceBytes("FP32_IR", 1),
                                T.info().arena_bytes, T.info().nsuper)
            T.close()
    for eng in ("tcgen05-tma", "tcgen05"):
        assert got[("FP64", eng)][:2] == got[("FP32_IR", eng)][:2]
    fp64_tma, fp32_tma, arena, ns = got[("FP64", "tcgen05-tma")]
    assert got[("FP64", "tcgen05")][0] == fp64_tma  # the FP32 engine does not change an FP64 footprint
    extra = fp32_tma - got[("FP64", "tcgen05")][1]
    assert 0 < extra <= arena + 256 * ns  # two FP32 copies = one FP64 arena, plus maps and alignment
