"""Generate the golden fixtures of tests/golden/ from the reference's own MMD, RCM
and AMD Fortran, executed here through oracle/mmd_reference.py (translated from
the reference sources and compiled with gcc).  Run in the development container:

    python tests/golden/make_golden.py [mmd] [rcm] [amd]

mmd_golden.npz / rcm_golden.npz / amd_golden.npz hold, per case, the input graph (lower CSC of a
seeded generator) and the invp the reference ordering returns for it; for the
full-size configurations they hold the SHA-256 of that invp instead.
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import mmd_reference as mr, symbolic_oracle as so  # noqa: E402
from sympack_b200 import generators as G  # noqa: E402

SMALL = {
    "lap2d_64": lambda: G.laplacian_2d(64, 64),
    "lap2d_7x13": lambda: G.laplacian_2d(7, 13),
    "lap3d_12": lambda: G.laplacian_3d(12, 12, 12, 1e-3),
    "lap3d_5x7x3": lambda: G.laplacian_3d(5, 7, 3, 1e-3),
    "st27_9": lambda: G.stencil27(9, 9, 9, 1e-2),
    "rand_2000": lambda: G.random_graph_spd(2000, 10, 1.05, seed=1),
    "rand_300_sparse": lambda: G.random_graph_spd(300, 2.5, 1.05, seed=7),
}
FULL = {
    "lap3d_60": lambda: G.laplacian_3d(60, 60, 60, 1e-3),
    "st27_80": lambda: G.stencil27(80, 80, 80, 1e-2),
}


def ref_invp(n, cp, ri, ordering="mmd"):
    xadj, adj = so.expand_symmetric(n, cp, ri)
    sx, sa = so.set_keep_diag(n, xadj, adj, False)
    return {"mmd": mr.ordmmd, "rcm": mr.genrcm, "amd": mr.amdbar}[ordering](n, sx, sa)


RCM_EXTRA = {
    "rand_400_forest": lambda: G.random_graph_spd(400, 1.2, 1.05, seed=5),  # many components
    "lap2d_1x50": lambda: G.laplacian_2d(1, 50),
}


def write(ordering):
    out = {}
    cases = dict(SMALL, **(RCM_EXTRA if ordering != "mmd" else {}))
    for name, gen in cases.items():
        n, cp, ri, _ = gen()
        out[f"{name}/colptr"] = cp
        out[f"{name}/rowind"] = ri
        out[f"{name}/invp"] = ref_invp(n, cp, ri, ordering)
    for name, gen in FULL.items():
        n, cp, ri, _ = gen()
        inv = ref_invp(n, cp, ri, ordering)
        out[f"{name}/invp_sha256"] = np.frombuffer(hashlib.sha256(inv.astype("<i4").tobytes()).digest(), np.uint8)
        out[f"{name}/invp_head"] = inv[:64]
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"{ordering}_golden.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    for ordering in (sys.argv[1:] or ["mmd", "rcm", "amd"]):
        write(ordering)
