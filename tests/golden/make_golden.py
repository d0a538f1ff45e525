"""Generate tests/golden/v2rdm_maps.npz from hilbert's own compiled map code.

Requires oracle/_ref/libv2rdm_ref.so (oracle/build_ref.sh, which compiles the
reference sources in place).  Each case stores seeded inputs and the
reference's outputs: block dims, geminal tables, b, c, the random and HF
guesses, A.x and A^T.y.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.maps import RefProblem  # noqa: E402

# (name, n, na, nb, positivity, constrain_spin, constrain_sz, hubbard (t, U) or None)
CASES = [
    ("hub2_dqg", 2, 1, 1, "DQG", True, True, (1.0, 4.0)),
    ("hub4_dqg", 4, 2, 2, "DQG", True, True, (1.0, 4.0)),
    ("hub4_d_nospin", 4, 2, 2, "D", False, True, (1.0, 2.0)),
    ("ext3_dqg_triplet", 3, 2, 1, "DQG", True, True, None),
    ("ext4_dq_nosz", 4, 2, 2, "DQ", True, False, None),
    ("ext4_dg_doublet", 4, 2, 1, "DG", True, False, None),
    ("ext5_dqg", 5, 3, 3, "DQG", True, True, None),
    ("ext1_dqg", 1, 1, 0, "DQG", True, True, None),
    ("hub3_dqgt2", 3, 1, 1, "DQGT2", True, True, (1.0, 4.0)),
    ("ext3_dqgt2_doublet", 3, 2, 1, "DQGT2", True, True, None),
    ("hub4_dqgt1", 4, 2, 2, "DQGT1", True, True, (1.0, 4.0)),
    ("ext4_dqgt1t2_doublet", 4, 2, 1, "DQGT1T2", True, True, None),
    ("hub4_dqg_d3", 4, 2, 2, "DQG+D3", True, True, (1.0, 4.0)),
    ("ext3_d_d3_nosz_doublet", 3, 2, 1, "D+D3", True, False, None),
    ("ext3_dqg_q3_doublet", 3, 2, 1, "DQG+Q3", True, True, None),
    ("hub3_d_e3", 3, 1, 1, "D+E3", True, True, (1.0, 4.0)),
    ("ext3_d_f3_doublet", 3, 2, 1, "D+F3", True, True, None),
    ("ext4_d_d4_quartet", 4, 4, 3, "D+D4", True, True, None),
]


def main(out=os.path.join(ROOT, "tests", "golden", "v2rdm_maps.npz")):
    data = {}
    for k, (name, n, na, nb, pos, spin, sz, hub) in enumerate(CASES):
        rng = np.random.default_rng(1000 + k)
        kw = {}
        if hub is None:
            h = rng.standard_normal((n, n))
            g = rng.standard_normal((n, n, n, n))
            kw = dict(h=h, g=g)
            data[f"{name}/h"] = h
            data[f"{name}/g"] = g
        else:
            kw = dict(hubbard=hub)
        r = RefProblem(n, na, nb, pos, spin, sz, **kw)
        rh = RefProblem(n, na, nb, pos, spin, sz, guess="hf", **kw)
        x = rng.standard_normal(r.n_primal)
        y = rng.standard_normal(r.n_dual)
        bas_ab, ibas_ab, bas_aa, ibas_aa = r.tables()
        data[f"{name}/spec"] = np.array([n, na, nb, spin, sz, -1 if hub is None else 1], np.int64)
        data[f"{name}/positivity"] = np.array(pos)
        data[f"{name}/hubbard"] = np.array(hub if hub is not None else (0.0, 0.0))
        data[f"{name}/dims"] = r.dims
        data[f"{name}/bas_ab"] = bas_ab
        data[f"{name}/ibas_ab"] = ibas_ab
        data[f"{name}/bas_aa"] = bas_aa
        data[f"{name}/ibas_aa"] = ibas_aa
        data[f"{name}/b"] = r.b
        data[f"{name}/c"] = r.c
        data[f"{name}/x_random"] = r.x0
        data[f"{name}/x_hf"] = rh.x0
        data[f"{name}/x"] = x
        data[f"{name}/y"] = y
        data[f"{name}/Ax"] = r.Au(x)
        data[f"{name}/ATy"] = r.ATu(y)
        print(f"{name}: n_primal={r.n_primal} n_dual={r.n_dual} dims={list(r.dims)}")
    np.savez_compressed(out, **data)
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()
