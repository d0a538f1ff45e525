"""Generate tests/golden/doci_maps.npz from hilbert's own compiled v2RDM-DOCI
code.

Requires oracle/_ref/libdoci_ref.so (oracle/build_ref.sh, which compiles the
reference's src/v2rdm_doci sources in place).  Each case stores seeded
integrals and inputs with the reference's outputs: block dims, b, c, the
random guess, A.x, A^T.y and the packed densities of PackSpatialDensity.
Run from the repository root:

    python tests/golden/make_doci_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.doci import DociRef, symmetric_integrals  # noqa: E402

# (name, n, nalpha, nbeta, positivity)
CASES = [
    ("doci3_d", 3, 1, 1, "D"),
    ("doci4_dq", 4, 2, 2, "DQ"),
    ("doci4_dg", 4, 2, 2, "DG"),
    ("doci5_dqg", 5, 2, 2, "DQG"),
    ("doci4_dqgt1", 4, 2, 2, "DQGT1"),
    ("doci4_dqgt2", 4, 2, 2, "DQGT2"),
    ("doci5_dqgt1t2", 5, 3, 3, "DQGT1T2"),
    ("doci4_dqg_d3", 4, 2, 2, "DQG+D3"),
    ("doci5_dqgt1t2_d3", 5, 2, 2, "DQGT1T2+D3"),
]


def main():
    rng = np.random.default_rng(20260312)
    out = {}
    for name, n, na, nb, pos in CASES:
        h, g = symmetric_integrals(rng, n)
        r = DociRef(n, na, nb, pos, h=h, g=g)
        x = rng.standard_normal(r.n_primal)
        y = rng.standard_normal(r.n_dual)
        meta = np.array([n, na, nb], dtype=np.int64)
        out.update({f"{name}/meta": meta, f"{name}/positivity": np.array(pos),
                    f"{name}/dims": r.dims, f"{name}/h": h, f"{name}/g": g,
                    f"{name}/b": r.b, f"{name}/c": r.c, f"{name}/x0": r.x0,
                    f"{name}/x": x, f"{name}/Ax": r.Au(x), f"{name}/y": y, f"{name}/ATy": r.ATu(y)})
        pd2, pd1 = r.pack_spatial_density(x)   # PackSpatialDensity of the same x
        out.update({f"{name}/pd2": pd2, f"{name}/pd1": pd1})
        r.close()
    path = os.path.join(ROOT, "tests", "golden", "doci_maps.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(CASES)} cases")


if __name__ == "__main__":
    main()
