"""Batched instances on the B200: rings solved together in one BatchProblem
(every launch covers all of them) against each ring solved alone."""
import numpy as np
import pytest

from hilbert_b200.batch import RingInstance, solve_in_one_launch, solve_on_device
from hilbert_b200.v2rdm import Options

pytestmark = pytest.mark.gpu


def test_rings_in_one_launch_match_each_alone(cuda_device):
    # five electrons on five sites (odd N) take the external-Hamiltonian path
    rings = [RingInstance(0, 4, 4, 4.0), RingInstance(1, 5, 5, 2.0), RingInstance(2, 6, 6, 6.0),
             RingInstance(3, 5, 4, 3.0)]
    opts = Options({"R_CONVERGENCE": 1e-7, "E_CONVERGENCE": 1e-7, "MAXITER": 400000,
                    "MU_UPDATE_FREQUENCY": 500})
    together = solve_in_one_launch(rings, opts)
    assert all(r["converged"] and r["group"] == len(rings) for r in together)
    for ring, r in zip(rings, together):
        alone = solve_on_device(ring, opts)
        assert alone["converged"]
        assert abs(r["energy"] - alone["energy"]) <= 1e-6, (ring, r["energy"], alone["energy"])
