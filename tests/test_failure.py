"""Failure detection on the host: non-finite inputs are refused before any
device work, with the vector and index named (no GPU needed)."""
import numpy as np
import pytest

import hilbert_b200 as hb
from hilbert_b200 import _capi


@pytest.mark.parametrize("which", ["x", "b", "c"])
def test_nonfinite_host_input_is_refused(which):
    p = hb.V2RDMProblem(4, 2, 2, "DQG", hubbard_multiplicity=True)
    x, b, c = p.guess("RANDOM"), p.b(), p.c_hubbard(1.0, 4.0)
    arr = {"x": x, "b": b, "c": c}[which]
    arr[7] = np.nan if which != "b" else np.inf
    opts = hb.Options({"MAXITER": 10})
    with pytest.raises(_capi.V2BError) as e:
        p.solve(x, b, c, opts)
    assert e.value.code == _capi.V2B_NAN
    assert f"non-finite value in {which} at index 7" in str(e.value)
    p.close()


def test_wait_limit_argument_checks():
    p = hb.V2RDMProblem(3, 1, 1, "DQG")
    p.set_wait_limit(1000)
    p.set_wait_limit(0)
    with pytest.raises(_capi.V2BError) as e:
        p.set_wait_limit(-1)
    assert e.value.code == _capi.V2B_BAD_ARG
    with pytest.raises(_capi.V2BError) as e:
        p.continue_state()   # no device solve has run
    assert e.value.code == _capi.V2B_BAD_ARG
    p.close()
