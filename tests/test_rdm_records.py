"""The density-matrix records hilbert writes after a solve (WriteTPDM,
WriteTPDMSpinFree, WriteOPDM), from the product library against what the
reference's own compiled writers emit into the PSIO stand-in."""
import itertools
import os

import numpy as np
import pytest

import hilbert_b200 as hb
from oracle.maps import ref_available

pytestmark = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")


def cases():
    for n, na, nb in itertools.product([1, 2, 3, 4], [0, 1, 2, 3], [0, 1, 2]):
        if na <= n and nb <= n:
            yield n, na, nb


@pytest.mark.parametrize("ncore", [0, 1, 3])
def test_rdm_entries_match_the_reference_writers(ncore):
    """Every record and every metadata entry, byte for byte, with and without
    restricted doubly occupied orbitals."""
    from oracle.maps import RefProblem
    rng = np.random.default_rng(17 + ncore)
    for n, na, nb in cases():
        r = RefProblem(n, na, nb, "DQG", True, True, h=rng.standard_normal((n, n)),
                       g=rng.standard_normal((n,) * 4))
        x = rng.standard_normal(r.n_primal)
        _, ref_entries = r.write_rdms(x, ncore)
        p = hb.V2RDMProblem(n, na, nb, "DQG")
        mine = p.rdm_entries(x, ncore)
        assert set(mine) == set(ref_entries)
        for name, entries in ref_entries.items():
            assert set(mine[name]) == set(entries), (ncore, name)
            for key, val in entries.items():
                assert mine[name][key] == val, (n, na, nb, ncore, name, key)
        p.close()


def test_spin_free_sign_follows_the_reference():
    """WriteTPDMSpinFree signs the aa and bb terms -1 when either pair is
    reversed (write_tpdm.cc:349-351), so an element with both pairs reversed
    differs from the spin sum of the D2aa/D2bb records."""
    p = hb.V2RDMProblem(3, 1, 1, "D")
    rng = np.random.default_rng(1)
    x = rng.standard_normal(p.n_primal)
    rec = p.rdm_records(x)
    d2, aa, bb, ab = rec["D2"], rec["D2aa"], rec["D2bb"], rec["D2ab"]
    key = lambda r: (int(r["i"]), int(r["j"]), int(r["k"]), int(r["l"]))
    vab = {key(r): r["value"] for r in ab}
    vaa = {key(r): r["value"] for r in aa}
    vbb = {key(r): r["value"] for r in bb}
    for r in d2:
        i, j, k, l = key(r)
        if i == j or k == l:
            continue
        sum_spin = vab[(i, j, k, l)] + vab[(j, i, l, k)] + vaa[(i, j, k, l)] + vbb[(i, j, k, l)]
        if i > j and k > l:
            assert r["value"] != pytest.approx(sum_spin)
        else:
            assert r["value"] == pytest.approx(sum_spin, abs=1e-12)


def test_rdm_files_round_trip(tmp_path):
    p = hb.V2RDMProblem(3, 2, 1, "DQG")
    x = np.random.default_rng(2).standard_normal(p.n_primal)
    path = os.path.join(tmp_path, "rdms.npz")
    p.write_rdm_files(path, x)
    assert hb.V2RDMProblem.read_rdm_files(path) == p.rdm_entries(x)
    d = hb.DOCIProblem(3, 1, 1, "DQG")   # DOCI writes the three spin blocks only
    assert set(d.rdm_records(np.zeros(d.n_primal))) == {"D2aa", "D2bb", "D2ab"}


@pytest.mark.parametrize("ncore", [0, 2])
def test_iwl_records_match_the_reference_iwl_writer(ncore):
    """WriteTPDM_IWL's write_value calls, in order: labels and values."""
    from oracle.maps import RefProblem
    rng = np.random.default_rng(19 + ncore)
    for n, na, nb in cases():
        r = RefProblem(n, na, nb, "DQG", True, True, h=rng.standard_normal((n, n)),
                       g=rng.standard_normal((n,) * 4))
        x = rng.standard_normal(r.n_primal)
        r.write_rdms(x, ncore)
        want, cutoff = r.iwl_records()
        assert cutoff == 1e-14
        p = hb.V2RDMProblem(n, na, nb, "DQG")
        got = p.tpdm_iwl_records(x, ncore)
        for name, (labels, values) in want.items():
            g = got[name]
            assert np.array_equal(np.stack([g["i"], g["j"], g["k"], g["l"]], axis=1), labels), (n, name)
            assert np.array_equal(g["value"], values), (n, na, nb, name)
        p.close()


def test_helper_write_options_select_the_reference_files():
    """v2RDMHelper.written_files follows hilbert's write options: TPDM_WRITE is
    WriteActiveTPDM (the leading active records, "length" only)."""
    from oracle.maps import RefProblem
    n = 3
    rng = np.random.default_rng(6)
    h, g = rng.standard_normal((n, n)), rng.standard_normal((n,) * 4)
    helper = hb.v2RDMHelper(2, 1, n, h.ravel(), g.ravel(),
                            {"TPDM_WRITE": True, "OPDM_WRITE_FULL": True, "TPDM_WRITE_SPIN_FREE": True})
    helper.x = rng.standard_normal(helper.problem.n_primal)   # stands in for a solved x
    files = helper.written_files()
    assert set(files) == {"D2aa", "D2bb", "D2ab", "D2", "D1a", "D1b"}
    r = RefProblem(n, 2, 1, "DQG", True, True, h=h, g=g)
    _, full = r.write_rdms(helper.x, 0)
    for name in ("D2aa", "D2bb", "D2ab"):
        assert set(files[name]) <= {name, "length"}
        assert files[name].get(name, b"") == full[name].get(name, b"")   # no core: active = full
    assert files["D2"] == full["D2"] and files["D1a"] == full["D1a"]


@pytest.mark.parametrize("ncore", [0, 2])
def test_d3_entries_match_the_reference_3pdm_writer(ncore):
    """WriteActive3PDM's D3aaa, D3aab, D3bba and D3bbb files, byte for byte."""
    from oracle.maps import RefProblem
    rng = np.random.default_rng(41 + ncore)
    for n, na, nb in [(3, 2, 1), (4, 2, 2), (4, 3, 1), (2, 1, 1), (5, 2, 2)]:
        r = RefProblem(n, na, nb, "DQG+D3", True, True, h=rng.standard_normal((n, n)),
                       g=rng.standard_normal((n,) * 4))
        x = rng.standard_normal(r.n_primal)
        _, ref_entries = r.write_rdms(x, ncore)
        p = hb.V2RDMProblem(n, na, nb, "DQG+D3")
        mine = p.d3_entries(x, ncore)
        for name, entries in mine.items():
            assert entries == ref_entries[name], (n, na, nb, ncore, name)
        p.close()
    with pytest.raises(hb.V2BError):
        hb.V2RDMProblem(3, 1, 1, "DQG").d3_entries(np.zeros(hb.V2RDMProblem(3, 1, 1, "DQG").n_primal))
