"""Host-side input handling: green-mbpt's file format and the k-point symmetry expansion.

The expansion is checked against the oracle's restatement of the reference's value_AO and
df_integral_t::symmetrize on the committed HF fixtures (hf.npz: 27 k-points, 4 irreducible,
196 irreducible k-pairs; hf_x2c.npz).  When GREEN_MBPT_TEST_DATA points at green-mbpt's
test/data directory, the readers are also run on the original HDF5 files.
"""
import os

import numpy as np
import pytest

import gw_oracle as O
from gb200 import inputs, lib

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden(name):
    return dict(np.load(os.path.join(HERE, "golden", name + ".npz")))


def _both(d):
    args = (d["bz2ibz"], d["ibz2bz"], d["tr_conj"], d["k_sym_transform_ao"], d["conj_pairs_list"],
            d["trans_pairs_list"], d["kpair_irre_list"], d["weight_ibz"])
    return inputs.KSymmetry(*args), O.RefSymmetry(*args)


@pytest.mark.parametrize("name", ["hf", "hf_x2c"])
def test_symmetry_expansion_matches_oracle(name):
    d = _golden(name)
    ks, ref = _both(d)
    nk = int(d["nk"])
    full = ks.full_from_ibz(d["S_ibz"])
    for s in range(int(d["ns"])):
        for k in range(nk):
            want = d["S_ibz"][s, ref.reduced_point(k)] if k in set(ref.ibz2bz.tolist()) else ref.value_AO(d["S_ibz"][s], k)
            np.testing.assert_array_equal(full[s, k], want)
    for k1 in range(nk):
        for k2 in range(nk):
            np.testing.assert_array_equal(ks.pair(d["V_chunk"], k1, k2), ref.integral(d["V_chunk"], k1, k2))
    half = ks.half_storage(d["V_chunk"])
    assert half.shape == (nk * (nk + 1) // 2,) + d["V_chunk"].shape[1:]
    np.testing.assert_array_equal(ks.ibz_from_full(full), d["S_ibz"])


def test_kq_maps_from_fractional_points():
    from gb200 import solvers
    for mesh in [(2, 3, 1), (3, 3, 3), (4, 1, 2)]:
        n1, n2, n3 = mesh
        idx = np.arange(n1 * n2 * n3)
        frac = np.stack([idx // (n2 * n3) / n1, (idx // n3) % n2 / n2, idx % n3 / n3], axis=1)
        frac = frac - (frac > 0.5)  # points given in (-1/2, 1/2] as the input files store them
        kp, km = inputs.kq_maps_from_points(frac)
        kp2, km2 = solvers.kq_maps(mesh)
        np.testing.assert_array_equal(kp, kp2)
        np.testing.assert_array_equal(km, km2)


def test_pair_index_layout():
    assert [inputs.pair_index(k1, k2) for k1 in range(3) for k2 in range(k1 + 1)] == list(range(6))
    assert inputs.pair_index(1, 2) == inputs.pair_index(2, 1) == 4


DATA = os.environ.get("GREEN_MBPT_TEST_DATA")


@pytest.mark.skipif(not DATA, reason="GREEN_MBPT_TEST_DATA (green-mbpt's test/data) not given")
@pytest.mark.parametrize("case,name", [("HF", "hf"), ("HF_X2C", "hf_x2c")])
def test_read_green_mbpt_files(case, name):
    d = _golden(name)
    inp = inputs.read_input(os.path.join(DATA, case, "input.h5"))
    sym = inp["symmetry"]
    store, version = inputs.read_integrals(os.path.join(DATA, case, "df_hf_int"), len(sym.kpair_irre))
    assert (inp["nk"], inp["ns"], inp["nao"], inp["nso"], inp["NQ"]) == (int(d["nk"]), int(d["ns"]), int(d["nao"]),
                                                                       int(d["nso"]), int(d["NQ"]))
    np.testing.assert_array_equal(inp["S_ibz"], d["S_ibz"])
    np.testing.assert_array_equal(store, d["V_chunk"][:store.shape[0]])
    assert inp["madelung"] == float(d["madelung"])
    assert version == str(d["version"].astype(str))
    assert lib.check_integral_version(version)


def test_q0_full_zone_layout():
    A = np.arange(6).reshape(3, 2) + 1j
    A2, q2 = inputs.q0_full_zone(A, [0.0, 0.4, 0.7], [0, 2, 5], 6)
    np.testing.assert_array_equal(A2[[0, 2, 5]], A)
    np.testing.assert_array_equal(q2, [0.0, 0.0, 0.4, 0.0, 0.0, 0.7])
    with pytest.raises(ValueError):
        inputs.q0_full_zone(A, [0.0, 0.4, 0.7], [0, 5, 2], 6)


@pytest.mark.skipif(not DATA, reason="GREEN_MBPT_TEST_DATA (green-mbpt's test/data) not given")
def test_read_aqq_file():
    A, q_abs, mad = inputs.read_q0(os.path.join(DATA, "GW", "df_hf_int", "AqQ.h5"))
    assert A.shape == (q_abs.shape[0], 36) and q_abs[0] == 0.0 and (q_abs[1:] > 0).all()
    assert mad is not None and mad > 0


def test_reader_handles_new_format_files():
    """Files written in HDF5's newer format (superblock v2, version-2 object headers, links stored
    in the header) read like the old ones: the orth-invariance result file of green-mbpt's tests,
    when GREEN_MBPT_TEST_DATA names that directory."""
    import os
    root = os.environ.get("GREEN_MBPT_TEST_DATA")
    if not root:
        pytest.skip("GREEN_MBPT_TEST_DATA not set")
    from gb200.h5lite import H5File
    f = H5File(os.path.join(root, "HF_orth_invariance", "none", "data.h5"))
    assert "iter1" in f.keys("/")
    g = f.read("iter1/G_tau/data")
    assert g.shape == (110, 2, 1, 10, 10)
    assert abs(float(f.read("iter1/Energy_1b")) + 2.5027877905876) < 1e-10
