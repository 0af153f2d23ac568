"""Extract the reference's HF golden fixtures into small numpy files.

Run once in a checkout that has the green-mbpt sources (read-only) next to
this repository:

    python tests/golden/make_golden.py /path/to/green-mbpt

It reads test/data/{HF,HF_X2C}/{input.h5,data.h5,df_hf_int/*} of the
reference with the minimal HDF5 reader gb200.h5lite and writes
tests/golden/{hf,hf_x2c}.npz holding exactly what one call of the reference's
``solve_hf`` test (test/solvers_test.cpp:27-78) consumes and produces:
G(tau = beta) (the last tau slice of ``G_tau``), the irreducible k-pair chunk of
V, the overlap S_k at the irreducible points, the Madelung constant, the
k-point / k-pair symmetry tables and the expected ``result/Sigma1``.

It also writes tests/golden/hf_orth.npz from test/data/HF_orth_invariance/<basis>/
(basis = none, lowdin, mo, natural: one H2 molecule written in four orbital bases), the
inputs of the HF part of the reference's orth-invariance test (test/solvers_test.cpp:296-430):
G(beta) of ``iter1/G_tau/data``, S_k and H_k, the integral chunk, the Madelung constant and
the nuclear repulsion, with what the reference's own run wrote next to them:
``iter1/Sigma1`` (the Fock matrix of that G), ``iter1/Energy_1b`` and ``iter1/Energy_HF``
(E_HF + E_nuc, dyson.cpp:325-326).  The whole ``iter1/G_tau/data`` (on the IR grid described below) is
kept as well, for the GW part of the same test: one GW self-energy per basis and the energies of
mbpt::compute_energy, which must agree across the four bases (solvers_test.cpp:432-445).

It writes tests/golden/gw.npz from test/data/{GW,GW_X2C}: the inputs and the expected output of
the reference's three GW self-energy tests (test/solvers_test.cpp:80-135,389-391), under the
prefixes ``gw/`` (input.h5 + df_int, q0 "IGNORE_G0"), ``gw_c/`` (input_tr_symm.h5 + df_hf_int with
the "EXTRAPOLATE" q -> 0 correction of df_hf_int/AqQ.h5) and ``gw_x2c/`` (a two-component
molecule): G_tau and ``result/Sigma_tau`` at the irreducible k-points, the irreducible k-pair chunk
of V, the k-point / k-pair symmetry tables and fractional k coordinates, S_k and H_k at the
irreducible points, the Madelung constant and, for ``gw_c/``, AqQ, |q| and the irreducible q-points.
Those tests run on the IR grid file ``ir/1e4.h5`` of the external green-grids package
(Lambda = 1e4, 110 tau points at beta = 100), which the reference does not ship; its tau points are
the ``iter1/G_tau/mesh`` that the orth-invariance run (same grid file, same beta,
solvers_test.cpp:317-320) wrote into test/data/HF_orth_invariance/none/data.h5, stored here as
``tau`` with ``beta`` and ``wmax = Lambda / beta``.  The replay builds its transforms for those
points (gb200.grids.SampledGrid).
"""
from __future__ import annotations

import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..", "green-mbpt_b200"))
from gb200.h5lite import H5File  # noqa: E402


def _cplx(a):
    if a.dtype.names:
        return a["r"] + 1j * a["i"]
    v = np.ascontiguousarray(a, dtype=np.float64).view(np.complex128)
    return v[..., 0] if v.shape[-1] == 1 else v


def extract(ref_root: str, case: str, intdir: str = "df_hf_int") -> dict:
    base = os.path.join(ref_root, "test", "data", case)
    inp = H5File(os.path.join(base, "input.h5"))
    dat = H5File(os.path.join(base, "data.h5"))
    meta = H5File(os.path.join(base, intdir, "meta.h5"))
    nk = int(inp.read("params/nk"))
    ns = int(inp.read("params/ns"))
    nao = int(inp.read("params/nao"))
    nso = int(inp.read("params/nso"))
    NQ = int(inp.read("params/NQ"))
    chunk = int(meta.read("chunk_size"))
    idx = meta.read("chunk_indices")
    if len(idx) != 1 or int(idx[0]) != 0:
        raise RuntimeError("fixture is expected to hold a single integral chunk")
    sym = lambda p: inp.read("symmetry/" + p)
    ibz2bz = sym("k/ibz2bz")
    S = _cplx(inp.read("HF/S-k")).reshape(ns, nk, nso, nso)[:, ibz2bz]
    G = _cplx(dat.read("G_tau"))
    out = dict(
        nk=nk, ns=ns, nao=nao, nso=nso, NQ=NQ,
        madelung=float(inp.read("HF/madelung")),
        version=np.bytes_(meta.attr("/", "__green_version__")),
        chunk_size=chunk,
        G_beta=G[-1],
        S_ibz=S,
        V_chunk=_cplx(H5File(os.path.join(base, intdir, "VQ_0.h5")).read("/0")),
        bz2ibz=sym("k/bz2ibz"), ibz2bz=ibz2bz, tr_conj=sym("k/tr_conj"),
        k_sym_transform_ao=_cplx(sym("k/k_sym_transform_ao")),
        weight_ibz=sym("k/weight_ibz"),
        conj_pairs_list=sym("pairs/conj_pairs_list"),
        trans_pairs_list=sym("pairs/trans_pairs_list"),
        kpair_irre_list=sym("pairs/kpair_irre_list"),
        Sigma1=_cplx(dat.read("result/Sigma1")),
        k_frac=np.asarray(sym("k/mesh_scaled"), dtype=np.float64).reshape(nk, 3),
    )
    return out


ORTH_BASES = ("none", "lowdin", "mo", "natural")


def extract_orth(ref_root: str) -> dict:
    out = {}
    for basis in ORTH_BASES:
        base = os.path.join(ref_root, "test", "data", "HF_orth_invariance", basis)
        inp = H5File(os.path.join(base, "input.h5"))
        dat = H5File(os.path.join(base, "data.h5"))
        ns, nk = int(inp.read("params/ns")), int(inp.read("params/nk"))
        nso, nao, NQ = int(inp.read("params/nso")), int(inp.read("params/nao")), int(inp.read("params/NQ"))
        if nk != 1:
            raise RuntimeError("the orth-invariance fixture is expected to be a molecule (nk = 1)")
        meta = H5File(os.path.join(base, "df_hf_int", "meta.h5"))
        idx = meta.read("chunk_indices")
        if len(idx) != 1 or int(idx[0]) != 0:
            raise RuntimeError("fixture is expected to hold a single integral chunk")
        shape = (ns, nk, nso, nso)
        out.update({
            f"{basis}/G_beta": _cplx(dat.read("iter1/G_tau/data"))[-1],
            f"{basis}/G_tau": _cplx(dat.read("iter1/G_tau/data")),
            f"{basis}/S": _cplx(inp.read("HF/S-k")).reshape(shape),
            f"{basis}/H": _cplx(inp.read("HF/H-k")).reshape(shape),
            f"{basis}/V_chunk": _cplx(H5File(os.path.join(base, "df_hf_int", "VQ_0.h5")).read("/0")),
            f"{basis}/madelung": float(inp.read("HF/madelung")),
            f"{basis}/E_nuc": float(inp.read("HF/Energy_nuc")),
            f"{basis}/Sigma1": _cplx(dat.read("iter1/Sigma1")),
            f"{basis}/Energy_1b": float(dat.read("iter1/Energy_1b")),
            f"{basis}/Energy_HF": float(dat.read("iter1/Energy_HF")),
            f"{basis}/dims": np.array([ns, nk, nao, nso, NQ]),
        })
    return out


GW_CASES = (("gw", "GW/input.h5", "GW/df_int", "GW/data.h5", None),
            ("gw_c", "GW/input_tr_symm.h5", "GW/df_hf_int", "GW/data_c.h5", "GW/df_hf_int/AqQ.h5"),
            ("gw_x2c", "GW_X2C/input.h5", "GW_X2C/df_hf_int", "GW_X2C/data.h5", None))
IR_LAMBDA, IR_BETA = 1e4, 100.0


def extract_gw(ref_root: str) -> dict:
    data = os.path.join(ref_root, "test", "data")
    tau = np.asarray(H5File(os.path.join(data, "HF_orth_invariance", "none", "data.h5")).read("iter1/G_tau/mesh"))
    out = dict(tau=tau, beta=IR_BETA, wmax=IR_LAMBDA / IR_BETA)
    for name, inp_f, int_d, dat_f, q0_f in GW_CASES:
        inp = H5File(os.path.join(data, inp_f))
        dat = H5File(os.path.join(data, dat_f))
        meta = H5File(os.path.join(data, int_d, "meta.h5"))
        idx = meta.read("chunk_indices")
        if len(idx) != 1 or int(idx[0]) != 0:
            raise RuntimeError("fixture is expected to hold a single integral chunk")
        ns, nk = int(inp.read("params/ns")), int(inp.read("params/nk"))
        nso, nao, NQ = int(inp.read("params/nso")), int(inp.read("params/nao")), int(inp.read("params/NQ"))
        sym = lambda p: inp.read("symmetry/" + p)
        ibz2bz = sym("k/ibz2bz")
        full = lambda key: _cplx(inp.read(key)).reshape(ns, nk, nso, nso)[:, ibz2bz]
        G = _cplx(dat.read("G_tau"))
        if G.shape[0] != len(tau):
            raise RuntimeError(f"{dat_f}: {G.shape[0]} tau points, the grid has {len(tau)}")
        d = {
            "dims": np.array([ns, nk, nao, nso, NQ]),
            "madelung": float(inp.read("HF/madelung")),
            "G_tau": G,
            "Sigma_tau": _cplx(dat.read("result/Sigma_tau")),
            "V_chunk": _cplx(H5File(os.path.join(data, int_d, "VQ_0.h5")).read("/0")),
            "S_ibz": full("HF/S-k"), "H_ibz": full("HF/H-k"),
            "bz2ibz": sym("k/bz2ibz"), "ibz2bz": ibz2bz, "tr_conj": sym("k/tr_conj"),
            "k_sym_transform_ao": _cplx(sym("k/k_sym_transform_ao")), "weight_ibz": sym("k/weight_ibz"),
            "conj_pairs_list": sym("pairs/conj_pairs_list"), "trans_pairs_list": sym("pairs/trans_pairs_list"),
            "kpair_irre_list": sym("pairs/kpair_irre_list"),
            "k_frac": np.asarray(sym("k/mesh_scaled"), dtype=np.float64).reshape(nk, 3),
        }
        if q0_f is not None:
            q0 = H5File(os.path.join(data, q0_f))
            d["AqQ"] = _cplx(q0.read("AqQ"))
            d["q_abs"] = np.asarray(q0.read("q_abs"), dtype=np.float64).reshape(-1)
            d["q_ibz2bz"] = sym("q/ibz2bz")
        out.update({f"{name}/{k}": v for k, v in d.items()})
    return out


def main(argv):
    if len(argv) != 2:
        print(__doc__)
        return 2
    ref = argv[1]
    here = os.path.dirname(os.path.abspath(__file__))
    for case, name in (("HF", "hf"), ("HF_X2C", "hf_x2c")):
        d = extract(ref, case)
        np.savez_compressed(os.path.join(here, name + ".npz"), **d)
        print(f"wrote {name}.npz: nk={d['nk']} ns={d['ns']} nao={d['nao']} nso={d['nso']} NQ={d['NQ']}")
    np.savez_compressed(os.path.join(here, "hf_orth.npz"), **extract_orth(ref))
    print("wrote hf_orth.npz: " + ", ".join(ORTH_BASES))
    np.savez_compressed(os.path.join(here, "gw.npz"), **extract_gw(ref))
    print("wrote gw.npz: " + ", ".join(c[0] for c in GW_CASES))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
