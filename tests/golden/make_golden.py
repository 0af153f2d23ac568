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
(E_HF + E_nuc, dyson.cpp:325-326).

The GW fixtures (test/data/GW) are not extracted: replaying them needs the IR
grid file ``ir/1e4.h5`` of the external green-grids package, which the
reference does not ship.
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
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
