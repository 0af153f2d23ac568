"""The GPU GW path against the reference's own GW golden fixtures, through the C ABI.

The fixture's G_tau at the irreducible k-points is expanded to the full zone by the library's host
side (gb200.inputs.KSymmetry, as context_from_files does for green-mbpt input files), the
irreducible k-pair integrals likewise, and gb200_gw_sigma runs on the transforms of the fixture's
110 IR tau points.  Sigma at the irreducible points is compared with the reference's stored
``result/Sigma_tau`` at the reference test's absolute 1e-6 (test/solvers_test.cpp:80-135) and with
the oracle's replay at 1e-10 relative; the split-precision path (5 slices) meets the reference's
1e-6 too.
"""
import functools

import numpy as np
import pytest

import _gw_golden as GG
from gb200 import lib, solvers

pytestmark = pytest.mark.gpu


@functools.lru_cache(maxsize=None)
def _inputs(name):
    d = GG.case(name)
    inp = GG.product_inputs(d)
    q0 = (d["AqQ"], d["q_abs"], d["q_ibz2bz"]) if "AqQ" in d else None
    return d, inp, q0


def _sigma(name, precision=lib.PREC_FP64, slices=4):
    d, inp, q0 = _inputs(name)
    ctx, inp = solvers.context_from_arrays(dict(inp), gw_store=d["V_chunk"], grid=GG.grid(), beta=d["beta"], q0=q0)
    try:
        ctx.set_precision(precision, slices)
        G = inp["symmetry"].full_from_ibz(d["G_tau"])
        return d, ctx.gw_sigma(G)[:, :, d["ibz2bz"]]
    finally:
        ctx.close()


@pytest.mark.parametrize("name", GG.CASES)
def test_gpu_fp64_reproduces_reference_sigma(name, gpu):
    d, sig = _sigma(name)
    assert np.isfinite(sig).all()
    err = float(np.abs(sig - d["Sigma_tau"]).max())
    assert err < GG.REF_TOL, err
    ref = GG.oracle_sigma(name)
    rel = float(np.abs(sig - ref).max() / np.abs(ref).max())
    assert rel < 1e-10, rel


@pytest.mark.parametrize("name", GG.CASES)
def test_gpu_split_reproduces_reference_sigma(name, gpu):
    d, sig = _sigma(name, lib.PREC_SPLIT, 5)
    err = float(np.abs(sig - d["Sigma_tau"]).max())
    assert err < GG.REF_TOL, err


def test_gpu_gw_orth_invariance_golden(gpu):
    """GW part of the reference's orth-invariance test (test/solvers_test.cpp:432-445) with the
    self-energy from gb200_gw_sigma: e_1b, e_HF and e_corr agree across the four bases to 1e-10."""
    from test_gw_golden import ORTH_BASES, orth_energies
    g = GG.grid()

    def gpu_sigma(G, V, ns, NQ):
        nao = G.shape[-1]
        with lib.Context(1, nao, ns, NQ, g.nts, g.nw, g.nw_b, g.beta) as c:
            c.set_kq_maps(np.zeros((1, 1), np.int32), np.zeros((1, 1), np.int32))
            c.set_grid(g.Tnt_f, g.Ttn_f, g.Tnt_b, g.Ttn_b, g.wsample_f)
            c.set_integrals(np.ascontiguousarray(V[:1]), lib.INTEGRALS_GW)
            return c.gw_sigma(G)

    E = orth_energies(gpu_sigma)
    assert abs(E["none"][2]) > 1e-3
    for b in ORTH_BASES[1:]:
        for i in range(3):
            assert abs(E[b][i] - E["none"][i]) < 1e-10, (b, i, E[b][i], E["none"][i])
