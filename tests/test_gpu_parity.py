"""GPU FP64 path against the CPU oracle, through the C ABI.

Tolerance: 1e-10 relative to the largest element (the FP64 parity bar of the
plain GPU path); the HF golden fixture is compared at the reference's own
1e-10 absolute tolerance (test/tensor_test.h:41).
"""
import os

import numpy as np
import pytest

import gw_oracle as O
from gb200 import lib, solvers
from _systems import oracle_fock, oracle_sigma, rel, system

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.fixture(scope="module")
def ctx_small(gpu):
    s = system("small")
    c = solvers.make_context(s)
    yield s, c
    c.close()


@pytest.mark.parametrize("name", ["small", "small_ns2", "odd_mesh", "c0"])
def test_gw_sigma_parity(gpu, name):
    s = system(name)
    with solvers.make_context(s) as c:
        sig = c.gw_sigma(s.G)
    ref = oracle_sigma(name)
    assert rel(sig, ref) < TOL


@pytest.mark.parametrize("name", ["small", "small_ns2", "c0"])
def test_hf_parity(gpu, name):
    s = system(name)
    with solvers.make_context(s) as c:
        for mad in (0.0, 0.37):
            dm = O.hf_density(s.G, s.ns)
            F = c.hf_fock(dm, s.S, mad)
            assert rel(F, oracle_fock(s, mad)) < TOL


def test_hf_golden_through_gpu(gpu):
    """The reference's HF fixture through the GPU kernel, the k-point symmetry expanded by the
    library's own host code (gb200.inputs.KSymmetry), compared with the reference's Sigma1."""
    from gb200 import inputs
    d = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "hf.npz")))
    sym = inputs.KSymmetry(d["bz2ibz"], d["ibz2bz"], d["tr_conj"], d["k_sym_transform_ao"], d["conj_pairs_list"],
                           d["trans_pairs_list"], d["kpair_irre_list"], d["weight_ibz"])
    ns, nk, nao, NQ = int(d["ns"]), int(d["nk"]), int(d["nao"]), int(d["NQ"])
    pref = -1.0 if ns == 2 else -2.0                   # hf_solver.h:38
    dm = sym.full_from_ibz(pref * d["G_beta"])
    S = sym.full_from_ibz(d["S_ibz"])
    Vh = sym.half_storage(d["V_chunk"])
    with lib.Context(nk, nao, ns, NQ, 2, 2, 2, 100.0) as c:
        c.set_integrals(Vh, lib.INTEGRALS_HF)
        F = c.hf_fock(dm, S, float(d["madelung"]))
    np.testing.assert_allclose(sym.ibz_from_full(F), d["Sigma1"], rtol=0, atol=1e-10)


def test_dyson_parity(gpu, ctx_small):
    s, c = ctx_small
    g = s.grid
    sig = oracle_sigma("small")
    F = oracle_fock(s)
    mu = -0.3
    G, S1h, Sth = c.compute_G(F, sig, mu)
    Gref = O.compute_G(F, sig, s.F, s.S, mu, g.Tnt_f, g.Ttn_f, g.wsample_f)
    assert rel(G, Gref) < TOL
    assert rel(S1h, O.make_hermitian(F)) < 1e-14
    ev = O.selfenergy_eigenspectra(F, sig, s.F, s.S, g.Tnt_f)
    n_ref = O.number_of_electrons(mu, ev, g.Ttn_beta, g.wsample_f, s.ns, 1.0 / s.nk)
    n_gpu = c.electrons(F, sig, mu)
    assert abs(n_gpu - n_ref) < 1e-10 * abs(n_ref)
    target = s.nel_from_G0()
    nel_g, mu_g = c.find_mu(F, sig, 0.0, target, 1e-9)
    nel_o, mu_o = O.find_mu(0.0, target, ev, g.Ttn_beta, g.wsample_f, s.ns, 1.0 / s.nk, 1e-9)
    assert abs(mu_g - mu_o) < 1e-8
    assert abs(nel_g - target) <= 1e-9 * target
    e_gpu = c.energy(Gref, F, sig)
    e_ref = O.compute_energy(Gref, F, sig, s.F, g.Tnt_f, g.Ttn_beta, 1.0 / s.nk)
    np.testing.assert_allclose(e_gpu, e_ref, rtol=1e-10, atol=1e-12)


def test_solver_mirror_iteration(gpu, ctx_small):
    """gw_solver / hf_solver / dyson in the order of one reference SC iteration."""
    s, c = ctx_small
    G = s.G.copy()
    S1 = np.zeros(c.shape_F, dtype=np.complex128)
    St = np.zeros(c.shape_G, dtype=np.complex128)
    solvers.hf_solver(c, s.S, 0.0, s.ns).solve(G, S1, St)
    solvers.gw_solver(c).solve(G, S1, St)
    dy = solvers.dyson(c, nel=s.nel_from_G0())
    dy.solve(G, S1, St)
    assert np.isfinite(G).all()
    assert dy.diff(G, S1, St) > 0


def test_determinism(gpu, ctx_small):
    s, c = ctx_small
    a = c.gw_sigma(s.G)
    b = c.gw_sigma(s.G)
    assert np.array_equal(a, b)


def test_sigma_hermitian_and_finite(gpu, ctx_small):
    s, c = ctx_small
    sig = c.gw_sigma(s.G)
    assert np.isfinite(sig).all()
    assert np.abs(sig - np.conj(np.swapaxes(sig, -1, -2))).max() < 1e-9 * np.abs(sig).max()


def test_wrong_grid_rejected(gpu):
    with pytest.raises(lib.mbpt_wrong_grid):
        lib.Context(4, 6, 1, 20, 21, 20, 21, 20.0)


def test_missing_setup_is_an_error(gpu):
    s = system("small")
    g = s.grid
    with lib.Context(s.nk, s.nao, s.ns, s.NQ, g.nts, g.nw, g.nw_b, s.beta) as c:
        with pytest.raises(lib.mbpt_kernel_error):
            c.gw_sigma(s.G)


@pytest.mark.parametrize("prec", [lib.PREC_FP64, lib.PREC_SPLIT])
def test_q_shards_sum_to_full_sigma(gpu, prec):
    """Partial Sigma over the q ranges of 3 ranks add up to the full Sigma (gw_cpu_kernel.cpp:45-54)."""
    from gb200 import shard
    s = system("odd_mesh")
    with solvers.make_context(s, precision=prec, slices=5) as c:
        full = c.gw_sigma(s.G)
        parts = []
        for r in range(3):
            c.set_q_range(*shard.q_shard(s.nk, 3, r))
            parts.append(c.gw_sigma(s.G))
    assert rel(sum(parts), full) < 1e-13


def test_device_integrals_in_chunks_match_host_upload(gpu):
    """gb200_set_integrals_device with uneven chunks gives the same Sigma as gb200_set_integrals."""
    import torch
    s = system("small_ns2")
    with solvers.make_context(s) as c:
        want = c.gw_sigma(s.G)
        V = torch.from_numpy(np.ascontiguousarray(s.V_half)).cuda()
        npair = V.shape[0]
        cuts = [0, 1, 4, npair]
        for a, b in zip(cuts, cuts[1:]):
            c.set_integrals_device(V[a].data_ptr(), a, b - a)
        torch.cuda.synchronize()
        got = c.gw_sigma(s.G)
    assert rel(got, want) < 1e-14


def test_hf_x2c_golden_through_gpu(gpu):
    """Two-component (X2C) Fock build on the GPU against the reference's HF_X2C fixture
    (hf_x2c_cpu_kernel::solve, hf_cpu_kernels.cpp:148-279), at the reference's 1e-10."""
    from gb200 import inputs
    d = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "hf_x2c.npz")))
    sym = inputs.KSymmetry(d["bz2ibz"], d["ibz2bz"], d["tr_conj"], d["k_sym_transform_ao"], d["conj_pairs_list"],
                           d["trans_pairs_list"], d["kpair_irre_list"], d["weight_ibz"])
    ns, nk, nao, nso, NQ = int(d["ns"]), int(d["nk"]), int(d["nao"]), int(d["nso"]), int(d["NQ"])
    assert nso == 2 * nao and ns == 1
    dm = sym.full_from_ibz(-1.0 * d["G_beta"])         # spin_prefactor -1 for X2C (hf_solver.h:38)
    S = sym.full_from_ibz(d["S_ibz"])
    with lib.Context(nk, nao, ns, NQ, 2, 2, 2, 100.0, nso=nso) as c:
        c.set_integrals(sym.half_storage(d["V_chunk"]), lib.INTEGRALS_HF)
        F = c.hf_fock(dm, S, float(d["madelung"]))
        with pytest.raises(lib.mbpt_kernel_error):
            c.gw_sigma(np.zeros((2, ns, nk, nso, nso), dtype=np.complex128))
    np.testing.assert_allclose(sym.ibz_from_full(F), d["Sigma1"], rtol=0, atol=1e-10)
    # Hermitian to round-off (the reference does not hermitize the diagonal blocks either)
    assert np.abs(F - np.conj(np.swapaxes(F, -1, -2))).max() < 1e-11 * np.abs(F).max()


def test_hf_orth_invariance_golden_through_gpu(gpu):
    """HF part of the reference's orth-invariance test (test/solvers_test.cpp:296-430) through the
    GPU Fock build: one H2 molecule in four orbital bases; F equals the reference run's Sigma1,
    E_1b and E_HF + E_nuc the energies it wrote (dyson.cpp:325-326), and the energies agree across
    the bases, all to 1e-10."""
    d = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "hf_orth.npz")))
    E = {}
    for basis in ("none", "lowdin", "mo", "natural"):
        ns, nk, nao, nso, NQ = (int(x) for x in d[f"{basis}/dims"])
        dm = -1.0 * d[f"{basis}/G_beta"]  # ns = 2: spin prefactor -1 (hf_solver.h:38)
        H = d[f"{basis}/H"]
        with lib.Context(nk, nao, ns, NQ, 2, 2, 2, 100.0) as c:
            c.set_integrals(np.ascontiguousarray(d[f"{basis}/V_chunk"].reshape(1, NQ, nao, nao)), lib.INTEGRALS_HF)
            F = c.hf_fock(dm, d[f"{basis}/S"], float(d[f"{basis}/madelung"]))
        np.testing.assert_allclose(F, d[f"{basis}/Sigma1"], rtol=0, atol=1e-10)
        e1 = sum(np.trace(dm[s, 0] @ H[s, 0]).real for s in range(ns))
        ehf = sum(0.5 * np.trace(dm[s, 0] @ (F[s, 0] + 2.0 * H[s, 0])).real for s in range(ns))
        assert abs(e1 - float(d[f"{basis}/Energy_1b"])) < 1e-10
        assert abs(ehf + float(d[f"{basis}/E_nuc"]) - float(d[f"{basis}/Energy_HF"])) < 1e-10
        E[basis] = (e1, ehf)
    for basis in ("lowdin", "mo", "natural"):
        assert abs(E[basis][0] - E["none"][0]) < 1e-10
        assert abs(E[basis][1] - E["none"][1]) < 1e-10


def test_hf_x2c_matches_oracle_with_madelung(gpu):
    """X2C Fock build with a non-zero Madelung constant and several k-points against the oracle."""
    s = system("small")
    nk, nao, NQ = s.nk, s.nao, s.NQ
    rng = np.random.default_rng(3)
    nso = 2 * nao
    a = rng.standard_normal((1, nk, nso, nso)) + 1j * rng.standard_normal((1, nk, nso, nso))
    dm = 0.05 * (a + np.conj(np.swapaxes(a, -1, -2)))
    b = rng.standard_normal((nk, nao, nao)) + 1j * rng.standard_normal((nk, nao, nao))
    Saa = np.eye(nao) + 0.02 * (b + np.conj(np.swapaxes(b, -1, -2)))
    S = np.zeros((1, nk, nso, nso), dtype=np.complex128)
    S[0, :, :nao, :nao] = Saa
    S[0, :, nao:, nao:] = Saa
    mad = 0.21
    integ = O.HalfStoredIntegrals(s.V_half)
    want = O.hf_x2c(dm, S, mad, integ.pair, lambda X, k: X[k], nk, lambda ik: ik, NQ, nao)
    with lib.Context(nk, nao, 1, NQ, 2, 2, 2, 20.0, nso=nso) as c:
        c.set_integrals(s.V_half, lib.INTEGRALS_HF)
        F = c.hf_fock(dm, S, mad)
    assert rel(F, want) < TOL


@pytest.mark.parametrize("prec", [lib.PREC_FP64, lib.PREC_SPLIT])
def test_gw_x2c_matches_oracle(gpu, prec):
    """Two-component (X2C) GW self-energy: the 4 spin blocks of G (gw_cpu_kernel.cpp:166-187,
    326-351) against the oracle; FP64 at 1e-10, split precision (S = 5) at 1e-8."""
    s = system("small")
    nk, nao, NQ, g = s.nk, s.nao, s.NQ, s.grid
    rng = np.random.default_rng(7)
    nso = 2 * nao
    G2 = np.zeros((g.nts, 1, nk, nso, nso), dtype=np.complex128)
    X = rng.standard_normal((nk, nao, nao)) + 1j * rng.standard_normal((nk, nao, nao))
    for t in range(g.nts):
        G2[t, 0, :, :nao, :nao] = s.G[t, 0]
        G2[t, 0, :, nao:, nao:] = 0.7 * s.G[t, 0]
        G2[t, 0, :, :nao, nao:] = 0.05 * X
        G2[t, 0, :, nao:, :nao] = 0.05 * np.conj(np.swapaxes(X, -1, -2))
    want = O.gw_solve(G2, O.HalfStoredIntegrals(s.V_half), O.NoSymBZ(s.mesh), g.Tnt_b, g.Ttn_b, 1, NQ, X2C=True)
    with lib.Context(nk, nao, 1, NQ, g.nts, g.nw, g.nw_b, s.beta, nso=nso) as c:
        kp, km = solvers.kq_maps(s.mesh)
        c.set_kq_maps(kp, km)
        c.set_grid(g.Tnt_f, g.Ttn_f, g.Tnt_b, g.Ttn_b, g.wsample_f)
        c.set_integrals(s.V_half, lib.INTEGRALS_GW)
        c.set_precision(prec, 5)
        got = c.gw_sigma(G2)
    assert rel(got, want) < (TOL if prec == lib.PREC_FP64 else 1e-8)


def test_dyson_x2c_matches_oracle(gpu):
    """Dyson step, electron count, chemical potential and energies for two-component input
    (prefactors of dyson.cpp:95 and common_utils.cpp:18,37 with X2C) against the oracle."""
    s = system("small")
    nk, nao, g = s.nk, s.nao, s.grid
    nso = 2 * nao
    rng = np.random.default_rng(11)

    def herm(shape, scale):
        a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        return scale * (a + np.conj(np.swapaxes(a, -1, -2)))

    H = np.zeros((1, nk, nso, nso), dtype=np.complex128)
    S = np.zeros_like(H)
    H[0, :, :nao, :nao] = s.F[0]
    H[0, :, nao:, nao:] = s.F[0]
    H[0] += herm((nk, nso, nso), 0.02)
    S[0, :, :nao, :nao] = s.S[0]
    S[0, :, nao:, nao:] = s.S[0]
    F1 = herm((1, nk, nso, nso), 0.05)
    sig = herm((g.nts, 1, nk, nso, nso), 0.01)
    with lib.Context(nk, nao, 1, s.NQ, g.nts, g.nw, g.nw_b, s.beta, nso=nso) as c:
        c.set_grid(g.Tnt_f, g.Ttn_f, g.Tnt_b, g.Ttn_b, g.wsample_f)
        c.set_hamiltonian(H, S)
        mu = -0.2
        G, _, _ = c.compute_G(F1, sig, mu)
        Gref = O.compute_G(F1, sig, H, S, mu, g.Tnt_f, g.Ttn_f, g.wsample_f)
        assert rel(G, Gref) < TOL
        ev = O.selfenergy_eigenspectra(F1, sig, H, S, g.Tnt_f)
        n_ref = O.number_of_electrons(mu, ev, g.Ttn_beta, g.wsample_f, 1, 1.0 / nk, X2C=True)
        assert abs(c.electrons(F1, sig, mu) - n_ref) < 1e-10 * abs(n_ref)
        target = n_ref + 0.5
        nel_g, mu_g = c.find_mu(F1, sig, 0.0, target, 1e-9)
        nel_o, mu_o = O.find_mu(0.0, target, ev, g.Ttn_beta, g.wsample_f, 1, 1.0 / nk, 1e-9, X2C=True)
        assert abs(mu_g - mu_o) < 1e-8
        e_gpu = c.energy(Gref, F1, sig)
    e_ref = O.compute_energy(Gref, F1, sig, H, g.Tnt_f, g.Ttn_beta, 1.0 / nk, X2C=True)
    np.testing.assert_allclose(e_gpu, e_ref, rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("x2c", [False, True])
def test_gw_q0_correction_matches_oracle(gpu, x2c):
    """The "extrapolate" q -> 0 correction (mbpt_q0_utils_t.cpp:11-178) on top of Sigma: scalar
    and two-component input against the oracle at 1e-10."""
    s = system("small")
    nk, nao, NQ, g = s.nk, s.nao, s.NQ, s.grid
    rng = np.random.default_rng(5)
    A = rng.standard_normal((nk, NQ)) + 1j * rng.standard_normal((nk, NQ))
    A /= np.linalg.norm(A, axis=1, keepdims=True)
    q_abs = np.array([0.0, 0.21, 0.34, 0.52])
    mad = 0.37
    nso = 2 * nao if x2c else nao
    ns = 1 if x2c else s.ns
    if x2c:
        G = np.zeros((g.nts, 1, nk, nso, nso), dtype=np.complex128)
        G[:, 0, :, :nao, :nao] = s.G[:, 0]
        G[:, 0, :, nao:, nao:] = 0.6 * s.G[:, 0]
        X = rng.standard_normal((nk, nao, nao)) + 1j * rng.standard_normal((nk, nao, nao))
        G[:, 0, :, :nao, nao:] = 0.05 * X
        G[:, 0, :, nao:, :nao] = 0.03 * np.conj(np.swapaxes(X, -1, -2))
    else:
        G = s.G.copy()
    b = rng.standard_normal((nk, nao, nao)) + 1j * rng.standard_normal((nk, nao, nao))
    Saa = np.eye(nao) + 0.02 * (b + np.conj(np.swapaxes(b, -1, -2)))
    S = np.zeros((ns, nk, nso, nso), dtype=np.complex128)
    H = np.zeros_like(S)
    for sp in range(ns):
        S[sp, :, :nao, :nao] = Saa
        H[sp, :, :nao, :nao] = s.F[0]
        if x2c:
            S[sp, :, nao:, nao:] = Saa
            H[sp, :, nao:, nao:] = s.F[0]
    want = O.gw_solve(G, O.HalfStoredIntegrals(s.V_half), O.NoSymBZ(s.mesh), g.Tnt_b, g.Ttn_b, ns, NQ, X2C=x2c,
                      q0=(A, q_abs, mad, S))
    with lib.Context(nk, nao, ns, NQ, g.nts, g.nw, g.nw_b, s.beta, nso=nso) as c:
        kp, km = solvers.kq_maps(s.mesh)
        c.set_kq_maps(kp, km)
        c.set_grid(g.Tnt_f, g.Ttn_f, g.Tnt_b, g.Ttn_b, g.wsample_f)
        c.set_integrals(s.V_half, lib.INTEGRALS_GW)
        c.set_hamiltonian(H, S)
        c.set_q0_correction(A, q_abs, mad)
        got = c.gw_sigma(G)
        c.set_q_range(0, 2)
        with pytest.raises(lib.mbpt_kernel_error):
            c.gw_sigma(G)
    assert rel(got, want) < TOL
