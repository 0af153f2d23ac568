"""gb200_hf_fock_noalloc: the Fock build for callers that cannot allocate device memory.

Some hosts cannot call cudaMalloc once they are running: their memory pool has
already taken the free HBM, or they must not pay the device-wide
synchronisation that cudaMalloc/cudaFree imply.  For them the library offers a
Fock build that works in one fixed device array inside the library.  These
tests call it through the C ABI twice in a row (the second call sees the
workspace the first one left) and compare each result with
gb200_hf_fock_device, which runs the same contraction with its own workspace.
The file sorts last so that it runs after every other test in one process; it
also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from gb200 import lib, solvers
from _systems import rel, system

TOL = 1e-10  # relative, the tolerance of the FP64 Fock parity tests


def _hermitian(rng, shape, n):
    a = rng.standard_normal(shape + (n, n)) + 1j * rng.standard_normal(shape + (n, n))
    return 0.5 * (a + np.conj(np.swapaxes(a, -1, -2)))


def _full_from_half(V_half, nk):
    """Full pair storage [nk, nk, NQ, nao, nao] on the device from the stored pairs k1 >= k2."""
    import torch
    h = torch.from_numpy(V_half).cuda()
    rows = []
    for k1 in range(nk):
        row = []
        for k2 in range(nk):
            if k1 >= k2:
                row.append(h[k1 * (k1 + 1) // 2 + k2])
            else:
                row.append(h[k2 * (k2 + 1) // 2 + k1].transpose(-1, -2).conj())
        rows.append(torch.stack(row))
    return torch.stack(rows).resolve_conj().contiguous()


def _case_small(name):
    s = system(name)
    ctx = solvers.make_context(s)
    pref = -1.0 if s.ns == 2 else -2.0
    dms = [pref * np.ascontiguousarray(s.G[-1])]
    rng = np.random.default_rng(11)
    dms.append(dms[0] + 0.1 * _hermitian(rng, (s.ns, s.nk), s.nao))
    return ctx, (s.nk, s.nao, s.ns, s.NQ), s.V_half, np.ascontiguousarray(s.S), dms


def _case_blocked():
    """nk = 9, nao = 32, NQ = 400, ns = 2: the exchange work area holds 5 of the 9 k' at once, so the
    exchange term runs in two blocks of k' (5 and 4)."""
    mesh, nao, NQ, ns = (3, 3, 1), 32, 400, 2
    nk = 9
    rng = np.random.default_rng(5)
    npair = nk * (nk + 1) // 2
    V_half = (rng.standard_normal((npair, NQ, nao, nao)) + 1j * rng.standard_normal((npair, NQ, nao, nao))) * 0.05
    for k in range(nk):
        d = V_half[k * (k + 1) // 2 + k]
        V_half[k * (k + 1) // 2 + k] = 0.5 * (d + np.conj(np.swapaxes(d, -1, -2)))
    S = _hermitian(rng, (ns, nk), nao) * 0.05 + np.eye(nao)
    dms = [_hermitian(rng, (ns, nk), nao) * 0.1 for _ in range(2)]
    ctx = lib.Context(nk, nao, ns, NQ, 4, 2, 3, 10.0)
    kp, km = solvers.kq_maps(mesh)
    ctx.set_kq_maps(kp, km)
    ctx.set_integrals(V_half, lib.INTEGRALS_GW)
    return ctx, (nk, nao, ns, NQ), V_half, np.ascontiguousarray(S), dms


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["small", "small_ns2", "blocked"])
def test_noalloc_matches_device_entry_point(gpu, case):
    import torch
    ctx, (nk, nao, ns, NQ), V_half, S, dms = _case_blocked() if case == "blocked" else _case_small(case)
    madelung = 0.37
    stream = torch.cuda.current_stream().cuda_stream
    V = _full_from_half(V_half, nk)
    S_d = torch.from_numpy(S).cuda()
    dm_d = [torch.from_numpy(np.ascontiguousarray(d)).cuda() for d in dms]
    want = []
    for d in dm_d:
        F = torch.empty_like(d)
        ctx.hf_fock_device(d.data_ptr(), S_d.data_ptr(), madelung, F.data_ptr(), stream)
        want.append(F)
    got = [torch.full_like(d, float("nan")) for d in dm_d]
    torch.cuda.synchronize()
    for i, d in enumerate(dm_d):
        if i == 1:
            free_before = torch.cuda.mem_get_info()[0]
        lib.hf_fock_noalloc(nk, nao, ns, NQ, V.data_ptr(), d.data_ptr(), S_d.data_ptr(), madelung,
                            got[i].data_ptr(), stream)
        torch.cuda.synchronize()
        if i == 1:
            assert torch.cuda.mem_get_info()[0] == free_before, "second call changed the free device memory"
    for i in range(2):
        w, g = want[i].cpu().numpy(), got[i].cpu().numpy()
        assert np.isfinite(g).all()
        assert rel(g, w) < TOL, (case, i, rel(g, w))
    assert rel(want[1].cpu().numpy(), want[0].cpu().numpy()) > 1e-6  # the two calls had different inputs


@pytest.mark.gpu
def test_noalloc_matches_oracle(gpu):
    """The allocation-free Fock build against the CPU oracle's restatement of hf_scalar_cpu_kernel, with a
    nonzero Madelung constant, on the spin-polarised small system."""
    import torch
    from _systems import oracle_fock
    s = system("small_ns2")
    madelung = 0.37
    want = oracle_fock(s, madelung)
    pref = -1.0 if s.ns == 2 else -2.0
    dm = torch.from_numpy(np.ascontiguousarray(pref * s.G[-1])).cuda()
    V = _full_from_half(s.V_half, s.nk)
    S_d = torch.from_numpy(np.ascontiguousarray(s.S)).cuda()
    F = torch.full_like(dm, float("nan"))
    stream = torch.cuda.current_stream().cuda_stream
    lib.hf_fock_noalloc(s.nk, s.nao, s.ns, s.NQ, V.data_ptr(), dm.data_ptr(), S_d.data_ptr(), madelung,
                        F.data_ptr(), stream)
    torch.cuda.synchronize()
    assert rel(F.cpu().numpy(), want) < TOL


def test_noalloc_rejects_two_component_input():
    """Two-component dimensions (nso = 2 nao) fail with GB200_ERR_INVALID before any device work."""
    L = lib.load()
    d = lib.Dims(4, 3, 6, 1, 10, 0, 0, 0, 0.0)
    fake = ctypes.c_void_p(256)  # never dereferenced: the dimension check comes first
    rc = L.gb200_hf_fock_noalloc(ctypes.byref(d), fake, fake, fake, 0.0, fake, None)
    assert rc == lib.ERR_INVALID
    assert "two-component" in L.gb200_last_error(None).decode()


def test_noalloc_rejects_sizes_beyond_the_workspace():
    """Sizes whose workspace exceeds the fixed array fail before any device work."""
    L = lib.load()
    d = lib.Dims(125, 80, 80, 2, 2000, 0, 0, 0, 0.0)
    fake = ctypes.c_void_p(256)  # never dereferenced: the size check comes first
    rc = L.gb200_hf_fock_noalloc(ctypes.byref(d), fake, fake, fake, 0.0, fake, None)
    assert rc == lib.ERR_INVALID
    msg = L.gb200_last_error(None).decode()
    assert "above the fixed maximum" in msg and "bytes" in msg
