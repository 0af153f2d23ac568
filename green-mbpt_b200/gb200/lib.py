"""ctypes binding of libgb200.so (the C ABI declared in include/gb200.h).

Only plain pointers cross the boundary: numpy complex128 arrays (host entry
points) or raw device addresses such as ``torch.Tensor.data_ptr()`` (device
entry points).  Status codes become the exception classes of the reference
(green-mbpt src/green/mbpt/except.h:28-56).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgb200.so")

OK = 0
ERR_INVALID = 1
ERR_WRONG_GRID = 2
ERR_MU_SEARCH = 3
ERR_OUTDATED_INPUT = 4
ERR_CUDA = 5
ERR_OOM = 6
ERR_STATE = 7
ERR_NONFINITE = 8

PREC_FP64 = 0
PREC_SPLIT = 1
INTEGRALS_GW = 0
INTEGRALS_HF = 1


class mbpt_kernel_error(RuntimeError):
    """Kernel failure (except.h:28-31)."""


class mbpt_wrong_grid(RuntimeError):
    """Unsupported imaginary-time grid (except.h:33-36)."""


class mbpt_chemical_potential_search_failure(RuntimeError):
    """Stalled mu bisection (except.h:38-41)."""


class mbpt_outdated_input(RuntimeError):
    """Integral files older than the supported format (except.h:43-46)."""


_EXC = {
    ERR_WRONG_GRID: mbpt_wrong_grid,
    ERR_MU_SEARCH: mbpt_chemical_potential_search_failure,
    ERR_OUTDATED_INPUT: mbpt_outdated_input,
}

EXPORTED = [
    "gb200_version", "gb200_check_integral_version", "gb200_create", "gb200_destroy", "gb200_last_error",
    "gb200_set_kq_maps", "gb200_set_grid", "gb200_set_integrals", "gb200_set_precision", "gb200_gw_sigma",
    "gb200_gw_sigma_device", "gb200_hf_fock", "gb200_hf_fock_device", "gb200_dyson_set_hamiltonian",
    "gb200_dyson_find_mu", "gb200_dyson_compute_G", "gb200_dyson_electrons", "gb200_energy",
    "gb200_iteration_device", "gb200_last_timings", "gb200_set_split_engine", "gb200_set_integrals_device",
    "gb200_set_q_range", "gb200_dyson_solve_device", "gb200_energy_device", "gb200_stats_enable", "gb200_stats_read",
    "gb200_hf_fock_noalloc", "gb200_set_q0_correction", "gb200_gw_sigma_vjp", "gb200_gw_sigma_vjp_device",
    "gb200_set_contraction_slices", "gb200_set_memory_budget", "gb200_set_integrals_pairs",
    "gb200_gw_sigma_batch_device", "gb200_set_tile_width",
]


class Dims(ctypes.Structure):
    _fields_ = [("nk", ctypes.c_int32), ("nao", ctypes.c_int32), ("nso", ctypes.c_int32), ("ns", ctypes.c_int32),
                ("NQ", ctypes.c_int32), ("nts", ctypes.c_int32), ("nw", ctypes.c_int32), ("nw_b", ctypes.c_int32),
                ("beta", ctypes.c_double)]


_lib = None


def load(path: str | None = None):
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise mbpt_kernel_error(f"libgb200.so not found at {p}; build it with green-mbpt_b200/build.py")
    L = ctypes.CDLL(p)
    vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int
    L.gb200_version.restype = ctypes.c_char_p
    L.gb200_check_integral_version.argtypes = [ctypes.c_char_p]
    L.gb200_create.argtypes = [ctypes.POINTER(Dims), ip, ctypes.POINTER(vp)]
    L.gb200_destroy.argtypes = [vp]
    L.gb200_destroy.restype = None
    L.gb200_last_error.argtypes = [vp]
    L.gb200_last_error.restype = ctypes.c_char_p
    L.gb200_set_kq_maps.argtypes = [vp, vp, vp]
    L.gb200_set_grid.argtypes = [vp, vp, vp, vp, vp, vp]
    L.gb200_set_integrals.argtypes = [vp, ip, vp, ctypes.c_int64]
    L.gb200_set_precision.argtypes = [vp, ip, ip]
    L.gb200_gw_sigma.argtypes = [vp, vp, vp]
    L.gb200_gw_sigma_device.argtypes = [vp, vp, vp, vp]
    L.gb200_gw_sigma_vjp.argtypes = [vp, vp, vp, vp, vp]
    L.gb200_set_contraction_slices.argtypes = [vp, vp]
    L.gb200_set_memory_budget.argtypes = [vp, ctypes.c_double]
    L.gb200_gw_sigma_vjp_device.argtypes = [vp, vp, vp, vp, vp, vp]
    L.gb200_hf_fock.argtypes = [vp, vp, vp, ctypes.c_double, vp]
    L.gb200_hf_fock_device.argtypes = [vp, vp, vp, ctypes.c_double, vp, vp]
    L.gb200_dyson_set_hamiltonian.argtypes = [vp, vp, vp]
    L.gb200_dyson_find_mu.argtypes = [vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, dp, dp]
    L.gb200_dyson_compute_G.argtypes = [vp, vp, vp, ctypes.c_double, vp]
    L.gb200_dyson_electrons.argtypes = [vp, vp, vp, ctypes.c_double, dp]
    L.gb200_energy.argtypes = [vp, vp, vp, vp, dp]
    L.gb200_iteration_device.argtypes = [vp, vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, dp, dp, vp]
    L.gb200_last_timings.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    L.gb200_set_split_engine.argtypes = [vp, ip]
    L.gb200_set_integrals_device.argtypes = [vp, ip, vp, ctypes.c_int64, ctypes.c_int64, vp]
    L.gb200_set_q_range.argtypes = [vp, ip, ip]
    L.gb200_dyson_solve_device.argtypes = [vp, vp, vp, ctypes.c_double, ctypes.c_double, dp, vp, vp]
    L.gb200_energy_device.argtypes = [vp, vp, vp, vp, dp, vp]
    L.gb200_stats_enable.argtypes = [vp, ip]
    ll = ctypes.POINTER(ctypes.c_longlong)
    L.gb200_stats_read.argtypes = [vp, ll, ll, dp, dp]
    L.gb200_hf_fock_noalloc.argtypes = [ctypes.POINTER(Dims), vp, vp, vp, ctypes.c_double, vp, vp]
    L.gb200_set_q0_correction.argtypes = [vp, vp, vp, ctypes.c_double]
    L.gb200_set_integrals_pairs.argtypes = [vp, vp, vp, ctypes.c_int64, ip, vp]
    L.gb200_gw_sigma_batch_device.argtypes = [vp, ip, vp, vp, vp]
    L.gb200_set_tile_width.argtypes = [vp, ip]
    _lib = L
    return L


def _ptr(a: np.ndarray):
    if not a.flags.c_contiguous:
        raise ValueError("arrays passed to gb200 must be C-contiguous")
    return a.ctypes.data_as(ctypes.c_void_p)


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


class Context:
    """One engine context on one GPU (the kernel object of the plug-in factory)."""

    def __init__(self, nk, nao, ns, NQ, nts, nw, nw_b, beta, nso=None, device=0):
        L = load()
        self._L = L
        self.dims = Dims(nk, nao, nao if nso is None else nso, ns, NQ, nts, nw, nw_b, beta)
        h = ctypes.c_void_p()
        rc = L.gb200_create(ctypes.byref(self.dims), device, ctypes.byref(h))
        if rc != OK:
            msg = L.gb200_last_error(None).decode()
            raise _EXC.get(rc, mbpt_kernel_error)(f"gb200_create failed ({rc}): {msg}")
        self._h = h

    # -- plumbing -------------------------------------------------------------
    def _check(self, rc):
        if rc != OK:
            msg = self._L.gb200_last_error(self._h).decode()
            raise _EXC.get(rc, mbpt_kernel_error)(f"gb200 error {rc}: {msg}")

    def close(self):
        if getattr(self, "_h", None):
            self._L.gb200_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def shape_G(self):
        d = self.dims
        return (d.nts, d.ns, d.nk, d.nso, d.nso)

    @property
    def shape_F(self):
        d = self.dims
        return (d.ns, d.nk, d.nso, d.nso)

    # -- set-up -----------------------------------------------------------------
    def set_kq_maps(self, kplus, kminus):
        kp = np.ascontiguousarray(kplus, dtype=np.int32)
        km = np.ascontiguousarray(kminus, dtype=np.int32)
        self._check(self._L.gb200_set_kq_maps(self._h, _ptr(kp), _ptr(km)))

    def set_grid(self, Tnt_f, Ttn_f, Tnt_b, Ttn_b, wsample_f):
        arrs = [_c128(Tnt_f), _c128(Ttn_f), _c128(Tnt_b), _c128(Ttn_b)]
        w = np.ascontiguousarray(wsample_f, dtype=np.float64)
        self._check(self._L.gb200_set_grid(self._h, *[_ptr(a) for a in arrs], _ptr(w)))

    def set_integrals(self, V_half, which=INTEGRALS_GW):
        V = _c128(V_half)
        self._check(self._L.gb200_set_integrals(self._h, which, _ptr(V), V.shape[0]))

    def set_precision(self, mode=PREC_FP64, slices=4):
        self._check(self._L.gb200_set_precision(self._h, mode, slices))

    def set_contraction_slices(self, slices=None):
        """Slices of the six split contractions: P0 (a)-(c), Sigma (d)-(f); 0 keeps the count of
        set_precision, None resets all six."""
        if slices is None:
            self._check(self._L.gb200_set_contraction_slices(self._h, None))
            return
        if len(slices) != 6:
            raise ValueError("six slice counts: P0 (a)-(c), Sigma (d)-(f)")
        arr = (ctypes.c_int * 6)(*[int(x) for x in slices])
        self._check(self._L.gb200_set_contraction_slices(self._h, arr))

    def set_memory_budget(self, nbytes: float):
        """Bytes the blocked intermediates of one call may use (0: a share of the free memory)."""
        self._check(self._L.gb200_set_memory_budget(self._h, float(nbytes)))

    def set_split_engine(self, engine: int):
        """0: tcgen05 tensor cores, 1: CUDA-core validation engine (bit-identical INT32 sums)."""
        self._check(self._L.gb200_set_split_engine(self._h, engine))

    def set_hamiltonian(self, H, S):
        self._H, self._S = _c128(H), _c128(S)
        self._check(self._L.gb200_dyson_set_hamiltonian(self._h, _ptr(self._H), _ptr(self._S)))

    # -- host entry points --------------------------------------------------------
    def gw_sigma(self, G):
        G = _c128(G)
        out = np.empty(self.shape_G, dtype=np.complex128)
        self._check(self._L.gb200_gw_sigma(self._h, _ptr(G), _ptr(out)))
        return out

    def gw_sigma_vjp(self, G, Sigma_bar, with_V: bool = False):
        """Gb = d/dG of Re sum conj(Sigma_bar) Sigma(G, V) (FP64); with_V also returns Vb, the
        gradient with respect to the half-stored integrals: (Gb, Vb)."""
        G, Sb = _c128(G), _c128(Sigma_bar)
        out = np.empty(self.shape_G, dtype=np.complex128)
        d = self.dims
        Vb = np.empty((d.nk * (d.nk + 1) // 2, d.NQ, d.nao, d.nao), dtype=np.complex128) if with_V else None
        self._check(self._L.gb200_gw_sigma_vjp(self._h, _ptr(G), _ptr(Sb), _ptr(out),
                                               _ptr(Vb) if with_V else None))
        return (out, Vb) if with_V else out

    def hf_fock(self, dm, S, madelung=0.0):
        dm, S = _c128(dm), _c128(S)
        out = np.empty(self.shape_F, dtype=np.complex128)
        self._check(self._L.gb200_hf_fock(self._h, _ptr(dm), _ptr(S), float(madelung), _ptr(out)))
        return out

    def find_mu(self, Sigma1, Sigma_tau, mu0, nel, tol=1e-9):
        S1, St = _c128(Sigma1), _c128(Sigma_tau)
        mu = ctypes.c_double()
        n = ctypes.c_double()
        self._check(self._L.gb200_dyson_find_mu(self._h, _ptr(S1), _ptr(St), mu0, nel, tol, ctypes.byref(mu),
                                                ctypes.byref(n)))
        return n.value, mu.value

    def electrons(self, Sigma1, Sigma_tau, mu):
        S1, St = _c128(Sigma1), _c128(Sigma_tau)
        n = ctypes.c_double()
        self._check(self._L.gb200_dyson_electrons(self._h, _ptr(S1), _ptr(St), mu, ctypes.byref(n)))
        return n.value

    def compute_G(self, Sigma1, Sigma_tau, mu):
        """Returns (G_tau, Sigma1_hermitized, Sigma_tau_hermitized)."""
        S1, St = _c128(Sigma1).copy(), _c128(Sigma_tau).copy()
        G = np.empty(self.shape_G, dtype=np.complex128)
        self._check(self._L.gb200_dyson_compute_G(self._h, _ptr(S1), _ptr(St), mu, _ptr(G)))
        return G, S1, St

    def energy(self, G, Sigma1, Sigma_tau):
        G, S1, St = _c128(G), _c128(Sigma1), _c128(Sigma_tau)
        e = (ctypes.c_double * 3)()
        self._check(self._L.gb200_energy(self._h, _ptr(G), _ptr(S1), _ptr(St), e))
        return tuple(e)

    # -- device entry points (raw device addresses) --------------------------------
    def gw_sigma_device(self, G_ptr: int, Sigma_ptr: int, stream: int = 0):
        self._check(self._L.gb200_gw_sigma_device(self._h, ctypes.c_void_p(G_ptr), ctypes.c_void_p(Sigma_ptr),
                                                  ctypes.c_void_p(stream)))

    def gw_sigma_vjp_device(self, G_ptr: int, Sb_ptr: int, Gb_ptr: int, Vb_ptr: int = 0, stream: int = 0):
        self._check(self._L.gb200_gw_sigma_vjp_device(self._h, ctypes.c_void_p(G_ptr), ctypes.c_void_p(Sb_ptr),
                                                      ctypes.c_void_p(Gb_ptr), ctypes.c_void_p(Vb_ptr or None),
                                                      ctypes.c_void_p(stream)))

    def hf_fock_device(self, dm_ptr: int, S_ptr: int, madelung: float, F_ptr: int, stream: int = 0):
        self._check(self._L.gb200_hf_fock_device(self._h, ctypes.c_void_p(dm_ptr), ctypes.c_void_p(S_ptr),
                                                 float(madelung), ctypes.c_void_p(F_ptr), ctypes.c_void_p(stream)))

    def iteration_device(self, G_ptr, Sigma1_ptr, Sigma_ptr, madelung, nel, tol, mu, stream=0, energies=True):
        m = ctypes.c_double(mu)
        e = (ctypes.c_double * 3)()
        self._check(self._L.gb200_iteration_device(self._h, ctypes.c_void_p(G_ptr), ctypes.c_void_p(Sigma1_ptr),
                                                   ctypes.c_void_p(Sigma_ptr), float(madelung), float(nel),
                                                   float(tol), ctypes.byref(m), e if energies else None,
                                                   ctypes.c_void_p(stream)))
        return m.value, (tuple(e) if energies else None)

    def set_integrals_device(self, V_ptr: int, pair_begin: int, pair_count: int, which=INTEGRALS_GW, stream: int = 0):
        """Deliver stored pairs [pair_begin, pair_begin + pair_count) from device memory."""
        self._check(self._L.gb200_set_integrals_device(self._h, which, ctypes.c_void_p(V_ptr), pair_begin, pair_count,
                                                       ctypes.c_void_p(stream)))

    def set_tile_width(self, bn: int = 0):
        """Column tile of the split-precision contractions (0: the widest that fits)."""
        self._check(self._L.gb200_set_tile_width(self._h, int(bn)))

    def set_integrals_pairs(self, V_pairs, pair_ids, stream: int = 0):
        """q-sharded GW integrals: the stored pairs `pair_ids` (increasing half-storage indices,
        gb200.shard.pairs_for_q_range) with their blocks V_pairs [len, NQ, nao, nao]: a host
        array, or the device address of such an array (an int)."""
        ids = np.ascontiguousarray(pair_ids, dtype=np.int64)
        if isinstance(V_pairs, int):
            self._check(self._L.gb200_set_integrals_pairs(self._h, ctypes.c_void_p(V_pairs), _ptr(ids), len(ids), 1,
                                                          ctypes.c_void_p(stream)))
            return
        V = _c128(V_pairs)
        if V.shape[0] != len(ids):
            raise ValueError("set_integrals_pairs: one block per pair index")
        self._check(self._L.gb200_set_integrals_pairs(self._h, _ptr(V), _ptr(ids), len(ids), 0, None))

    def set_q0_correction(self, AqQ, q_abs, madelung: float):
        """The "extrapolate" q -> 0 correction (AqQ [nk, NQ] complex, q_abs [nk]); AqQ=None turns it off."""
        if AqQ is None:
            self._check(self._L.gb200_set_q0_correction(self._h, None, None, 0.0))
            return
        A = _c128(AqQ)
        q = np.ascontiguousarray(q_abs, dtype=np.float64)
        if A.shape != (self.dims.nk, self.dims.NQ) or q.shape != (self.dims.nk,):
            raise ValueError("AqQ must be [nk, NQ] and q_abs [nk]")
        self._check(self._L.gb200_set_q0_correction(self._h, _ptr(A), _ptr(q), float(madelung)))

    def set_q_range(self, q_begin: int, q_end: int):
        self._check(self._L.gb200_set_q_range(self._h, q_begin, q_end))

    def dyson_solve_device(self, Sigma1_ptr, Sigma_ptr, nel, tol, mu, G_ptr, stream=0):
        m = ctypes.c_double(mu)
        self._check(self._L.gb200_dyson_solve_device(self._h, ctypes.c_void_p(Sigma1_ptr), ctypes.c_void_p(Sigma_ptr),
                                                      float(nel), float(tol), ctypes.byref(m), ctypes.c_void_p(G_ptr),
                                                      ctypes.c_void_p(stream)))
        return m.value

    def energy_device(self, G_ptr, Sigma1_ptr, Sigma_ptr, stream=0):
        e = (ctypes.c_double * 3)()
        self._check(self._L.gb200_energy_device(self._h, ctypes.c_void_p(G_ptr), ctypes.c_void_p(Sigma1_ptr),
                                                ctypes.c_void_p(Sigma_ptr), e, ctypes.c_void_p(stream)))
        return tuple(e)

    def stats_enable(self, on=True):
        self._check(self._L.gb200_stats_enable(self._h, 1 if on else 0))

    def stats_read(self):
        """(library launches so far, contraction-kernel launches, their device ms, their FP64-equivalent flops)."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        ms, fl = ctypes.c_double(), ctypes.c_double()
        self._check(self._L.gb200_stats_read(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(ms),
                                             ctypes.byref(fl)))
        return a.value, b.value, ms.value, fl.value

    def last_timings(self):
        t = (ctypes.c_float * 4)()
        self._check(self._L.gb200_last_timings(self._h, t))
        return {"P0": t[0], "W": t[1], "Sigma": t[2], "total": t[3]}


def version():
    return load().gb200_version().decode()


def hf_fock_noalloc(nk: int, nao: int, ns: int, NQ: int, V_ptr: int, dm_ptr: int, S_ptr: int, madelung: float,
                    F_ptr: int, stream: int = 0):
    """Fock matrix into F_ptr with no device allocation by the library (gb200_hf_fock_noalloc).

    For callers that cannot allocate device memory while they run.  All
    pointers are device addresses of complex128 arrays: V [nk][nk][NQ][nao][nao]
    in full storage, dm, S, F [ns][nk][nao][nao].  The work is queued on
    `stream` and runs asynchronously; calls that overlap on the GPU share one
    fixed workspace and race.
    """
    L = load()
    d = Dims(nk, nao, nao, ns, NQ, 0, 0, 0, 0.0)
    rc = L.gb200_hf_fock_noalloc(ctypes.byref(d), ctypes.c_void_p(V_ptr), ctypes.c_void_p(dm_ptr),
                                 ctypes.c_void_p(S_ptr), float(madelung), ctypes.c_void_p(F_ptr),
                                 ctypes.c_void_p(stream))
    if rc != OK:
        msg = L.gb200_last_error(None).decode()
        raise _EXC.get(rc, mbpt_kernel_error)(f"gb200_hf_fock_noalloc failed ({rc}): {msg}")


def check_integral_version(v: str):
    rc = load().gb200_check_integral_version(v.encode())
    if rc == ERR_OUTDATED_INPUT:
        raise mbpt_outdated_input(
            f"Integral files are outdated (version {v}), please run migration script python/migrate.py")
    if rc != OK:
        raise ValueError("Version string format is incorrect. Expected format: major.minor.patch[suffix]")
    return True


def gw_sigma_batch_device(contexts, G_ptrs, Sigma_ptrs, stream: int = 0):
    """gb200_gw_sigma_batch_device: the self-energies of several contexts (device buffers) in one
    call, every contraction stage one grouped tensor-core launch over all systems."""
    n = len(contexts)
    if len(G_ptrs) != n or len(Sigma_ptrs) != n or n == 0:
        raise ValueError("one G and one Sigma buffer per context")
    L = load()
    hs = (ctypes.c_void_p * n)(*[c._h for c in contexts])
    gs = (ctypes.c_void_p * n)(*G_ptrs)
    ss = (ctypes.c_void_p * n)(*Sigma_ptrs)
    rc = L.gb200_gw_sigma_batch_device(hs, n, gs, ss, ctypes.c_void_p(stream))
    contexts[0]._check(rc)
