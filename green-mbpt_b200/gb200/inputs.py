"""green-mbpt's input and integral files, and the k-point symmetry expansion the kernels need.

The library's kernels work on the full Brillouin zone without point-group symmetry.  Inputs
written for green-mbpt (by its PySCF front end) store objects at the irreducible k-points and
the density-fitted integrals for the irreducible k-pairs only.  This module reads those files
and expands them on the host:

* ``read_input``: ``params/{nao,nso,ns,NQ,nk,nel_cell}``, ``HF/{S-k,H-k,Fock-k,madelung}``
  and the ``symmetry/`` tables (the keys of gw_solver.h:62-68, dyson.cpp:26-34 and the
  brillouin_zone_utils reader);
* ``read_integrals``: ``meta.h5`` (``chunk_size``, ``__green_version__``) and the chunk files
  ``VQ_<c>.h5`` holding dataset ``/<c>`` of shape [chunk, NQ, nao, nao] for the irreducible
  k-pairs c .. c + chunk - 1 (df_integral_t.h:40-53,86-92);
* ``KSymmetry``: an object at a full-zone point from its irreducible image, U_k X U_k^H,
  complex-conjugated for time-reversal partners (k_symmetry().value_AO), and a k-pair block of
  the integrals from the irreducible list with the stored-pair conjugate transpose and the
  conjugated / transposed pair symmetries (df_integral_t::read_integrals / wrap / v_type /
  symmetrize, df_integral_t.h:64-84,140-203).
"""
from __future__ import annotations

import os

import numpy as np

from . import lib
from .h5lite import H5File


def _complex(a):
    """HDF5 complex data: a compound {r, i} or a trailing dimension of 2 doubles."""
    a = np.asarray(a)
    if a.dtype.names:
        return a["r"] + 1j * a["i"]
    v = np.ascontiguousarray(a, dtype=np.float64).view(np.complex128)
    return v[..., 0] if v.shape[-1] == 1 else v


def pair_index(k1: int, k2: int) -> int:
    """Index of the stored pair of (k1, k2): k1 >= k2 only, k1 (k1 + 1) / 2 + k2 (df_integral_t.h:68)."""
    return k1 * (k1 + 1) // 2 + k2 if k1 >= k2 else k2 * (k2 + 1) // 2 + k1


class KSymmetry:
    """k-point and k-pair symmetry tables of a green-mbpt input file."""

    def __init__(self, bz2ibz, ibz2bz, tr_conj, transform_ao, conj_pairs, trans_pairs, kpair_irre, weight_ibz=None):
        self.bz2ibz = np.asarray(bz2ibz, dtype=np.int64)
        self.ibz2bz = np.asarray(ibz2bz, dtype=np.int64)
        self.tr_conj = np.asarray(tr_conj).astype(bool)
        self.U = np.asarray(transform_ao, dtype=np.complex128)
        self.conj_pairs = np.asarray(conj_pairs, dtype=np.int64)
        self.trans_pairs = np.asarray(trans_pairs, dtype=np.int64)
        self.kpair_irre = np.asarray(kpair_irre, dtype=np.int64)
        self.weight_ibz = None if weight_ibz is None else np.asarray(weight_ibz)
        self.nk = len(self.bz2ibz)
        self.ink = len(self.ibz2bz)
        # position of a full-zone point's irreducible representative in the ibz arrays
        ibz_pos = np.full(self.nk, -1, dtype=np.int64)
        ibz_pos[self.ibz2bz] = np.arange(self.ink)
        self.reduced = ibz_pos[self.bz2ibz]
        if (self.reduced < 0).any():
            raise ValueError("symmetry tables: bz2ibz points outside ibz2bz")
        # position of a stored irreducible pair in the integral files
        self.irre_pos = np.full(self.nk * (self.nk + 1) // 2, -1, dtype=np.int64)
        self.irre_pos[self.kpair_irre] = np.arange(len(self.kpair_irre))

    @classmethod
    def from_file(cls, f: H5File):
        r = lambda p: f.read("symmetry/" + p)
        return cls(r("k/bz2ibz"), r("k/ibz2bz"), r("k/tr_conj"), _complex(r("k/k_sym_transform_ao")),
                   r("pairs/conj_pairs_list"), r("pairs/trans_pairs_list"), r("pairs/kpair_irre_list"),
                   r("k/weight_ibz"))

    # -- one-point objects -------------------------------------------------------------------
    def value_AO(self, X_ibz, k: int):
        """X at full-zone point k from the irreducible objects X_ibz [ink, n, n]."""
        Y = X_ibz[self.reduced[k]]
        U = self.U[k]
        Y = U @ Y @ np.conj(U.T)
        return np.conj(Y) if self.tr_conj[k] else Y

    def full_from_ibz(self, X_ibz):
        """[..., ink, n, n] -> [..., nk, n, n]; irreducible points are copied unchanged."""
        X_ibz = np.asarray(X_ibz)
        lead = X_ibz.shape[:-3]
        flat = X_ibz.reshape((-1,) + X_ibz.shape[-3:])
        out = np.empty((flat.shape[0], self.nk) + X_ibz.shape[-2:], dtype=np.complex128)
        for b in range(flat.shape[0]):
            for k in range(self.nk):
                out[b, k] = self.value_AO(flat[b], k)
            out[b, self.ibz2bz] = flat[b]
        return out.reshape(lead + out.shape[1:])

    def ibz_from_full(self, X_full):
        """[..., nk, n, n] -> [..., ink, n, n] at the irreducible points."""
        return np.asarray(X_full)[..., self.ibz2bz, :, :]

    # -- k-pair integrals --------------------------------------------------------------------
    def pair(self, store, k1: int, k2: int):
        """V^Q(k1, k2) [NQ, nao, nao] from the irreducible pair blocks `store`."""
        idx = pair_index(k1, k2)
        kind = "direct"
        if self.conj_pairs[idx] != idx:
            idx, kind = int(self.conj_pairs[idx]), "conj"
        elif self.trans_pairs[idx] != idx:
            idx, kind = int(self.trans_pairs[idx]), "trans"
        pos = self.irre_pos[idx]
        if pos < 0:
            raise ValueError(f"k-pair ({k1}, {k2}) resolves to a pair that is not stored")
        v = store[pos]
        v = np.conj(np.swapaxes(v, -1, -2)) if k1 < k2 else np.array(v)
        if kind == "conj":
            v = np.conj(v)
        elif kind == "trans":
            v = np.swapaxes(v, -1, -2)
        return np.ascontiguousarray(v)

    def half_storage(self, store):
        """All stored pairs k1 >= k2 of the full zone, [nk (nk + 1) / 2, NQ, nao, nao]: the layout
        of gb200_set_integrals."""
        return np.stack([self.pair(store, k1, k2) for k1 in range(self.nk) for k2 in range(k1 + 1)])


def kq_maps_from_points(frac):
    """k + q and k - q tables of a k-mesh given by fractional coordinates [nk, 3].

    kplus[k, q] = index of frac(k) + frac(q) and kminus[k, q] = index of frac(k) - frac(q),
    modulo reciprocal lattice vectors: brillouin_zone_utils::k_q_map's k1_from_k2q / k2_from_k1q
    (call sites gw_cpu_kernel.cpp:90,117) for a mesh without symmetry reduction of q.
    """
    f = np.asarray(frac, dtype=np.float64)
    nk = f.shape[0]

    def lookup(target):  # target [nk, nk, 3] -> indices [nk, nk]
        d = target[:, :, None, :] - f[None, None, :, :]
        d = np.abs(d - np.round(d)).max(axis=-1)
        idx = np.argmin(d, axis=-1)
        if (np.take_along_axis(d, idx[..., None], axis=-1) > 1e-6).any():
            raise ValueError("k-point set is not closed under addition (not a full Monkhorst-Pack mesh)")
        return idx.astype(np.int32)

    return lookup(f[:, None, :] + f[None, :, :]), lookup(f[:, None, :] - f[None, :, :])


def read_input(path: str) -> dict:
    """Parameters, Hamiltonian blocks and symmetry of a green-mbpt input file (input.h5)."""
    f = H5File(path)
    p = lambda k: f.read("params/" + k)
    out = dict(nao=int(p("nao")), nso=int(p("nso")), ns=int(p("ns")), NQ=int(p("NQ")), nk=int(p("nk")))
    try:
        out["nel_cell"] = float(p("nel_cell"))
    except Exception:
        out["nel_cell"] = None
    sym = KSymmetry.from_file(f)
    ns, nso, ink = out["ns"], out["nso"], sym.ink
    for key, name in (("S-k", "S_ibz"), ("H-k", "H_ibz"), ("Fock-k", "F_ibz")):
        try:
            a = _complex(f.read("HF/" + key))
        except Exception:
            continue
        # stored for the full zone or for the irreducible points only
        a = a.reshape(ns, -1, nso, nso)
        out[name] = a[:, sym.ibz2bz] if a.shape[1] == sym.nk and ink != sym.nk else a
    try:
        out["madelung"] = float(f.read("HF/madelung"))
    except Exception:
        out["madelung"] = 0.0
    try:
        out["k_frac"] = np.asarray(f.read("symmetry/k/mesh_scaled"), dtype=np.float64)
    except Exception:
        out["k_frac"] = None
    out["symmetry"] = sym
    return out


def read_integrals(dirpath: str, npairs: int | None = None):
    """Irreducible k-pair blocks of the density-fitted integrals from an integral directory.

    Returns (store [npairs, NQ, nao, nao] complex128, version string).  The version attribute
    of meta.h5 is checked as CheckVersion does (mbpt_outdated_input when too old or missing).
    """
    meta = H5File(os.path.join(dirpath, "meta.h5"))
    try:
        version = meta.attr("/", "__green_version__")
    except Exception:
        version = None
    if version is None:
        raise lib.mbpt_outdated_input(
            f"Integral files at '{dirpath}' are outdated, please run migration script python/migrate.py")
    version = version.decode() if isinstance(version, (bytes, np.bytes_)) else str(version)
    lib.check_integral_version(version)
    chunk = int(meta.read("chunk_size"))
    try:
        starts = [int(c) for c in np.atleast_1d(meta.read("chunk_indices"))]
    except Exception:
        starts = None
    if starts is None:
        starts = []
        c = 0
        while os.path.exists(os.path.join(dirpath, f"VQ_{c}.h5")):
            starts.append(c)
            c += chunk
    blocks = []
    for c in sorted(starts):
        a = _complex(H5File(os.path.join(dirpath, f"VQ_{c}.h5")).read(f"/{c}"))
        blocks.append(a)
    store = np.concatenate(blocks, axis=0)
    if npairs is not None:
        if store.shape[0] < npairs:
            raise ValueError(f"integral files hold {store.shape[0]} k-pairs, {npairs} expected")
        store = store[:npairs]
    return np.ascontiguousarray(store), version


def read_q0(path: str):
    """AqQ.h5 of the "extrapolate" q -> 0 treatment (mbpt_q0_utils_t.h:18-36): returns
    (AqQ [nq_stored, NQ] complex, q_abs [nq_stored], madelung)."""
    f = H5File(path)
    A = _complex(f.read("AqQ"))
    q_abs = np.asarray(f.read("q_abs"), dtype=np.float64).reshape(-1)
    try:
        mad = float(np.asarray(f.read("madelung")))
    except Exception:
        mad = None
    if A.shape[0] != q_abs.shape[0]:
        raise ValueError("AqQ.h5: AqQ and q_abs disagree on the number of q-points")
    return np.ascontiguousarray(A), q_abs, mad


def q0_full_zone(AqQ_ibz, q_abs_ibz, ibz2bz_q, nq: int):
    """Full-zone arrays for gb200_set_q0_correction from the irreducible ones: the irreducible
    q-points keep their AqQ row and |q|, the others get |q| = 0, which excludes them from the
    q -> 0 fit, so the fit uses the same points as the reference's loop over irreducible q."""
    AqQ_ibz = np.asarray(AqQ_ibz)
    ibz2bz_q = np.asarray(ibz2bz_q, dtype=np.int64)
    if AqQ_ibz.shape[0] != len(ibz2bz_q):
        raise ValueError(f"AqQ holds {AqQ_ibz.shape[0]} q-points, the symmetry tables {len(ibz2bz_q)} irreducible ones")
    if len(ibz2bz_q) > 1 and (np.diff(ibz2bz_q) <= 0).any():
        raise ValueError("irreducible q-points must be listed in increasing full-zone order")
    A = np.zeros((nq, AqQ_ibz.shape[1]), dtype=np.complex128)
    q = np.zeros(nq)
    A[ibz2bz_q] = AqQ_ibz
    q[ibz2bz_q] = np.asarray(q_abs_ibz)
    return A, q

