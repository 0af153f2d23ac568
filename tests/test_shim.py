"""The green-mbpt plug-in (green-mbpt_b200/shim/gb200_green_kernel.{h,cpp}) built and driven.

The plug-in is C++ against green-mbpt's own types.  tests/shim/green/ holds stand-ins for the
members it uses (params, shared_object, transformer_t, brillouin_zone_utils, df_integral_t,
ztensor); tests/shim/shim_driver.cpp obtains the kernels from custom_hf_kernel / custom_gw_kernel
as green-mbpt's kernel factories do (kernel_factory.h:28-36,86-108) and runs one callback.

* CPU: the plug-in and the driver compile with warnings as errors and link against libgb200.so.
* GPU: the HF callback on the reference's HF fixture (27 k-points, 4 irreducible, symmetry-reduced
  G and integral chunk) reproduces ``result/Sigma1`` at the reference test's 1e-10
  (solvers_test.cpp:27-78), and the GW callback on the reference's GW fixture reproduces
  ``result/Sigma_tau`` at 1e-6 (solvers_test.cpp:80-135): the k-symmetry expansion, the integral
  symmetrization and the unit-vector transforms all run in the plug-in's C++.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "green-mbpt_b200", "shim")
STUBS = os.path.join(ROOT, "tests", "shim")
LIBDIR = os.path.join(ROOT, "green-mbpt_b200", "gb200")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _build(out_dir):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = os.path.join(out_dir, "shim_driver")
    cmd = [gxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", STUBS, "-I", os.path.join(ROOT, "include"),
           "-I", SHIM, os.path.join(STUBS, "shim_driver.cpp"), os.path.join(SHIM, "gb200_green_kernel.cpp"),
           "-L", LIBDIR, "-lgb200", "-Wl,--allow-shlib-undefined", "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def _save(d, name, a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    a.tofile(os.path.join(d, name + ".bin"))
    with open(os.path.join(d, name + ".shape"), "w") as f:
        f.write(" ".join(str(x) for x in a.shape))


def _write_case(d, fx, dims, q0="IGNORE_G0", grid=None):
    from gb200 import inputs
    os.makedirs(d, exist_ok=True)
    nao, nso, ns, NQ, madelung, beta = dims
    with open(os.path.join(d, "dims.txt"), "w") as f:
        f.write(f"{nao} {nso} {ns} {NQ} {madelung!r} {beta!r} {q0}\n")
    kp, km = inputs.kq_maps_from_points(fx["k_frac"])
    _save(d, "kplus", kp, np.int64)
    _save(d, "kminus", km, np.int64)
    for key in ("bz2ibz", "ibz2bz", "tr_conj", "conj_pairs_list", "trans_pairs_list", "kpair_irre_list"):
        _save(d, key, fx[key], np.int64)
    _save(d, "k_sym_transform_ao", fx["k_sym_transform_ao"], np.complex128)
    _save(d, "S_ibz", fx["S_ibz"], np.complex128)
    _save(d, "V_chunk", fx["V_chunk"], np.complex128)
    if grid is not None:
        for key in ("Tnt_f", "Ttn_f", "Tnt_b", "Ttn_b"):
            _save(d, key, getattr(grid, key), np.complex128)
        _save(d, "wsample_f", grid.wsample_f, np.float64)


def _run(exe, d, mode):
    r = subprocess.run([exe, d, mode], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr


def test_shim_builds_against_stub_headers(tmp_path):
    exe = _build(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_shim_hf_callback_reproduces_reference_fixture(tmp_path, gpu):
    fx = dict(np.load(os.path.join(GOLDEN, "hf.npz")))
    ns, nao, nso, NQ = int(fx["ns"]), int(fx["nao"]), int(fx["nso"]), int(fx["NQ"])
    d = str(tmp_path / "hf")
    _write_case(d, fx, (nao, nso, ns, NQ, float(fx["madelung"]), 100.0))
    dm = (-1.0 if ns == 2 else -2.0) * fx["G_beta"]  # spin prefactor (hf_solver.h:38)
    _save(d, "dm", dm, np.complex128)
    _run(_build(str(tmp_path)), d, "hf")
    F = np.fromfile(os.path.join(d, "F.bin"), dtype=np.complex128).reshape(fx["Sigma1"].shape)
    np.testing.assert_allclose(F, fx["Sigma1"], rtol=0, atol=1e-10)


@pytest.mark.gpu
def test_shim_gw_callback_reproduces_reference_fixture(tmp_path, gpu):
    import _gw_golden as GG
    fx = GG.case("gw")
    d = str(tmp_path / "gw")
    _write_case(d, fx, (fx["nao"], fx["nso"], fx["ns"], fx["NQ"], float(fx["madelung"]), fx["beta"]), grid=GG.grid())
    _save(d, "G", fx["G_tau"], np.complex128)
    _run(_build(str(tmp_path)), d, "gw")
    Sigma = np.fromfile(os.path.join(d, "Sigma.bin"), dtype=np.complex128).reshape(fx["Sigma_tau"].shape)
    assert float(np.abs(Sigma - fx["Sigma_tau"]).max()) < GG.REF_TOL
    ref = GG.oracle_sigma("gw")
    assert float(np.abs(Sigma - ref).max() / np.abs(ref).max()) < 1e-10
