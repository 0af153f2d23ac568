"""Split-precision (Ozaki INT8) contractions on the GPU.

* the CUDA-core validation engine and the tcgen05 engine form the same INT32
  diagonal sums from the same slice planes, so their self-energies must agree
  bit for bit;
* the error against the FP64 path falls with the slice count and meets the
  stated tolerance: max|dSigma| <= 1e-8 (absolute, Ha) at 5 slices for these
  systems.
"""
import numpy as np
import pytest

from gb200 import lib, solvers
from _systems import oracle_sigma, system

pytestmark = pytest.mark.gpu


def sigma_split(s, slices, engine):
    with solvers.make_context(s, precision=lib.PREC_SPLIT, slices=slices) as c:
        c.set_split_engine(engine)
        return c.gw_sigma(s.G)


@pytest.mark.parametrize("name", ["small", "small_ns2"])
def test_split_engines_bit_identical(gpu, name):
    s = system(name)
    a = sigma_split(s, 4, 1)
    b = sigma_split(s, 4, 0)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ["small", "c0"])
def test_split_error_vs_fp64(gpu, name):
    s = system(name)
    ref = oracle_sigma(name)
    errs = {}
    for S in (3, 4, 5, 6):
        errs[S] = float(np.abs(sigma_split(s, S, 0) - ref).max())
    assert errs[4] < errs[3] and errs[5] < errs[4]
    assert errs[5] <= 1e-8, errs


def test_full_sigma_within_bound_on_workload_shapes(gpu):
    """One whole iteration from G0, split (5 slices) against FP64, on a system with the headline
    workload's shapes (nao=40, naux=250, ntau=120, nw=120, beta=200, eps ~ U[-5,5]) and a 2x1x1
    mesh: the full self-energy within 1e-8 Ha (|Sigma| reaches about 32 Ha here).  G also goes
    through the chemical-potential bisection (tolerance 1e-9), which can stop one interval apart in
    the two runs, so it is held to 1e-8."""
    import torch
    from gb200 import synth
    s = synth.make_system(mesh=(2, 1, 1), nao=40, naux=250, ns=1, beta=200.0, nts=120, nw=120, eps_range=5.0,
                          seed=0)
    out = {}
    for name, prec in (("fp64", lib.PREC_FP64), ("split", lib.PREC_SPLIT)):
        with solvers.make_context(s, precision=prec, slices=5) as c:
            G = torch.tensor(s.G, dtype=torch.complex128, device="cuda")
            d = c.dims
            S1 = torch.empty((d.ns, d.nk, d.nso, d.nso), dtype=torch.complex128, device="cuda")
            Sig = torch.empty_like(G)
            torch.cuda.synchronize()
            c.iteration_device(G.data_ptr(), S1.data_ptr(), Sig.data_ptr(), 0.0, s.nel_from_G0(), 1e-9, 0.0,
                               stream=0x1, energies=True)
            torch.cuda.synchronize()
            out[name] = (G.cpu().numpy(), Sig.cpu().numpy())
    assert np.abs(out["split"][1] - out["fp64"][1]).max() <= 1e-8
    assert np.abs(out["split"][0] - out["fp64"][0]).max() <= 1e-8


@pytest.mark.parametrize("name", ["small", "small_ns2"])
def test_split_matches_cpu_model_of_its_arithmetic(gpu, name):
    """The GPU split engine against oracle/split_model.py, the CPU restatement of its arithmetic
    (exponents per row and column with one bit of headroom, rounded balanced base-128 digits, kept
    diagonals), at three slices.  On these systems all k-points form one block and no contraction
    is chunked, so both form the same exponent groups and the same exact integer digit products:
    they agree to 1e-10 relative, while both differ from the FP64 result by about 1e-6 relative and
    truncated digits would differ from balanced ones by as much.  (Three slices: the digit quantum,
    2^-21 of the row maximum, is far above the FP64 round-off in which the two differ, so no
    rounding decision of a later contraction's slicing flips between them.)"""
    import split_model as SM
    s = system(name)
    model = SM.gw_split_model(s, {c: 3 for c in "abcdef"})
    with solvers.make_context(s, precision=lib.PREC_SPLIT, slices=3) as c:
        got = c.gw_sigma(s.G)
    scale = np.abs(model).max()
    assert np.abs(got - model).max() <= 1e-10 * scale
    assert np.abs(model - oracle_sigma(name)).max() > 1e-8 * scale


@pytest.mark.parametrize("ns", [1, 2])
def test_exponent_sinks_match_separate_exponent_passes(gpu, ns):
    """With nao a multiple of 8 the tensor-core engine records the column exponents of Y2 (the
    operand of (f)) in the epilogue of (e) as it stores Y2, and skips the slicer's exponent pass
    for Y2; the validation engine still runs that pass.  No contraction is chunked here, so both
    see the same exponents and the self-energies agree bit for bit; at 5 slices both are within
    1e-8 of the FP64 path."""
    from gb200 import synth
    s = synth.make_system(mesh=(2, 2, 1), nao=8, naux=24, ns=ns, beta=20.0, nts=20, eps_range=2.0, seed=5 + ns)
    a = sigma_split(s, 5, 1)
    b = sigma_split(s, 5, 0)
    assert np.array_equal(a, b)
    with solvers.make_context(s, precision=lib.PREC_FP64) as c:
        ref = c.gw_sigma(s.G)
    assert np.abs(b - ref).max() <= 1e-8
