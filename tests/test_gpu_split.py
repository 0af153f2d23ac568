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
