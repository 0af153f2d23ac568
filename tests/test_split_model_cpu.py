"""The CPU model of the split-precision arithmetic (oracle/split_model.py), which attributes the
split-vs-FP64 error of the self-energy to the individual contractions."""
import numpy as np


def test_split_model_error_falls_by_the_digit_base():
    """The CPU model of the split arithmetic (oracle/split_model.py): each added slice divides the
    error of a product by about 2^7, and small integers are represented exactly."""
    import split_model as SM
    rng = np.random.default_rng(3)
    A = rng.standard_normal((24, 40)) + 1j * rng.standard_normal((24, 40))
    B = rng.standard_normal((40, 16)) + 1j * rng.standard_normal((40, 16))
    ref = A @ B
    errs = [np.abs(SM.split_mm(A, B, S) - ref).max() / np.abs(ref).max() for S in (2, 3, 4, 5, 6)]
    for a, b in zip(errs, errs[1:]):
        assert 40 < a / b < 400
    Ai = rng.integers(-50, 50, (8, 12)) + 1j * rng.integers(-50, 50, (8, 12))
    Bi = rng.integers(-50, 50, (12, 6)) + 1j * rng.integers(-50, 50, (12, 6))
    assert np.array_equal(SM.split_mm(Ai, Bi, 3), Ai @ Bi)


def test_balanced_digits_remove_the_bias_of_truncation():
    """For sums of same-signed products (the sign-correlated case), truncation toward zero biases
    every term the same way and its error grows with the contraction length; rounding to nearest
    with balanced digits does not."""
    import split_model as SM
    rng = np.random.default_rng(4)
    A = rng.uniform(0.5, 1.0, (16, 4000)) + 0j
    B = rng.uniform(0.5, 1.0, (4000, 8)) + 0j
    ref = A @ B
    trunc = np.abs(SM.split_mm(A, B, 4, "truncated") - ref).max()
    bal = np.abs(SM.split_mm(A, B, 4) - ref).max()
    assert bal < trunc / 10
