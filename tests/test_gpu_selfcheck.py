"""The FP64 right-hand sides divide by the model's constants with a reciprocal and
two FMA corrections (Markstein's theorem gives the correctly rounded quotient).
These tests run that division beside IEEE x / y on the device through
astrosim_selfcheck_division and require every quotient to agree in every bit, for
the model's divisors, for per-cell tau_IP3 values as the parameter draw makes them,
and for random divisors; half of the dividends put the quotient next to a rounding
midpoint, where a faithful-but-not-rounded quotient would show.
"""
import numpy as np
import pytest

import astrosimgpu_cuda_b200 as asg

pytestmark = pytest.mark.gpu

# C_m, tau_w, Delta_T of both populations and ratio_ER_cyt (src/astrosim_fused.cu:742-781)
MODEL_DIVISORS = [130.0, 104.0, 450.0, 264.0, 2.0, 0.185]


def test_model_constants_divide_exactly():
    assert asg.selfcheck_division(MODEL_DIVISORS, samples=1 << 24, seed=11) == 0


def test_cell_tau_ip3_divide_exactly():
    # tau_IP3 is drawn per astrocyte around 1058.76 within [0.9, 1.05] of the mean
    rng = np.random.default_rng(5)
    taus = 1058.7589568400845 * rng.uniform(0.9, 1.05, size=4096)
    assert asg.selfcheck_division(taus, samples=1 << 14, seed=12) == 0


def test_random_divisors_divide_exactly():
    rng = np.random.default_rng(6)
    ys = np.exp(rng.uniform(-20, 20, size=1024)) * rng.choice([-1.0, 1.0], size=1024)
    assert asg.selfcheck_division(ys, samples=1 << 14, seed=13) == 0


def test_selfcheck_rejects_bad_divisors():
    with pytest.raises(asg.AstrosimError):
        asg.selfcheck_division([1.0, 0.0])
