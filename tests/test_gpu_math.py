"""The library's short transport-law evaluation T^0.7 against CUDA's pow."""
import numpy as np
import pytest

from compchan3dmpi_b200 import _lib

pytestmark = pytest.mark.gpu


def test_pow07_within_few_ulp_of_libm():
    L = _lib.load()
    rng = np.random.default_rng(0)
    T = np.concatenate([np.linspace(0.05, 8.0, 200001), rng.uniform(0.3, 3.0, 100000), [1.0, 0.5, 2.0, 1.4]])
    mine = np.empty_like(T)
    ref = np.empty_like(T)
    assert L.chan_selftest_pow07(_lib.dptr(T), _lib.dptr(mine), _lib.dptr(ref), T.size, 0) == 0
    ulp = np.abs(mine - ref) / np.spacing(np.abs(ref))
    assert ulp.max() <= 4.0, ulp.max()
    # and both agree with the host's correctly-rounded-ish pow
    host = T ** 0.7
    assert np.max(np.abs(mine - host) / host) < 1e-15
