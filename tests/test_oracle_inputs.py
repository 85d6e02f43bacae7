"""The benchmark's CPU arms rebuild their inputs without the product library
(oracle/inputs.py): the numpy R-MAT and uniform generators, the source
selection and the SSSP weights must equal the product's exactly, so the
reference arm traverses the very graph and sources the GPU arm does."""
import numpy as np
import pytest

import xbtrav
from oracle import inputs


@pytest.mark.parametrize("scale,ef,seed", [(1, 4, 3), (5, 2, 7), (10, 8, 11), (15, 16, 0x5EED)])
def test_rmat_equals_the_product_generator(scale, ef, seed):
    ro, ci = xbtrav.HostCSR.rmat(scale, ef, 0.57, 0.19, 0.19, seed=seed).arrays()
    ro2, ci2 = inputs.rmat_csr(scale, ef, seed=seed)
    np.testing.assert_array_equal(ro2, ro)
    np.testing.assert_array_equal(ci2, ci)


def test_rmat_other_probabilities():
    ro, ci = xbtrav.HostCSR.rmat(9, 8, 0.25, 0.25, 0.25, seed=5).arrays()
    ro2, ci2 = inputs.rmat_csr(9, 8, 0.25, 0.25, 0.25, seed=5)
    np.testing.assert_array_equal(ro2, ro)
    np.testing.assert_array_equal(ci2, ci)


@pytest.mark.parametrize("n,pairs,seed", [(7, 100, 2), (1000, 3000, 1), (335_000, 1_850_000, 0x5EED)])
def test_uniform_equals_the_product_generator(n, pairs, seed):
    ro, ci = xbtrav.HostCSR.er(n, pairs, seed=seed).arrays()
    ro2, ci2 = inputs.er_csr(n, pairs, seed=seed)
    np.testing.assert_array_equal(ro2, ro)
    np.testing.assert_array_equal(ci2, ci)


def test_sources_and_weights_equal_the_product():
    ro, ci = xbtrav.HostCSR.rmat(12, 16, seed=9).arrays()
    for seed, k in ((10, 1), (0x5EED + 1, 64), (3, 1000)):
        np.testing.assert_array_equal(inputs.select_sources(ro, seed, k), xbtrav.select_sources_csr(ro, seed, k))
    np.testing.assert_array_equal(inputs.symmetric_weights(ro, ci, 0x5EED, 1, 100),
                                  xbtrav.symmetric_weights(ro, ci, 0x5EED, 1, 100))
    with pytest.raises(ValueError):
        inputs.select_sources(np.array([0, 0, 0], np.int64), 1, 1)
