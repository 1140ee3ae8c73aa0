"""Peano-Hilbert cell ordering (the reference's sort_local_data,
MPI/sort_local_data.cpp:17-55): the keys are a bijection onto the curve's
indices, consecutive keys are face neighbours of the integer grid, and the
permutation reorders arbitrary generator sets."""
import numpy as np
import pytest

from fvmhd3d_b200.ordering import hilbert_keys, sort_local_data


@pytest.mark.parametrize("bits", [1, 2, 3, 4, 5])
def test_keys_are_a_continuous_bijection(bits):
    n = 1 << bits
    g = np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3)
    k = hilbert_keys(g, bits)
    assert np.array_equal(np.sort(k), np.arange(n ** 3, dtype=np.uint64))
    walk = g[np.argsort(k)].astype(np.int64)
    step = np.abs(np.diff(walk, axis=0))
    assert np.all(step.sum(axis=1) == 1)          # one unit step along one axis
    assert np.array_equal(walk[0], [0, 0, 0])


def test_full_width_keys_fit_63_bits():
    top = (1 << 21) - 1
    g = np.array([[0, 0, 0], [top, top, top], [top, 0, 0], [0, top, 0], [0, 0, top]])
    k = hilbert_keys(g, 21)
    assert k.max() < (np.uint64(1) << np.uint64(63))
    assert len(set(k.tolist())) == len(k)


def test_sort_local_data_is_a_permutation_that_improves_locality():
    rng = np.random.default_rng(7)
    pos = rng.uniform(-1.5, 1.5, size=(20000, 3))
    order = sort_local_data(pos, 3.0)
    assert np.array_equal(np.sort(order), np.arange(pos.shape[0]))
    gap = lambda p: np.linalg.norm(np.diff(p, axis=0), axis=1).mean()
    assert gap(pos[order]) < 0.2 * gap(pos)


def test_sort_local_data_rejects_bad_shapes():
    with pytest.raises(ValueError):
        sort_local_data(np.zeros((4, 2)), 1.0)
    with pytest.raises(ValueError):
        hilbert_keys(np.zeros((4, 3), np.int64), 22)
