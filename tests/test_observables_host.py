"""Host post-processing of device observables (CPU only)."""
import numpy as np
import pytest

from energy_level_b200 import observables as ob


def test_normalize_pauli_strings_forms_and_errors():
    out = ob.normalize_pauli_strings([[[0, "x"], [2, "σy"]], {"label": "zz", "terms": [[1, "Z"], [3, "sigmaz"]]}], 4)
    assert out == [{"label": "x@0 y@2", "terms": [(0, "x"), (2, "y")]},
                   {"label": "zz", "terms": [(1, "z"), (3, "z")]}]
    assert ob.normalize_pauli_strings(None) is None
    assert ob.normalize_pauli_strings([]) == []
    for bad in ([[[0, "x"], [0, "y"]]], [[[5, "x"]]], [[[0, "w"]]], [[]], "x", [[[True, "x"]]], [{"label": "a"}]):
        with pytest.raises(ValueError):
            ob.normalize_pauli_strings(bad, 4)


def test_loop_observables():
    xy = np.zeros((3, 3), complex)
    xy[0, 1] = np.exp(0.3j)
    xy[1, 2] = np.exp(0.4j)
    xy[2, 0] = np.exp(0.5j)
    ph, wd = ob.loop_observables(xy, [[0, 1, 2]])
    assert abs(ph[0] - 1.2) < 1e-12 and abs(wd[0] - 1.2 / (2 * np.pi)) < 1e-12
    ph, _ = ob.loop_observables(xy, [[0, 2, 1]])
    assert np.isnan(ph[0])                 # xy[0, 2] = 0: missing edge
    with pytest.raises(ValueError):
        ob.loop_observables(xy, [[0]])
    assert ob.loop_observables(xy, None) == ([], [])


def test_link_loop_observables_orientation():
    link = np.array([[np.exp(0.3j), np.exp(0.4j), np.exp(-0.5j)]])
    ph, wd = ob.link_loop_observables(link, [(0, 1), (1, 2), (0, 2)], [[0, 1, 2]])
    # edge 2 -> 0 is the conjugate of the stored 0 -> 2 link
    assert abs(ph[0, 0] - 1.2) < 1e-12
    ph, _ = ob.link_loop_observables(link, [(0, 1), (1, 2)], [[0, 1, 2]])
    assert np.isnan(ph[0, 0])
    e = ob.link_loop_observables(link, [(0, 1)], None)
    assert e[0].shape == (0, 0)


def test_entropy_from_schmidt_and_labels():
    assert ob.entropy_from_schmidt([1.0], False) == 0.0
    s = ob.entropy_from_schmidt([np.sqrt(0.5), np.sqrt(0.5)], False)
    assert abs(s - np.log(2)) < 1e-14
    assert abs(ob.entropy_from_schmidt([2.0, 2.0], True) - np.log(2)) < 1e-14
    assert ob.entropy_from_schmidt([0.0], True) is None
    assert ob.product_label(3, 5) == "|rgr>" and ob.product_label(0, 0) == "|>"
