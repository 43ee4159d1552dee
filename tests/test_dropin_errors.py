"""f2py argument conventions of the drop-in, checked on the host (no GPU)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def cim():
    from imaged11_b200 import cImageD11
    return cImageD11


def test_inout_ubi_must_be_contiguous_f64(cim):
    gv = np.zeros((4, 3))
    with pytest.raises(ValueError, match="not contiguous"):
        cim.score_and_refine(np.asfortranarray(np.arange(9.).reshape(3, 3)), gv, 0.1)
    with pytest.raises(ValueError, match="elsize=8 but got 4"):
        cim.score_and_refine(np.eye(3, dtype=np.float32), gv, 0.1)


def test_inout_gv_of_compute_gv(cim):
    x = np.zeros((5, 3))
    om = np.zeros(5)
    with pytest.raises(ValueError, match="elsize=8 but got 4"):
        cim.compute_gv(x, om, 1., 0.3, 0., 0., [0, 0, 0], np.zeros((5, 3), np.float32))
    with pytest.raises(ValueError):
        cim.compute_gv(x, om, 1., 0.3, 0., 0., [0, 0, 0], np.zeros((4, 3)))


def test_inout_labels_dtype(cim):
    gv = np.zeros((4, 3))
    with pytest.raises(ValueError, match="elsize=4 but got 8"):
        cim.score_and_assign(np.eye(3), gv, 0.1, np.zeros(4), np.zeros(4, np.int64), 0)


def test_gv_shape(cim):
    with pytest.raises(ValueError, match="fixed to 3"):
        cim.score(np.eye(3), np.zeros((4, 2)), 0.1)


def test_omp_compat(cim):
    assert cim.OPENMP is False
    assert cim.cimaged11_omp_get_max_threads() == 0
    cim.cimaged11_omp_set_num_threads(4)
    assert cim.cores_available() >= 1
