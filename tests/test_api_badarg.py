"""CPU tests: descriptor validation and train/infer preconditions of the mirrored
API (cpp/oneapi/dal/algo/kmeans/test/badarg.cpp:113-224); all of them fail
before any device work."""
import numpy as np
import pytest

from onedal_b200 import kmeans

DTYPES = [np.float32, np.float64]
X = np.arange(20, dtype=np.float64).reshape(10, 2)


@pytest.mark.parametrize("dt", DTYPES)
def test_descriptor_defaults(dt):
    d = kmeans.descriptor(dt)
    assert d.get_cluster_count() == 2
    assert d.get_max_iteration_count() == 100
    assert d.get_accuracy_threshold() == 0.0
    assert not d.get_result_options()


@pytest.mark.parametrize("dt", DTYPES)
def test_cluster_count_checks(dt):
    d = kmeans.descriptor(dt)
    d.set_cluster_count(1)
    with pytest.raises(kmeans.domain_error):
        d.set_cluster_count(-1)
    with pytest.raises(kmeans.domain_error):
        d.set_cluster_count(0)
    with pytest.raises(kmeans.domain_error):
        d.set_cluster_count(2**31)


@pytest.mark.parametrize("dt", DTYPES)
def test_iteration_and_threshold_checks(dt):
    d = kmeans.descriptor(dt)
    d.set_max_iteration_count(1).set_max_iteration_count(0)
    with pytest.raises(kmeans.domain_error):
        d.set_max_iteration_count(-1)
    d.set_accuracy_threshold(0.01).set_accuracy_threshold(0.0)
    with pytest.raises(kmeans.domain_error):
        d.set_accuracy_threshold(-0.1)
    with pytest.raises(kmeans.domain_error):
        d.set_result_options(kmeans.result_option_id())


@pytest.mark.parametrize("dt", DTYPES)
def test_train_preconditions(dt):
    d = kmeans.descriptor(dt).set_cluster_count(2)
    with pytest.raises(kmeans.domain_error):
        kmeans.train(d, np.empty((0, 2)), np.zeros((2, 2)))
    with pytest.raises(kmeans.invalid_argument):  # init rows != cluster count
        kmeans.train(kmeans.descriptor(dt).set_cluster_count(3), X, np.zeros((2, 2)))
    with pytest.raises(kmeans.invalid_argument):  # init columns != data columns
        kmeans.train(d, X, np.zeros((2, 3)))
    with pytest.raises(kmeans.invalid_argument):  # k > rows
        kmeans.train(kmeans.descriptor(dt).set_cluster_count(11), X, np.zeros((11, 2)))


@pytest.mark.parametrize("dt", DTYPES)
def test_infer_preconditions(dt):
    d = kmeans.descriptor(dt).set_cluster_count(2)
    m = kmeans.model(np.zeros((2, 2)))
    with pytest.raises(kmeans.domain_error):
        kmeans.infer(d, m, np.empty((0, 2)))
    with pytest.raises(kmeans.domain_error):
        kmeans.infer(d, kmeans.model(), X)
    with pytest.raises(kmeans.invalid_argument):
        kmeans.infer(kmeans.descriptor(dt).set_cluster_count(3), m, X)
    with pytest.raises(kmeans.invalid_argument):
        kmeans.infer(d, kmeans.model(np.zeros((2, 3))), X)


def test_objective_getter_guard():
    r = kmeans.infer_result(kmeans.result_option_id())
    with pytest.raises(kmeans.domain_error):
        r.get_objective_function_value()
    r2 = kmeans.infer_result(kmeans.result_options.compute_exact_objective_function)
    r2._set_objective(1.0)
    assert r2.get_objective_function_value() == 1.0
    with pytest.raises(kmeans.domain_error):
        r2._set_objective(-1.0)
