"""GPU tests of the brute-force drop-in (GPU_DynamicalClustering): the same
labels and iteration counts as the reference's own GPU code
(simple_GPU_SynC.cu, fixtures made by tests/golden/make_golden.py
--gpu-simple), the first update within 1e-5 of the FP64 oracle, and the same
iteration count as the reference's CPU SynC."""
import numpy as np
import pytest

from conftest import load_golden
from eggsync import GPU_DynamicalClustering, simple_sync
from make_golden import checksum, simple_cases
from oracle import RefSync, ari

pytestmark = pytest.mark.gpu


def cases():
    return [(name, X, eps) for name, (X, eps) in sorted(simple_cases().items())]


@pytest.mark.parametrize("name,X,eps", cases())
def test_matches_reference_gpu_code(name, X, eps):
    G = load_golden("ref_simple_%s.npz" % name)
    assert checksum(X) == G["x_checksum"]
    lab, info = simple_sync(X, eps)
    for k in range(len(G["labels"])):
        assert np.array_equal(lab, G["labels"][k])
        assert info["iterations"] == int(G["iterations"][k])


@pytest.fixture(scope="module")
def ref():
    try:
        return RefSync()
    except FileNotFoundError:
        pytest.skip("reference CPU SynC not built")


@pytest.mark.parametrize("name,X,eps", cases())
def test_iterations_match_reference_cpu_sync(ref, name, X, eps):
    """Same update and stop rule as the CPU SynC; its labelling differs
    (synCluster_v2 assigns greedily, SynC.cpp:88-118; the GPU code takes the
    smallest index in each eps-ball), so the partitions agree up to the few
    points whose eps-balls overlap two groups."""
    lab, info = simple_sync(X, eps)
    rlab, rit = ref.run(X, eps)
    assert info["iterations"] == rit
    assert ari(lab, rlab) > 0.9999


def test_first_update_matches_oracle(oracle):
    """One iteration equals the FP64 brute-force update within 1e-5."""
    for name, X, eps in cases():
        P = np.empty_like(X)
        lab, info = simple_sync(X, eps, max_iter=1, positions_out=P)
        assert info["iterations"] == 1
        idx = np.arange(0, len(X), 7).astype(np.int32)
        xs, cnt = oracle.update_sample(X, eps, idx)
        assert np.abs(P[idx] - xs).max() <= 1e-5, name
        # the first iteration's order parameter is that of the input
        assert abs(info["r_local"] - oracle.order_parameter(X, eps)) <= 1e-5, name


def test_wrapper_shapes_and_device_input(gpu):
    import torch

    X, eps = cases()[0][1], cases()[0][2]
    C, itr, stages, space = GPU_DynamicalClustering(torch.from_numpy(X), eps)
    lab, info = simple_sync(torch.from_numpy(X).to(gpu), eps)
    assert C.shape == (len(X),) and itr.shape == (info["iterations"],) and stages.shape == (6,)
    assert np.array_equal(C.numpy().astype(np.int32), lab)
