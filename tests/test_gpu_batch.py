"""GPU tests of the batched runner: every instance of a batch gets exactly
the labels and iteration count of a single-instance run (bit-exact integer
work), whatever the launch configuration, loop mode or memory placement."""
import numpy as np
import pytest

from eggsync import EggError, data, egg_sync, egg_sync_batch
from make_golden import small_cases

pytestmark = pytest.mark.gpu


def mixed_instances():
    """Uneven sizes, dimensions 1-5 and several eps per dataset."""
    inst = []
    for name, (X, eps) in sorted(small_cases().items()):
        inst.append((X, eps))
    c1 = data.c1(0)["X"]
    for eps in (0.03, 0.05, 0.08):
        inst.append((c1, eps))
    for k, c in enumerate(data.c4(7, instances=6)):
        X = c["X"][:20000]
        for eps in c["eps"][::3]:
            inst.append((np.ascontiguousarray(X), eps))
    return inst


INST = mixed_instances()


@pytest.fixture(scope="module")
def singles():
    return [egg_sync(X, eps) for X, eps in INST]


def check_same(res, singles):
    assert len(res) == len(singles)
    for k, ((lab, info), (slab, sinfo)) in enumerate(zip(res, singles)):
        assert info["iterations"] == sinfo["iterations"], k
        assert info["converged"] == sinfo["converged"], k
        assert info["n_clusters"] == sinfo["n_clusters"], k
        assert np.array_equal(lab, slab), k


def test_batch_equals_single_runs(singles):
    res, binfo = egg_sync_batch(INST, tune="off")
    check_same(res, singles)
    assert binfo["groups"] == len({X.shape[1] for X, _ in INST})
    assert binfo["loop_iterations"] == max(s[1]["iterations"] for s in singles)


def test_autotuned_configurations_agree(singles):
    res, binfo = egg_sync_batch(INST, tune="again")
    assert binfo["tuned"] == 1
    check_same(res, singles)
    # cached: the second call does not tune again and gives the same bits
    res2, binfo2 = egg_sync_batch(INST)
    assert binfo2["tuned"] == 0
    assert (binfo2["update_threads"], binfo2["blocks_per_sm"], binfo2["order"]) == \
        (binfo["update_threads"], binfo["blocks_per_sm"], binfo["order"])
    check_same(res2, singles)


def test_host_loop_equals_graph(singles):
    res, _ = egg_sync_batch(INST, tune="off", loop="host")
    check_same(res, singles)


def test_device_inputs_and_outputs(singles, gpu):
    import torch

    dev = [(torch.from_numpy(X).to(gpu) if k % 2 == 0 else X, eps) for k, (X, eps) in enumerate(INST)]
    outs = [torch.empty(len(X), dtype=torch.int32, device=gpu) if k % 3 == 0 else np.empty(len(X), np.int32)
            for k, (X, _) in enumerate(INST)]
    res, _ = egg_sync_batch(dev, tune="off", labels_out=outs)
    res = [(lab.cpu().numpy() if hasattr(lab, "cpu") else lab, info) for lab, info in res]
    check_same(res, singles)


def test_max_iter_and_full_update(singles):
    res, _ = egg_sync_batch(INST, tune="off", max_iter=3)
    for (lab, info), X in zip(res, INST):
        ref, rinfo = egg_sync(X[0], X[1], max_iter=3)
        assert info["iterations"] == rinfo["iterations"] <= 3
        assert np.array_equal(lab, ref)
    res, _ = egg_sync_batch(INST, tune="off", full_update=True)
    check_same(res, singles)


def test_non_finite_instance_is_reported_alone(singles):
    bad = INST[0][0].copy()
    bad[5, 0] = np.inf
    inst = [INST[1], (bad, INST[0][1]), INST[2]]
    with pytest.raises(EggError) as e:
        egg_sync_batch(inst, tune="off")
    assert e.value.status == -3 and "instance 1" in str(e.value)


def test_single_instance_batch(singles):
    res, binfo = egg_sync_batch(INST[:1], tune="off")
    check_same(res, singles[:1])
    assert binfo["groups"] == 1
