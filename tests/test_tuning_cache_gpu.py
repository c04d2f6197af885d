"""The cached batch autotuner on the device: the first call searches and stores the winner under
the batch's class, the second returns it from the file without timing runs, and a batch built
with it renders every film bit-identical to pt_render."""
import pytest

from conftest import assert_bit_equal
import polytope_b200 as pb
from test_batch_serve_gpu import small_jobs, solo

pytestmark = pytest.mark.gpu


def test_autotune_cached_stores_then_reuses(cuda_device, tmp_path):
    jobs = small_jobs(4, seed=31)
    path = tmp_path / "tune.json"
    best, ms, hit = pb.autotune_cached(jobs, path)
    assert not hit and ms > 0
    cls = pb.tuning_class(jobs)
    d = cls.as_dict()
    assert d["device"] and d["sm_count"] > 0 and d["compute_capability"] >= 100 and d["items_log2"] == 2
    t, stored_ms = pb.tuning_cache_get(path, cls)
    assert t.as_dict() == best.as_dict() and stored_ms == ms
    best2, ms2, hit2 = pb.autotune_cached(jobs, path)
    assert hit2 and best2.as_dict() == best.as_dict() and ms2 == ms
    b = pb.Batch(jobs, best2)
    b.run()
    for i, (scene, rd) in enumerate(jobs):
        assert_bit_equal(b.output(i)[0], solo(scene, rd)[0], f"film {i}")
    b.close()
