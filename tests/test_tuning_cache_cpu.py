"""The autotuner cache (pt_tuning_cache_get / _put): a JSON file of batch tunings keyed by device and
workload class.  Round trips, replacement, files written by other JSON writers, malformed files
(reported, never overwritten), argument checks, concurrent writers in several processes, and a
bounded fuzz of the reader."""
import ctypes as C
import json
import multiprocessing as mp
import os

import numpy as np
import pytest

import polytope_b200 as pb


def make_class(device="NVIDIA B200", **kw):
    c = pb.TuningClass()
    c.device = device.encode() if isinstance(device, str) else device
    base = dict(sm_count=148, compute_capability=100, items_log2=8, pixels_log2=24, samples_log2=27, faces_log2=25,
                tree_depth=30, max_depth=6, flags=1)
    base.update(kw)
    for k, v in base.items():
        setattr(c, k, v)
    return c


def make_tuning(wave=1 << 25, tpb=256, stack=32, chunk=32, pipeline=pb.PIPELINE_WAVEFRONT):
    return pb.BatchTuning(wave, tpb, stack, chunk, pipeline)


def test_round_trip_replace_and_missing(tmp_path):
    path = tmp_path / "tune.json"
    a, b = make_class(), make_class(items_log2=5)
    assert pb.tuning_cache_get(path, a) is None  # no file yet: an empty cache
    pb.tuning_cache_put(path, a, make_tuning(), 12.5)
    pb.tuning_cache_put(path, b, make_tuning(wave=0, tpb=128, stack=0, chunk=64, pipeline=pb.PIPELINE_FUSED), 3.25)
    t, ms = pb.tuning_cache_get(path, a)
    assert t.as_dict() == make_tuning().as_dict() and ms == 12.5
    t, ms = pb.tuning_cache_get(path, b)
    assert (t.wave_pixels, t.threads_per_block, t.pipeline, ms) == (0, 128, pb.PIPELINE_FUSED, 3.25)
    assert pb.tuning_cache_get(path, make_class(samples_log2=28)) is None
    assert pb.tuning_cache_get(path, make_class(device="NVIDIA H100")) is None
    pb.tuning_cache_put(path, a, make_tuning(tpb=64), 0.1 + 0.2)  # replaces a's entry in place
    doc = json.loads(path.read_text())
    assert doc["format"] == "polytope_b200 tuning cache" and doc["version"] == 1
    assert len(doc["entries"]) == 2 and doc["entries"][0]["tuning"]["threads_per_block"] == 64
    t, ms = pb.tuning_cache_get(path, a)
    assert t.threads_per_block == 64 and ms == 0.1 + 0.2  # doubles survive the text form exactly
    assert not any(p.name.startswith("tune.json.tmp") for p in tmp_path.iterdir())


def test_device_names_with_quotes_and_utf8(tmp_path):
    path = tmp_path / "tune.json"
    names = ['GPU "quoted" \\ back', "Gerät Ä", "tab\there", "x" * 63]
    for k, n in enumerate(names):
        pb.tuning_cache_put(path, make_class(n), make_tuning(chunk=32 * (k + 1)), float(k))
    for k, n in enumerate(names):
        t, ms = pb.tuning_cache_get(path, make_class(n))
        assert t.queue_chunk == 32 * (k + 1) and ms == float(k)
    assert [e["class"]["device"] for e in json.loads(path.read_text())["entries"]] == names


def test_files_from_other_writers_are_read(tmp_path):
    """Any JSON writer's output of the same schema (other spacing, key order, escapes) reads back."""
    c = make_class()
    entry = {"ms": 7.0, "tuning": {"pipeline": 2, "queue_chunk": 128, "stack_depth": 48, "threads_per_block": 128,
                                   "wave_pixels": 4194304},
             "class": dict(sorted(make_class().as_dict().items()))}
    path = tmp_path / "tune.json"
    path.write_text(json.dumps({"entries": [entry], "version": 1, "format": "polytope_b200 tuning cache"},
                               indent=4, ensure_ascii=True))
    t, ms = pb.tuning_cache_get(path, c)
    assert (t.pipeline, t.queue_chunk, t.stack_depth, t.threads_per_block, t.wave_pixels, ms) == (2, 128, 48, 128, 4194304, 7.0)


BAD_FILES = [
    ("", "unexpected end"),
    ("{", "expected a key"),
    ('{"format": "something else", "version": 1, "entries": []}', "not a polytope_b200 tuning cache"),
    ('{"format": "polytope_b200 tuning cache", "version": 2, "entries": []}', "unsupported version"),
    ('{"format": "polytope_b200 tuning cache", "version": 1, "entries": {}}', "must be an array"),
    ('{"format": "polytope_b200 tuning cache", "version": 1, "entries": [1]}', "not an object"),
    ('{"format": "polytope_b200 tuning cache", "version": 1, "entries": []} x', "trailing"),
    ('[' * 40 + ']' * 40, "nesting too deep"),
    ('{"format": "polytope_b200 tuning cache\\ud800", "version": 1, "entries": []}', "unpaired surrogate"),
]


def bad_entry(**over):
    e = {"class": make_class().as_dict(), "tuning": make_tuning().as_dict(), "ms": 1.0}
    for k, v in over.items():
        part, _, field = k.partition("__")
        if field:
            e[part][field] = v
        else:
            e[part] = v
    return json.dumps({"format": "polytope_b200 tuning cache", "version": 1, "entries": [e]})


BAD_FILES += [
    (bad_entry(tuning__threads_per_block=100), "threads_per_block must be 64, 128 or 256"),
    (bad_entry(tuning__queue_chunk=48), "queue_chunk"),
    (bad_entry(tuning__pipeline=7), "unknown pipeline"),
    (bad_entry(tuning__stack_depth=65), "stack_depth"),
    (bad_entry(tuning__wave_pixels=-1), "wave_pixels"),
    (bad_entry(tuning__wave_pixels=1.5), "wave_pixels"),
    (bad_entry(class__sm_count=2 ** 32), "sm_count"),
    (bad_entry(class__device=""), "device"),
    (bad_entry(class__device="y" * 64), "device"),
    (bad_entry(class__flags="1"), "flags"),
    (bad_entry(ms=-1.0), "ms"),
    (bad_entry(ms="fast"), "ms"),
]


@pytest.mark.parametrize("text,why", BAD_FILES)
def test_malformed_files_are_reported_and_left_alone(tmp_path, text, why):
    path = tmp_path / "tune.json"
    path.write_text(text)
    with pytest.raises(pb.PolytopeError) as e:
        pb.tuning_cache_get(path, make_class())
    assert e.value.code == pb.PT_EINVAL and why in str(e.value), str(e.value)
    with pytest.raises(pb.PolytopeError) as e:
        pb.tuning_cache_put(path, make_class(), make_tuning(), 1.0)
    assert e.value.code == pb.PT_EINVAL and why in str(e.value)
    assert path.read_text() == text  # never overwritten


def test_put_argument_checks(tmp_path):
    path = tmp_path / "tune.json"
    for cls, tuning, ms, why in ((make_class(""), make_tuning(), 1.0, "device name"),
                                 (make_class(b"z" * 64), make_tuning(), 1.0, "device name"),
                                 (make_class(), make_tuning(tpb=32), 1.0, "threads_per_block"),
                                 (make_class(), make_tuning(chunk=8192), 1.0, "queue_chunk"),
                                 (make_class(), make_tuning(), float("nan"), "ms must be"),
                                 (make_class(), make_tuning(), -2.0, "ms must be")):
        with pytest.raises(pb.PolytopeError) as e:
            pb.tuning_cache_put(path, cls, tuning, ms)
        assert e.value.code == pb.PT_EINVAL and why in str(e.value)
    assert not path.exists()
    t, ms, found = pb.BatchTuning(), C.c_double(), C.c_int()
    assert pb.lib.pt_tuning_cache_get(None, C.byref(make_class()), C.byref(t), C.byref(ms), C.byref(found)) == pb.PT_EINVAL
    assert pb.lib.pt_tuning_cache_put(b"", C.byref(make_class()), C.byref(t), 1.0) == pb.PT_EINVAL
    assert pb.lib.pt_tuning_class_of(None, 0, C.byref(make_class())) == pb.PT_EINVAL
    assert pb.lib.pt_batch_autotune_cached(None, 0, os.fsencode(path), C.byref(t), None, None) == pb.PT_EINVAL
    with pytest.raises(pb.PolytopeError):
        pb.tuning_cache_get(tmp_path, make_class())  # a directory is not a cache file


def _writer(path, worker, count):
    import polytope_b200 as pbw
    for k in range(count):
        c = make_class(items_log2=worker, pixels_log2=k)
        pbw.tuning_cache_put(path, c, make_tuning(chunk=32 * (1 + k % 8)), worker + k / 100)


def test_concurrent_writers_keep_every_entry(tmp_path):
    path = str(tmp_path / "tune.json")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_writer, args=(path, w, 25)) for w in range(4)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    entries = json.loads(open(path).read())["entries"]
    assert len(entries) == 100
    for w in range(4):
        for k in range(25):
            t, ms = pb.tuning_cache_get(path, make_class(items_log2=w, pixels_log2=k))
            assert t.queue_chunk == 32 * (1 + k % 8) and ms == w + k / 100


def test_reader_survives_mutated_files(tmp_path):
    """Bounded fuzz: byte-level mutations of a valid cache either read back or fail with PT_EINVAL."""
    path = tmp_path / "tune.json"
    for k in range(3):
        pb.tuning_cache_put(path, make_class(items_log2=k, device=f"dev{k} \"q\""), make_tuning(), k + 0.5)
    good = path.read_bytes()
    rng = np.random.default_rng(5)
    ok = bad = 0
    for _ in range(400):
        b = bytearray(good)
        for _ in range(int(rng.integers(1, 4))):
            op, pos = int(rng.integers(3)), int(rng.integers(len(b)))
            if op == 0:
                b[pos] = int(rng.integers(256))
            elif op == 1:
                del b[pos:pos + int(rng.integers(1, 8))]
            else:
                b[pos:pos] = bytes(rng.choice(list(b'{}[]",:\\u0e-9 '), int(rng.integers(1, 4))))
        path.write_bytes(bytes(b))
        try:
            pb.tuning_cache_get(path, make_class(items_log2=1, device='dev1 "q"'))
            ok += 1
        except pb.PolytopeError as e:
            assert e.code == pb.PT_EINVAL
            bad += 1
    assert ok > 0 and bad > 0
