"""The autotuner's bookkeeping on CPU: shape buckets, cache keys, and the
JSON cache round trip (a tuned choice is reused without re-timing)."""
import json

import autotune


def test_buckets_and_keys():
    assert [autotune._bucket(v) for v in (1, 2, 3, 255, 256, 257)] == [1, 2, 4, 256, 256, 512]
    import torch

    t = autotune.Autotuner()
    k1 = t.key((256, 256, 256), 0, torch.float64)
    k2 = t.key((250, 200, 256), 0, torch.float64)
    k3 = t.key((256, 256, 256), 1, torch.float64)
    k4 = t.key((256, 256, 256), 0, torch.float32)
    assert k1 == k2 and len({k1, k3, k4}) == 3


def test_cache_round_trip(tmp_path):
    import torch

    path = tmp_path / "tune.json"
    t = autotune.Autotuner(cache_path=path)
    key = t.key((64, 64, 64), 2, torch.float32)
    entry = {"best": {"label": "tmem 3/4", "spec": "tmem=3,4", "algo": "thomas-pcr", "lanes": 2,
                      "variant": "v", "ms": 0.1}, "table": []}
    t.cache[key] = entry
    t.save()
    again = autotune.Autotuner(cache_path=path)
    assert json.loads(path.read_text())[key] == entry
    # a cached shape is answered without touching the GPU
    assert again.tune_solve((64, 64, 64), 2, torch.float32) == entry
