"""The library's tuning table on CPU: shape-class keys, the file round trip
(what a tuned process leaves for the next one, or for PENTA_TUNING_CACHE),
validation, and a cached shape answered without touching a GPU."""
import subprocess
import sys
from pathlib import Path

import pytest

import autotune
import pentadsolver as ps

REPO = Path(__file__).resolve().parents[1]
GPU = "NVIDIA B200"


@pytest.fixture(autouse=True)
def _empty_table():
    ps.tuning_clear()
    yield
    ps.tuning_clear()


def test_buckets_and_keys():
    assert [autotune._bucket(v) for v in (1, 2, 3, 255, 256, 257)] == [1, 2, 4, 256, 256, 512]
    k1 = ps.tuning_key([256, 256, 256], 0, 8, gpu_name=GPU)
    k2 = ps.tuning_key([250, 200, 256], 0, 8, gpu_name=GPU)   # same buckets
    k3 = ps.tuning_key([256, 256, 256], 1, 8, gpu_name=GPU)
    k4 = ps.tuning_key([256, 256, 256], 0, 4, gpu_name=GPU)
    k5 = ps.tuning_key([256, 256, 256], 2, 8, gpu_name=GPU)
    assert k1 == f"{GPU}|solve|f64|x|n256|l65536" and k1 == k2
    assert k3 == k5 == f"{GPU}|solve|f64|yz|n256|l65536"   # y and z share a class
    assert len({k1, k3, k4}) == 3
    assert ps.tuning_key([33, 17, 9], 1, 4, "plan", GPU) == f"{GPU}|plan|f32|yz|n32|l512"
    with pytest.raises(ps.PentadError):
        ps.tuning_key([256, 256, 256], 0, 8, "bogus", GPU)
    with pytest.raises(ps.PentadError):
        ps.tuning_key([4, 8, 8], 0, 8, gpu_name=GPU)   # the shape rules apply


def test_table_file_round_trip(tmp_path):
    k = ps.tuning_key([64, 64, 64], 2, 4, gpu_name=GPU)
    ps.tuning_set(k, "tmem=3,4", "thomas-pcr", 2, 0, 0.125)
    kp = ps.tuning_key([64, 64, 64], 0, 8, "plan", GPU)
    ps.tuning_set(kp, ctas=111, ms=1.5)
    path = tmp_path / "tune.tsv"
    ps.tuning_save(path)
    text = path.read_text()
    assert f"{k}\ttmem=3,4\tthomas-pcr\t2\t0\t0.125" in text
    assert f"{kp}\tauto\tauto\t0\t111\t1.5" in text
    ps.tuning_clear()
    assert ps.tuning_lookup(k) is None
    ps.tuning_load(path)
    assert ps.tuning_lookup(k) == {"spec": "tmem=3,4", "algo": "thomas-pcr", "lanes": 2,
                                   "ctas": 0, "ms": 0.125}
    assert ps.tuning_lookup(kp)["ctas"] == 111


def test_malformed_lines_are_skipped(tmp_path):
    good = f"{GPU}|solve|f64|x|n64|l4096"
    path = tmp_path / "t.tsv"
    path.write_text("# comment\n"
                    f"{good}\tno-tmem\tthomas-pcr\t2\t0\t0.5\n"
                    "too\tfew\tfields\n"
                    f"{GPU}|solve|f64|x|n8|l8\tauto\tauto\tnotanint\t0\t1\n"
                    f"{GPU}|solve|f64|x|n16|l8\tauto\tauto\t64\t0\t1\n")
    ps.tuning_load(path)
    assert ps.tuning_lookup(good)["spec"] == "no-tmem"
    assert ps.tuning_lookup(f"{GPU}|solve|f64|x|n8|l8") is None
    assert ps.tuning_lookup(f"{GPU}|solve|f64|x|n16|l8") is None   # lanes out of range
    with pytest.raises(ps.PentadError):
        ps.tuning_load(tmp_path / "missing.tsv")


def test_tuning_set_validates():
    for spec, algo, lanes in (("bogus", "auto", 0), ("auto", "bogus", 0), ("auto", "auto", 33)):
        with pytest.raises(ps.PentadError):
            ps.tuning_set("k", spec, algo, lanes)


def test_cached_shape_is_answered_without_a_gpu(tmp_path):
    import torch

    path = tmp_path / "tune.tsv"
    t = autotune.Autotuner(cache_path=path)
    key = t.key((64, 64, 64), 2, torch.float32)
    ps.tuning_set(key, "tmem=3,4", "thomas-pcr", 2, 0, 0.1)
    t.save()
    ps.tuning_clear()
    again = autotune.Autotuner(cache_path=path)
    assert again.tune_solve((64, 64, 64), 2, torch.float32) == {
        "best": {"spec": "tmem=3,4", "algo": "thomas-pcr", "lanes": 2, "ctas": 0, "ms": 0.1},
        "table": []}


def test_environment_file_is_read_at_first_use(tmp_path):
    # a fresh process with PENTA_TUNING_CACHE set sees the file's entries
    path = tmp_path / "env.tsv"
    key = f"{GPU}|solve|f64|yz|n128|l16384"
    path.write_text(f"{key}\tno-tmem\tthomas-pcr\t2\t0\t0.25\n")
    code = ("import sys; sys.path[:0] = [%r, %r]; import pentadsolver as ps; "
            "print(ps.tuning_lookup(%r))" % (str(REPO / "pentadiagonal-solver_b200"),
                                             str(REPO), key))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         env={"PENTA_TUNING_CACHE": str(path), "PATH": "/usr/bin:/bin"},
                         timeout=120)
    assert out.returncode == 0, out.stderr
    assert "'spec': 'no-tmem'" in out.stdout and "'ms': 0.25" in out.stdout
