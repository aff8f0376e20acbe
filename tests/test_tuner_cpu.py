"""The launch-shape cache of the autotuner (no GPU): merging under a file
lock from several writers, and a missing or damaged file read as empty."""
import threading

from pyugks_b200 import tuner


def test_cache_merges_concurrent_writers(tmp_path):
    path = str(tmp_path / "shapes.json")
    assert tuner.load_cache(path) == {}

    def writer(k):
        for j in range(20):
            tuner.update_cache({"w%d_%d" % (k, j): (k + j) % 4 + 1}, path)

    threads = [threading.Thread(target=writer, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    cache = tuner.load_cache(path)
    assert len(cache) == 80
    assert cache["w3_5"] == (3 + 5) % 4 + 1


def test_damaged_cache_reads_empty(tmp_path):
    path = tmp_path / "shapes.json"
    path.write_text("{not json")
    assert tuner.load_cache(str(path)) == {}
    assert tuner.update_cache({"a": 1}, str(path)) == {"a": 1}
