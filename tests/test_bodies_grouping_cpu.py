"""Host logic of the batching across bodies: the band plan of solve_bodies
and the batch-size tuner's cache (no GPU)."""
import json

from capytaine_b200.engine import band_batches
from capytaine_b200.tuning import BatchTuner


def test_band_batches_cover_every_pair_once_within_the_band():
    sizes = [384, 3072, 2560, 640, 2944, 384, 1024, 896]
    nq = 3
    plan = band_batches(sizes, nq, 1.3, lambda top: 64 if top <= 1024 else 8)
    seen = sorted(p for _, pairs in plan for p in pairs)
    assert seen == sorted((i, q) for i in range(len(sizes)) for q in range(nq))
    for top, pairs in plan:
        assert all(sizes[i] <= top and sizes[i] * 1.3 >= top for i, _ in pairs)
        assert len(pairs) <= (64 if top <= 1024 else 8)
        assert top == max(sizes[i] for i, _ in pairs)
    # largest first, and one body's frequencies stay together in a batch
    assert plan[0][0] == 3072
    for _, pairs in plan:
        bodies = [i for i, _ in pairs]
        assert bodies == sorted(bodies, key=lambda i: (-sizes[i], i))


def test_band_batches_split_by_capacity():
    plan = band_batches([512] * 5, 4, 1.3, lambda top: 6)
    assert [len(p) for _, p in plan] == [6, 6, 6, 2]


def test_tuner_cache_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "tuner.json"
    path.write_text(json.dumps({"dev/mixed/1024": 32}))
    t = BatchTuner(cache_path=str(path), measure=False, default=16)
    monkeypatch.setattr(BatchTuner, "_key", lambda self, engine, cls: f"dev/mixed/{cls}")

    class Eng:
        precision = "mixed"
    monkeypatch.setattr("capytaine_b200.engine._Factors.estimate_bytes",
                        staticmethod(lambda n, b, p, lu=True: b * 16 * n * n))
    assert BatchTuner.size_class(900) == 1024 and BatchTuner.size_class(100) == 512
    assert t.batch_for(Eng(), 900, 1e12) == 32          # from the file
    assert t.batch_for(Eng(), 2000, 1e12) == 16         # not measured: the default, then written
    assert json.loads(path.read_text())["dev/mixed/2048"] == 16
    assert t.batch_for(Eng(), 900, 16 * 900 * 900 * 3) == 3  # capped by memory
