"""Host logic of the drop-in's resident scene cache (no GPU: the device scene is a stand-in)."""
from __future__ import annotations

import threading

import pytest


class FakeScene:
    def __init__(self, arrays, device=0):
        self.arrays = arrays
        self.closed = False

    def close(self):
        assert not self.closed, "closed twice"
        self.closed = True


@pytest.fixture()
def cache(monkeypatch):
    from acoustic_agent_b200 import backend, runtime
    monkeypatch.setattr(runtime, "DeviceScene", FakeScene)
    return backend._SceneCache(limit=2)


def test_scenes_in_use_are_never_evicted(cache):
    arrays = [{"k": i} for i in range(4)]
    held = [cache.acquire(a, 0)[0] for a in arrays]          # four users, limit two
    assert not any(s.closed for s in held)
    assert len(cache.entries) == 4
    cache.release(held[0])
    cache.release(held[1])
    extra = {"k": 9}
    s, hit = cache.acquire(extra, 0)
    assert not hit
    # the two idle scenes go (least recent first) until the limit allows, the three in use stay
    assert held[0].closed and held[1].closed
    assert not any(x.closed for x in held[2:]) and not s.closed


def test_hits_reuse_the_resident_scene(cache):
    a = {"k": 1}
    s1, hit1 = cache.acquire(a, 0)
    s2, hit2 = cache.acquire(a, 0)
    assert (hit1, hit2) == (False, True) and s1 is s2
    cache.release(s1)
    cache.release(s2)
    for i in range(3):
        x, _ = cache.acquire({"k": 10 + i}, 0)
        cache.release(x)
    assert s1.closed


def test_concurrent_acquires_never_close_a_scene_in_use(cache):
    errors = []
    shared = [{"k": i} for i in range(6)]

    def worker(seed):
        import random
        rnd = random.Random(seed)
        for _ in range(300):
            s, _ = cache.acquire(rnd.choice(shared), 0)
            if s.closed:
                errors.append("a scene was closed while a user held it")
            cache.release(s)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors
    assert all(e[2] == 0 for e in cache.entries.values())
