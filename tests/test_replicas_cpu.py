"""Per-device replicas of the filter facade (filter.hpp:98-101,128-152,
205-218), without a GPU: the replica logic runs against a fake device copy.

* a replica is made once per device, on first use, also when many threads
  ask for it at once (the reference's lock + second check);
* the home device never copies;
* an insert drops the replicas (they would be stale);
* a probe instance probes the replica of the keys' device -- not the
  original words, which is what the reference's operator() does
  (filter.hpp:234-240).
"""
import contextlib
import importlib
import threading
import time

import numpy as np

F = importlib.import_module("dtlg.filter")   # the module (dtlg.filter is also the facade class)


def test_replica_made_once_per_device_on_first_use():
    copies = []

    def copy(words, dev):
        copies.append(dev)
        time.sleep(0.02)   # a slow copy: concurrent first users must wait, not copy again
        return words + 100 * dev

    home = np.arange(8, dtype=np.uint64)
    r = F.DeviceReplicas(home, 0, copy)
    assert r.get(0) is home and copies == []
    got = [None] * 16

    def user(i):
        got[i] = r.get(3)

    th = [threading.Thread(target=user, args=(i,)) for i in range(16)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert copies == [3]
    assert all(g is got[0] for g in got)
    assert np.array_equal(got[0], home + 300)
    r.get(1)
    r.get(1)
    assert copies == [3, 1] and r.devices() == [0, 1, 3]
    r.invalidate()
    assert r.devices() == [0]
    r.get(3)
    assert copies == [3, 1, 3]


class _FakeInstance:
    def __init__(self):
        self.seen = []

    def batch_contains_host(self, data, keys, match_pos, match_offset):
        self.seen.append(int(data[0]))
        return 0


class _FakeFilter:
    def __init__(self):
        self.filter_instance = _FakeInstance()
        self.replicas = F.DeviceReplicas(np.zeros(4, dtype=np.uint64), 0, lambda w, d: w + d)

    def filter_data_on(self, device):
        return self.replicas.get(device)


def test_probe_instance_uses_the_replica_of_the_keys_device(monkeypatch):
    import torch
    monkeypatch.setattr(torch.cuda, "device", lambda d: contextlib.nullcontext())
    f = _FakeFilter()
    p = F.probe_t(f)
    keys = np.arange(10, dtype=np.uint32)
    for dev in (2, 0, 5, 2):
        monkeypatch.setattr(F.probe_t, "device_of", lambda self, k, d=dev: d)
        p(keys, np.zeros(10, dtype=np.uint32), 0)
    # each call probed the words of its own device; devices 2 and 5 were copied once
    assert f.filter_instance.seen == [2, 0, 5, 2]
    assert f.replicas.devices() == [0, 2, 5]
