"""Admission policy of the serving loop (s2dw_b200/serving.py), host logic
only: slots are reused while idle, at most `slots_per_config` per
configuration, a new slot is admitted only within the HBM budget, and idle
slots of other configurations are evicted least recently used first (never a
busy slot, never one of the requesting configuration).  The slot class is
replaced by a stub of known size, so no GPU is needed."""
import pytest

from s2dw_b200 import serving


class _StubSlot:
    closed = []

    def __init__(self, key, tables, device, form="fp64", max_batch=32, batch_bytes=0, priority=None,
                 split_min_batch=1):
        self.key = key
        self.priority = priority
        self.split = form == "split"
        self.bytes = _StubSlot.estimate_bytes(*key, form, max_batch, batch_bytes)
        self.busy = False
        self.last_used = 0.0
        self.cap = 1

    @staticmethod
    def estimate_bytes(B, N, alpha, J, form="fp64", max_batch=32, batch_bytes=0):
        return 10 * B

    def close(self):
        _StubSlot.closed.append(self.key)


@pytest.fixture
def srv(monkeypatch):
    monkeypatch.setattr(serving, "Slot", _StubSlot)
    _StubSlot.closed = []
    s = serving.Server(hbm_budget_bytes=2500, slots_per_config=2)
    monkeypatch.setattr(s, "config_tables", lambda *k: None)
    return s


A, Bk, C = (100, 1, 2.0, 3), (100, 2, 2.0, 3), (50, 3, 2.0, 2)  # 1000, 1000, 500 bytes


def test_idle_slot_is_reused(srv):
    a1 = srv._acquire(A, 0.0)
    assert srv._acquire(A, 1.0) is a1 and srv.used == 1000


def test_slots_per_config_and_budget(srv):
    a1 = srv._acquire(A, 0.0)
    a1.busy = True
    a2 = srv._acquire(A, 0.0)
    assert a2 is not a1 and srv.used == 2000
    a2.busy = True
    assert srv._acquire(A, 0.0) is None            # two slots of A, both busy
    assert srv._acquire(Bk, 0.0) is None           # 3000 > 2500 and nothing idle to evict
    assert srv.used == 2000 and not _StubSlot.closed
    assert srv._acquire(C, 0.0) is not None        # 2500 fits exactly
    assert srv.used == 2500


def test_lru_eviction_of_idle_slots_of_other_configs(srv):
    a1 = srv._acquire(A, 0.0)
    a1.busy = True
    a2 = srv._acquire(A, 0.0)
    a1.busy, a1.last_used = False, 2.0
    a2.busy, a2.last_used = False, 1.0
    b1 = srv._acquire(Bk, 3.0)                     # evicts a2, the least recently used
    assert b1 is not None and _StubSlot.closed == [A]
    assert srv.slots[A] == [a1] and srv.used == 2000
    b1.busy = True
    b2 = srv._acquire(Bk, 4.0)                     # evicts a1; b1 is busy, and B's own slots are kept
    assert b2 is not None and _StubSlot.closed == [A, A] and srv.used == 2000
    assert srv.used <= srv.budget


def test_size_priority_orders_small_transforms_first(monkeypatch):
    """With priorities on, a slot's stream priority follows its band limit:
    smaller transforms get numerically lower (higher) CUDA priorities."""
    prios = [serving.size_priority(B) for B in (32, 64, 128, 256, 512, 1024, 2048)]
    assert prios == sorted(prios) and prios[0] < prios[-1] == 0
    monkeypatch.setattr(serving, "Slot", _StubSlot)
    s = serving.Server(hbm_budget_bytes=1 << 20, priorities=True)
    monkeypatch.setattr(s, "config_tables", lambda *k: None)
    small, big = s._acquire((64, 2, 2.0, 6), 0.0), s._acquire((1024, 2, 2.0, 10), 0.0)
    assert small.priority < big.priority == 0
    s2 = serving.Server(hbm_budget_bytes=1 << 20)
    monkeypatch.setattr(s2, "config_tables", lambda *k: None)
    assert s2._acquire((64, 2, 2.0, 6), 0.0).priority is None


def test_auto_form_picks_split_slots_only_for_large_batches(monkeypatch):
    """form="auto": a split slot when at least split_min_batch requests of one
    configuration and kind wait, an FP64 slot otherwise."""
    monkeypatch.setattr(serving, "Slot", _StubSlot)
    s = serving.Server(hbm_budget_bytes=1 << 20, form="auto", split_min_batch=3)
    monkeypatch.setattr(s, "config_tables", lambda *k: None)
    key = (64, 2, 2.0, 6)
    a = s._acquire(key, 0.0, "fp64")
    b = s._acquire(key, 0.0, "split")
    assert not a.split and b.split and a is not b
    b.busy = True
    assert s._acquire(key, 0.0, "split") is not b  # a second split slot (slots_per_config=2)
