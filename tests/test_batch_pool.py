"""The batch layer's pool of idle contexts (host logic, no GPU): a finished
solve's context is kept for the next solve on the same device, a failed
one is closed, the pool holds at most its cap, and release_contexts()
closes what it holds."""

import prtlb_gpu.batch as B


class FakeContext(object):
    made = 0

    def __init__(self, device=0):
        FakeContext.made += 1
        self.device = device
        self.handle = object()
        self.closed = False
        self.ended = 0

    def close(self):
        self.closed = True
        self.handle = None


class FakeLib(object):
    def prt_adr_end(self, handle):
        for c in FakeLib.live:
            if c.handle is handle:
                c.ended += 1
        return 0


def _setup(monkeypatch, cap=3):
    FakeContext.made = 0
    FakeLib.live = []
    monkeypatch.setattr(B._lib, "Context", FakeContext)
    monkeypatch.setattr(B._lib, "lib", lambda: FakeLib())
    monkeypatch.setattr(B, "_POOL_CAP", cap)
    monkeypatch.setattr(B, "_pool", {})


def test_finished_contexts_are_reused_per_device(monkeypatch):
    _setup(monkeypatch)
    a = B._take_context(0)
    b = B._take_context(1)
    FakeLib.live += [a, b]
    assert FakeContext.made == 2
    B._return_context(a, 0)
    B._return_context(b, 1)
    assert not a.closed and a.ended == 1  # its transport state was ended, not freed
    assert B._take_context(0) is a  # same device: reused
    assert B._take_context(1) is b
    assert FakeContext.made == 2
    c = B._take_context(0)  # the pool is empty again: a new one
    assert c is not a and FakeContext.made == 3


def test_failed_contexts_are_closed_and_the_cap_holds(monkeypatch):
    _setup(monkeypatch, cap=2)
    bad = B._take_context(0)
    bad.broken = True
    FakeLib.live.append(bad)
    B._return_context(bad, 0)
    assert bad.closed and B._pool.get(0, []) == []
    ctxs = [B._take_context(0) for _ in range(4)]
    FakeLib.live += ctxs
    for c in ctxs:
        B._return_context(c, 0)
    assert len(B._pool[0]) == 2
    assert [c.closed for c in ctxs] == [False, False, True, True]
    B.release_contexts()
    assert all(c.closed for c in ctxs) and B._pool == {}
    # a context closed elsewhere is not kept
    d = B._take_context(0)
    d.close()
    B._return_context(d, 0)
    assert B._pool.get(0, []) == []
