"""Host-side tests of the continuous-batching server with fake device pieces:
admission against the memory budget, FIFO completion, overlap of in-flight
batches, rejection, and failure of a launch -- no GPU, no device fault."""
import threading
import time

import numpy as np
import pytest

from gamma_smc_cu_b200 import serve


class NumpyArena(serve.PinnedArena):
    """The arena's allocator over ordinary host memory."""

    def __init__(self, nbytes):
        self.size = int(nbytes)
        self._buf = np.zeros(max(self.size, 1), np.uint8)
        self.base = self._buf.ctypes.data
        self._free = [(0, self.size)]
        self._lock = threading.Lock()
        self.in_use = 0


class FakeCtx:
    n_haps = 20
    n_sites = 500
    device_id = 0


class FakeExecutor:
    def __init__(self, ctx, **cfg):
        self.cfg = cfg

    def close(self):
        pass


class FakeEvent:
    def __init__(self, delay):
        self.t = time.perf_counter() + delay

    def query(self):
        return time.perf_counter() >= self.t

    def synchronize(self):
        while not self.query():
            time.sleep(1e-4)


class _Host:
    def __init__(self, a):
        self.a = a

    def numpy(self):
        return self.a


class Recorder:
    inflight = 0
    max_inflight = 0
    overlaps = 0
    launches = 0
    max_bytes = 0
    fail_tag = None
    fail_results_tag = None
    delay = 0.01
    lock = threading.Lock()


def make_batch_cls(rec, server_ref):
    class FakeBatch:
        repaired = 0

        def __init__(self, layout, device):
            self.layout = layout
            self.done = None

        def results(self, redo=None):
            for j in self.layout.jobs:
                if (rec.fail_results_tag is not None and j.pairs.size
                        and j.pairs[0, 0] == rec.fail_results_tag):
                    raise RuntimeError("injected collection failure")
            return self.layout.results(self.h_out)

        def launch(self, executor, stream, host=None):
            for j in self.layout.jobs:
                if rec.fail_tag is not None and j.pairs.size and j.pairs[0, 0] == rec.fail_tag:
                    raise RuntimeError("injected launch failure")
            out = host
            for j, offs in zip(self.layout.jobs, self.layout.out_off):
                for o in offs:
                    if o >= 0:
                        # value = site index + 1000 * first pair's i
                        v = (np.arange(j.site_begin, j.site_end)[:, None]
                             + 1000.0 * (j.pairs[0, 0] if j.n_pairs else 0))
                        out[o:o + j.rows * j.n_pairs] = np.broadcast_to(
                            v, (j.rows, j.n_pairs)).ravel()
            self.h_out = out
            with rec.lock:
                busy = sum(1 for s in server_ref[0].slots if s.batch is not None)
                rec.overlaps += busy > 0
                rec.launches += 1
                rec.max_bytes = max(rec.max_bytes, server_ref[0]._in_use)
            self.done = FakeEvent(rec.delay)
            return self.done
    return FakeBatch


@pytest.fixture
def server_factory(monkeypatch):
    made = []

    def make(**kw):
        rec = Recorder()
        ref = [None]
        monkeypatch.setattr(serve, "Executor", FakeExecutor)
        monkeypatch.setattr(serve, "DeviceBatch", make_batch_cls(rec, ref))
        monkeypatch.setattr(serve, "_new_stream", lambda d: object())
        monkeypatch.setattr(serve, "_free_device_bytes", lambda d: 1 << 30)
        monkeypatch.setattr(serve, "_bind_thread", lambda d: None)
        monkeypatch.setattr(serve, "_new_arena", NumpyArena)
        monkeypatch.setattr(serve, "_prewarm", lambda *a: None)
        monkeypatch.setattr(serve, "_pinned_floats", lambda n: np.zeros(max(n, 1), np.float32))
        positions = np.arange(500, dtype=np.float64) * 10.0
        s = serve.TmrcaServer(FakeCtx(), positions=positions, **kw)
        ref[0] = s
        made.append(s)
        return s, rec

    yield make
    for s in made:
        s.close()


def _check_result(fut, i, s0, s1, n_pairs, keys):
    r = fut.result(timeout=10)
    assert set(r) == set(keys)
    for k in keys:
        assert r[k].shape == (s1 - s0, n_pairs)
        assert np.array_equal(r[k][:, 0], np.arange(s0, s1) + 1000.0 * i)


def test_results_and_overlapping_batches(server_factory):
    s, rec = server_factory(max_inflight=3)
    futs = []
    rng = np.random.default_rng(0)
    lock = threading.Lock()

    def client(seed):
        r = np.random.default_rng(seed)
        for _ in range(15):
            i = int(r.integers(1, 20))
            s0 = int(r.integers(0, 400))
            s1 = s0 + int(r.integers(1, 100))
            f = s.submit([(i, 0), (i, 1)], s0, s1, mean_only=bool(r.integers(0, 2)))
            with lock:
                futs.append((f, i, s0, s1))
            time.sleep(float(r.uniform(0, 0.004)))

    ts = [threading.Thread(target=client, args=(k,)) for k in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for f, i, s0, s1 in futs:
        r = f.result(timeout=10)
        for k, v in r.items():
            assert v.shape == (s1 - s0, 2)
            assert np.array_equal(v[:, 0], np.arange(s0, s1) + 1000.0 * i)
    st = s.stats()
    assert st["completed"] == 60 and st["admitted"] == 60
    assert st["p99_ms"] >= st["p50_ms"] > 0
    assert rec.overlaps > 0          # batches launched while others were in flight
    assert s._in_use == 0


def test_memory_budget_and_rejection(server_factory):
    # each mean-only query over 100 sites x 5 pairs needs 2,000 bytes
    s, rec = server_factory(max_inflight=3, hbm_budget=5000)
    rec.delay = 0.02
    futs = [s.submit([(i, 0) for i in range(1, 6)], 0, 100) for _ in range(12)]
    too_big = s.submit([(i, 0) for i in range(1, 6)], 0, 400)  # 8,000 bytes
    for f in futs:
        assert f.result(timeout=10)["mean"].shape == (100, 5)
    with pytest.raises(MemoryError):
        too_big.result(timeout=10)
    assert rec.max_bytes <= 5000
    st = s.stats()
    assert st["rejected"] == 1 and st["completed"] == 12
    assert s._in_use == 0


def test_launch_failure_fails_only_its_batch(server_factory):
    s, rec = server_factory(max_inflight=1)
    rec.fail_tag = 13
    ok1 = s.submit([(3, 0)], 0, 10)
    ok1.result(timeout=10)
    bad = s.submit([(13, 0)], 0, 10)
    with pytest.raises(RuntimeError, match="injected"):
        bad.result(timeout=10)
    rec.fail_tag = None
    ok2 = s.submit([(4, 0)], 5, 15)
    _check_result(ok2, 4, 5, 15, 1, ["mean"])
    assert s._in_use == 0 and s.stats()["failed"] == 1


def test_submit_validation_and_regions(server_factory):
    s, rec = server_factory()
    with pytest.raises(ValueError, match="out of range"):
        s.submit([(1, 0)], 0, 501)
    with pytest.raises(ValueError, match="pair index"):
        s.submit([(20, 0)], 0, 10)
    assert s.sites_of(100.0, 205.0) == (10, 21)
    f = s.submit([(2, 1)], region_bp=(100.0, 205.0), mean_only=False, return_posterior=True)
    _check_result(f, 2, 10, 21, 1, ["mean", "lower", "upper", "posterior_alpha",
                                    "posterior_beta"])
    s.close()
    with pytest.raises(RuntimeError, match="closed"):
        s.submit([(1, 0)], 0, 5)


def test_arena_views_return_memory_when_dropped():
    import gc
    a = NumpyArena(4096)
    v1 = a.alloc(1000)           # 1024 bytes
    v2 = a.alloc(2000)           # 2048 bytes
    assert v1.dtype == np.float32 and v1.size == 256 and v2.size == 512
    assert a.alloc(2048) is None and a.in_use == 3072
    part = v1[10:20].reshape(2, 5)   # a view keeps the region alive
    v1[:] = 1.0
    del v1
    gc.collect()
    assert a.in_use == 3072 and part.sum() == 10.0
    del part, v2
    gc.collect()
    assert a.in_use == 0 and a._free == [(0, 4096)]
    assert a.alloc(4096).size == 1024


def test_results_outlive_arena_pressure(server_factory):
    """Callers that keep results do not stall the server: batches that no
    longer fit the arena get their own pinned buffer."""
    s, rec = server_factory(max_inflight=2, pinned_bytes=8192)
    kept = [s.submit([(i, 0), (i, 1)], 0, 400) for i in range(1, 8)]   # 3.2 kB each
    res = [f.result(timeout=10) for f in kept]
    for i, r in enumerate(res, start=1):
        assert np.array_equal(r["mean"][:, 1], np.arange(400) + 1000.0 * i)
    assert s.stats()["outside_arena"] >= 1


def test_batches_fit_the_arena_when_results_are_dropped(server_factory):
    """A burst larger than the arena is split into batches that each fit its
    largest free block; with results dropped as they complete nothing is
    allocated outside the arena."""
    s, rec = server_factory(max_inflight=2, pinned_bytes=16384)
    ok, done = [], threading.Event()
    n = 24

    def check(i):
        def cb(f):
            r = f.result()
            ok.append(bool(np.array_equal(r["mean"][:, 1], np.arange(400) + 1000.0 * i)))
            if len(ok) == n:
                done.set()
        return cb

    for i in range(1, n + 1):
        s.submit([(i % 20, 0), (i % 20, 1)], 0, 400).add_done_callback(check(i % 20))
    assert done.wait(timeout=20)
    assert all(ok)
    st = s.stats()
    assert st.get("outside_arena", 0) == 0
    assert rec.launches >= n * 3200 // 16384


def test_collection_failure_fails_only_its_batch(server_factory):
    """A batch whose results cannot be collected (e.g. a failed whole-window
    redo) fails its own queries; the server keeps serving."""
    s, rec = server_factory(max_inflight=1)
    rec.fail_results_tag = 17
    bad = s.submit([(17, 0)], 0, 50)
    with pytest.raises(RuntimeError, match="injected collection"):
        bad.result(timeout=10)
    rec.fail_results_tag = None
    _check_result(s.submit([(3, 1)], 10, 60), 3, 10, 60, 1, ("mean",))
    st = s.stats()
    assert st["failed"] >= 1 and st["completed"] >= 1


def test_tail_diagnostics(server_factory):
    """The server reports why queries waited (no free executor, HBM budget),
    its longest scheduler stalls and the collector's pauses while serving."""
    import gc
    s, rec = server_factory(max_inflight=1, hbm_budget=4 * 500 * 20)
    rec.delay = 0.02
    futs = [s.submit([(1, 0)], 0, 500)]
    time.sleep(0.005)   # the first query's batch is on the (only) executor now
    futs += [s.submit([(1 + (i % 19), 0)], 0, 500) for i in range(5)]
    for f in futs:
        f.result(timeout=10)
    gc.collect()   # a collection while the server runs is recorded (>= 1 ms only)
    st = s.stats()
    assert st["wait_executor"] > 0            # one executor: the others queued behind it
    assert isinstance(st["loop_stalls_ms"], list) and isinstance(st["gc_pauses"], int)
    assert st["gc_max_ms"] >= 0.0
    s2, _ = server_factory(max_inflight=2, hbm_budget=6000)   # room for one query
    fa = [s2.submit([(1, 0), (2, 0)], 0, 500) for _ in range(3)]
    for f in fa:
        f.result(timeout=10)
    assert s2.stats()["wait_hbm"] > 0
