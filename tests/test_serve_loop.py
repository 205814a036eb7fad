"""Host logic of the serving loop, on a fake serving handle (no GPU): FIFO
admission by capacity, advance in fixed chunks, latency
bookkeeping, and the one-at-a-time queue model."""
import numpy as np

from awsemmd_b200 import serve


class FakeServer:
    """Residue capacity only; a request finishes after `nsteps` + 1 advance
    steps (its setup evaluation, then nsteps steps), like the real handle."""

    def __init__(self, capacity: int):
        self.capacity = capacity
        self.used = 0
        self.step = 0
        self.slots = {}
        self.next = 0
        self.admitted = []
        self.advances = []

    def admit(self, chain, nsteps, t_start, t_stop, seed):
        n = int(chain["n_res"])
        if self.used + n > self.capacity:
            return None
        self.used += n
        s = self.next
        self.next += 1
        self.slots[s] = [self.step + 1, self.step + 1 + nsteps, n]
        self.admitted.append(chain["rid"])
        return s

    def progress(self, s):
        b, e, _ = self.slots[s]
        return max(0, min(self.step, e) - b), e - b

    def advance(self, k):
        self.advances.append(k)
        self.step += k

    def collect(self, s):
        b, e, n = self.slots.pop(s)
        assert self.step >= e
        self.used -= n
        return np.zeros((3 * n, 3)), None, np.zeros(21)


def make(rid, arrival, n, nsteps):
    return serve.Request(rid, arrival, {"n_res": n, "rid": rid}, nsteps)


def test_fifo_admission_and_completion():
    fake = FakeServer(capacity=100)
    reqs = [make(0, 0.0, 60, 10), make(1, 0.0, 60, 5), make(2, 0.0, 30, 3)]
    t = [0.0]
    done = serve.run_stream(fake, reqs, chunk=4, clock=lambda: t[0], sleep=lambda s: None)
    # request 1 does not fit next to request 0; request 2 (which would fit)
    # waits behind it: first come first served
    assert fake.admitted == [0, 1, 2]
    # 1 and 2 then run side by side; the shorter one finishes first
    assert [d.rid for d in done] == [0, 2, 1]
    # fixed chunks: request 0 (setup evaluation + 10 steps) finishes inside
    # the third chunk and is collected at its end; 2 and 1 likewise
    assert fake.advances == [4, 4, 4, 4, 4]
    assert all(d.finished >= d.admitted >= d.arrival for d in done)


def test_stats_and_fifo_model():
    arrivals = np.array([0.0, 0.1, 0.2, 5.0])
    service = np.array([1.0, 1.0, 1.0, 1.0])
    lat = serve.fifo_latencies(arrivals, service)
    np.testing.assert_allclose(lat, [1.0, 1.9, 2.8, 1.0])
    done = [serve.Completed(k, a, a, a + l, 10, 100) for k, (a, l) in enumerate(zip(arrivals, lat))]
    st = serve.stream_stats(done)
    assert st["requests"] == 4 and abs(st["p50_s"] - np.percentile(lat, 50)) < 1e-12
    assert abs(st["residue_steps"] - 4000) < 1e-9


def test_stream_generators():
    rng = np.random.default_rng(4)
    a = serve.poisson_arrivals(2000, 50.0, rng)
    assert np.all(np.diff(a) > 0) and abs(a[-1] / 2000 - 1 / 50) < 0.003
    L = serve.log_uniform_lengths(5000, 30, 1000, rng)
    assert L.min() >= 30 and L.max() <= 1000
    assert abs(np.median(L) - np.sqrt(30 * 1000)) < 25  # log-uniform: median is the geometric mean


class PreparingServer(FakeServer):
    """A fake handle that also prepares requests on the host (as AwsemServer):
    the loop must prepare each request once, admit the prepared object in
    arrival order and free every prepared object."""

    class Prepared:
        def __init__(self, chain, seed, log):
            self.chain, self.seed, self.freed = chain, seed, False
            log.append(self)

        def free(self):
            self.freed = True

    def __init__(self, capacity):
        super().__init__(capacity)
        self.prepared = []

    def prepare(self, chain, seed=1):
        return PreparingServer.Prepared(chain, seed, self.prepared)

    def admit(self, what, nsteps, t_start, t_stop, seed):
        assert isinstance(what, PreparingServer.Prepared) and what.seed == seed and not what.freed
        return super().admit(what.chain, nsteps, t_start, t_stop, seed)


def test_prepared_admission_keeps_fifo_and_frees():
    fake = PreparingServer(capacity=100)
    reqs = [make(0, 0.0, 60, 10), make(1, 0.0, 60, 5), make(2, 0.0, 30, 3)]
    for k, r in enumerate(reqs):
        r.seed = 40 + k
    t = [0.0]
    done = serve.run_stream(fake, reqs, chunk=4, clock=lambda: t[0], sleep=lambda s: None)
    assert fake.admitted == [0, 1, 2]
    assert sorted(d.rid for d in done) == [0, 1, 2]
    assert len(fake.prepared) == 3 and all(p.freed for p in fake.prepared)


def test_request_that_never_fits_is_refused():
    import pytest

    fake = FakeServer(capacity=50)
    with pytest.raises(ValueError, match="does not fit"):
        serve.run_stream(fake, [make(0, 0.0, 60, 10)], chunk=4, clock=lambda: 0.0, sleep=lambda s: None)
