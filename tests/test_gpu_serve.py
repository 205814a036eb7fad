"""Serving handle on the GPU: a request's result is the same alone and in the
mix (bit for bit: forces are exact fixed-point sums, the noise is keyed by
the request's own step count), equals the plain batch run of the same
system, and admission answers busy when the handle is full."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ff(tmp_path_factory):
    from awsemmd_b200 import synth

    return synth.forcefield_dir(str(tmp_path_factory.mktemp("ff")))


def chains():
    from awsemmd_b200 import synth

    return {name: synth.chain_arrays(L, seed=7000 + k, n_mem_per_window=4)
            for k, (name, L) in enumerate([("A", 61), ("B", 45), ("C", 90)])}


def serve_until_done(srv, slots):
    out = {}
    while slots:
        left = min(t - d for d, t in (srv.progress(s) for s in slots.values()))
        srv.advance(max(1, min(25, left)))
        for name, s in list(slots.items()):
            d, t = srv.progress(s)
            if d >= t:
                out[name] = srv.collect(s)
                del slots[name]
    return out


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_request_alone_equals_request_in_the_mix(prec, ff, gpu_lib):
    from awsemmd_b200.engine import AwsemBatch, AwsemServer

    c = chains()
    nsteps, ramp = 120, (600.0, 300.0)
    with AwsemServer(ff, max_residues=512, max_requests=8, max_memory_records=200000, precision=prec) as srv:
        s = srv.admit(c["A"], nsteps, *ramp, seed=11)
        alone = serve_until_done(srv, {"A": s})["A"]
    with AwsemServer(ff, max_residues=512, max_requests=8, max_memory_records=200000, precision=prec) as srv:
        slots = {"B": srv.admit(c["B"], 200, 300.0, 300.0, seed=12)}
        srv.advance(17)
        slots["A"] = srv.admit(c["A"], nsteps, *ramp, seed=11)
        srv.advance(9)
        slots["C"] = srv.admit(c["C"], 60, 450.0, 350.0, seed=13)
        mixed = serve_until_done(srv, slots)
        assert srv.usage()["requests"] == 0
    x0, v0, e0 = alone
    x1, v1, e1 = mixed["A"]
    assert np.array_equal(x0, x1) and np.array_equal(v0, v1)
    np.testing.assert_allclose(e1, e0, rtol=1e-12, atol=1e-9)
    assert not np.array_equal(x0, c["A"]["x"].reshape(-1, 3))
    # the same run through the plain batch path
    with AwsemBatch.from_arrays(ff, [c["A"]], precision=prec, seeds=[11]) as b:
        b.run(nsteps, t_start=ramp[0], t_stop=ramp[1])
        xb, vb = b.get_state(0)
    assert np.array_equal(x0, xb) and np.array_equal(v0, vb)


def test_admission_is_bounded_by_capacity(ff, gpu_lib):
    from awsemmd_b200.engine import AwsemServer

    c = chains()
    with AwsemServer(ff, max_residues=96, max_requests=4, max_memory_records=200000) as srv:
        a = srv.admit(c["A"], 10)  # 61 residues: two 32-residue groups
        assert a is not None
        assert srv.admit(c["B"], 10) is None  # 45 more residues need two more groups
        u = srv.usage()
        assert u["requests"] == 1 and u["residues"] == 64 and u["residue_capacity"] == 96
        assert u["device_bytes"] > 0
        serve_until_done(srv, {"A": a})
        b = srv.admit(c["B"], 10)
        assert b is not None
        serve_until_done(srv, {"B": b})
    with AwsemServer(ff, max_residues=512, max_requests=1, max_memory_records=200000) as srv:
        assert srv.admit(c["A"], 5) is not None
        assert srv.admit(c["B"], 5) is None  # request slots


def test_stream_serves_every_request(ff, gpu_lib):
    from awsemmd_b200 import serve, synth
    from awsemmd_b200.engine import AwsemServer

    rng = np.random.default_rng(3)
    lens = serve.log_uniform_lengths(12, 30, 150, rng)
    arr = serve.poisson_arrivals(12, 200.0, rng)
    reqs = [serve.Request(k, float(arr[k]), synth.chain_arrays(int(L), seed=8000 + k, n_mem_per_window=2), 80,
                          600.0, 300.0, seed=100 + k) for k, L in enumerate(lens)]
    with AwsemServer(ff, max_residues=640, max_requests=6, max_memory_records=400000) as srv:
        done = serve.run_stream(srv, reqs, chunk=25)
    assert sorted(d.rid for d in done) == list(range(12))
    for d in done:
        assert np.all(np.isfinite(d.x)) and np.isfinite(d.energies).all()
    st = serve.stream_stats(done)
    assert st["p99_s"] >= st["p50_s"] > 0


def test_prepared_admission_equals_direct_admission(ff, gpu_lib):
    """awsem_server_prepare + awsem_server_admit_prepared place the same
    request as awsem_server_admit, bit for bit; a request prepared for one
    handle is refused by another; a request that does not fit now stays
    valid and is admitted later."""
    from awsemmd_b200.engine import AwsemError, AwsemServer

    c = chains()
    kw = dict(max_residues=512, max_requests=8, max_memory_records=200000)
    with AwsemServer(ff, **kw) as srv:
        a = srv.admit(c["C"], 70, 500.0, 300.0, seed=21)
        direct = serve_until_done(srv, {"C": a})["C"]
    with AwsemServer(ff, **kw) as srv, AwsemServer(ff, **kw) as other:
        p = srv.prepare(c["C"], seed=21)
        with pytest.raises(AwsemError, match="not prepared for this handle"):
            other.admit(p, 70, 500.0, 300.0)
        a = srv.admit(p, 70, 500.0, 300.0)
        p.free()
        prepared = serve_until_done(srv, {"C": a})["C"]
    for u, w in zip(direct, prepared):
        assert np.array_equal(u, w)
    with AwsemServer(ff, max_residues=96, max_requests=4, max_memory_records=200000) as srv:
        a = srv.admit(c["A"], 10)  # 61 residues: two of three 32-residue groups
        p = srv.prepare(c["B"], seed=3)  # 45 residues: two more groups
        assert srv.admit(p, 10) is None
        serve_until_done(srv, {"A": a})
        b = srv.admit(p, 10)
        assert b is not None
        p.free()
        serve_until_done(srv, {"B": b})
