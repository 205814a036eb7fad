"""Persistent step kernel (one cooperative launch per MD step): trajectories,
energies and thermo rows must equal the per-pass kernel chain's bit for bit
(every sum is exact fixed point), for any persistent grid size and number of
fragment-memory stream warps, across pair-list rebuilds, on batch, single
system and serving handles."""
import numpy as np
import pytest

from conftest import write_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ff(tmp_path_factory):
    from awsemmd_b200 import synth

    return synth.forcefield_dir(str(tmp_path_factory.mktemp("ff")))


def chains():
    from awsemmd_b200 import synth

    return [synth.chain_arrays(L, seed=9100 + k, n_mem_per_window=4) for k, L in enumerate([64, 150, 41, 233, 97])]


def batch_run(ff, prec, form, nsteps=60, **shape):
    from awsemmd_b200.engine import AwsemBatch

    with AwsemBatch.from_arrays(ff, chains(), precision=prec, seeds=[5, 6, 7, 8, 9]) as b:
        if form == "persistent":
            b.set_step_form("persistent", **shape)
            assert b.step_form()["step_form"] == "persistent"
        rows = b.run(nsteps, t_start=500.0, t_stop=300.0, neigh_every=10, thermo=True)
        assert b.neighbor_stats()["overflow"] == 0
        # a second run continues from the first
        b.run(25, neigh_every=10)
        x, v = b.get_state_all()
        e = np.array([b.energies(r) for r in range(b.nreplicas)])
        return x, v, e, rows, b.neighbor_stats()["builds"]


@pytest.mark.parametrize("nsteps", [60, 37])
@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_persistent_step_equals_kernel_chain(prec, nsteps, ff, gpu_lib):
    x0, v0, e0, r0, nb0 = batch_run(ff, prec, "kernels", nsteps)
    assert nb0 >= 6  # rebuilds every 10 steps are inside both runs
    for shape in [dict(blocks=0, stream_warps=2), dict(blocks=3, stream_warps=1), dict(blocks=1, stream_warps=4),
                  dict(blocks=37, stream_warps=7)]:
        x1, v1, e1, r1, nb1 = batch_run(ff, prec, "persistent", nsteps, **shape)
        assert nb1 == nb0, shape
        assert np.array_equal(x0, x1) and np.array_equal(v0, v1), shape
        assert np.array_equal(e0, e1), shape
        assert np.array_equal(r0, r1), shape


def test_persistent_single_system_parity(tmp_path, gpu_lib):
    """FP64 single system in the persistent form: a run equals the kernel
    chain's, and the final forces still match the golden evaluation path."""
    from awsemmd_b200.engine import AwsemSystem

    files, _ = write_case("c0", tmp_path)
    out = {}
    for form in ["kernels", "persistent"]:
        with AwsemSystem(files, precision="fp64") as s:
            if form == "persistent":
                s.set_step_form("persistent")
            s.run(40, seed=3)
            x, v = s.get_state()
            out[form] = (x, v, s.energies())
    assert np.array_equal(out["kernels"][0], out["persistent"][0])
    assert np.array_equal(out["kernels"][1], out["persistent"][1])
    assert np.array_equal(out["kernels"][2], out["persistent"][2])


def test_persistent_serving_equals_kernel_chain(ff, gpu_lib):
    from awsemmd_b200.engine import AwsemServer

    c = chains()
    res = {}
    for form in ["kernels", "persistent"]:
        with AwsemServer(ff, max_residues=1024, max_requests=8, max_memory_records=400000) as srv:
            if form == "persistent":
                srv.set_step_form("persistent", stream_warps=3)
            a = srv.admit(c[1], 70, 600.0, 300.0, seed=21)
            srv.advance(13)
            b = srv.admit(c[3], 30, 400.0, 400.0, seed=22)
            srv.advance(31)
            srv.advance(40)
            res[form] = (srv.collect(a), srv.collect(b))
    for k in range(2):
        for m in range(3):
            assert np.array_equal(res["kernels"][k][m], res["persistent"][k][m]), (k, m)


def test_step_form_arguments(ff, gpu_lib):
    from awsemmd_b200.engine import AwsemBatch, AwsemError

    with AwsemBatch.from_arrays(ff, chains()[:2], precision="mixed") as b:
        for bad in [dict(blocks=-1), dict(stream_warps=0), dict(stream_warps=8)]:
            with pytest.raises(AwsemError):
                b.set_step_form("persistent", **bad)
        b.set_step_form("persistent", blocks=5, stream_warps=3)
        b.run(3)
        f = b.step_form()
        assert f["step_form"] == "persistent" and f["persistent_blocks"] == 5 and f["stream_warps"] == 3
        b.set_step_form("kernels")
        assert b.step_form()["step_form"] == "kernels"


def test_launch_shapes_do_not_change_results(ff, gpu_lib):
    """awsem_set_launch_shapes: any valid shapes give the same trajectory bit
    for bit; out-of-range shapes are refused."""
    from awsemmd_b200.engine import AwsemBatch, AwsemError

    out = []
    for shapes in [(1, 148, 148, 0), (3, 592, 37, 296), (2, 1, 1, 1)]:
        with AwsemBatch.from_arrays(ff, chains(), precision="mixed", seeds=[5, 6, 7, 8, 9]) as b:
            b.set_launch_shapes(shapes)
            b.run(30, t_start=500.0, t_stop=300.0, neigh_every=10)
            out.append(b.get_state_all())
    for x, v in out[1:]:
        assert np.array_equal(out[0][0], x) and np.array_equal(out[0][1], v)
    with AwsemBatch.from_arrays(ff, chains()[:1], precision="mixed") as b:
        for bad in [(0, 1, 1, 0), (1, 0, 1, 0), (1, 1, 0, 0), (1, 1, 1, -1), (99, 1, 1, 0)]:
            with pytest.raises(AwsemError):
                b.set_launch_shapes(bad)
