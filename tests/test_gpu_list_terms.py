"""Terms that read the fix's neighbour lists themselves ([AMH-Go]; the
solvent barrier and Debye-Hueckel on the CA pairs of the half list) on the
GPU beyond the single-system golden runs: the lists are kept per replica, so a
replica in a batch, a run cut into continuation calls, and the persistent step
form all follow the reference's list rebuilds exactly.  c0go: the 100-residue
chain with a compact native structure; c0x: the same chain with the three
pair terms; both run with neighbor 0.6 and neigh_modify delay 3 every 2 check
yes (the lists are rebuilt during the run and pairs cross their reach)."""
import numpy as np
import pytest

from conftest import neigh_of, write_case

pytestmark = pytest.mark.gpu


def _kw(g, seed=None):
    nsteps, dt, t0, t1, damp, gseed = g["run"]
    return int(nsteps), dict(dt=dt, langevin=True, t_start=t0, t_stop=t1, damp=damp,
                             seed=int(gseed if seed is None else seed), skin=neigh_of(g)[0])


@pytest.mark.parametrize("case", ["c0go", "c0x"])
def test_batch_replicas_keep_their_own_lists(case, tmp_path, gpu_lib):
    """Two replicas with different seeds rebuild at different steps: the
    one with the reference's seed reproduces the reference's trajectory, the
    other equals its single-system run bit for bit."""
    from awsemmd_b200.engine import AwsemBatch, AwsemSystem

    files, g = write_case(case, tmp_path)
    nsteps, kw = _kw(g)
    skin, delay, every, check = neigh_of(g)
    with AwsemSystem(files, precision="fp64") as s:
        s.set_neighbor(skin, delay, every, check)
        s.set_state(g["x0"], g["v0"])
        s.run(nsteps, **{**kw, "seed": 77})
        x_alone, v_alone = s.get_state()
    with AwsemBatch([files, files], precision="fp64", seeds=[kw["seed"], 77]) as b:
        b.set_neighbor(skin, delay, every, check)
        b.set_state(g["x0"], g["v0"], r=0)
        b.set_state(g["x0"], g["v0"], r=1)
        b.run(nsteps, **kw)
        x0, v0 = b.get_state(0)
        x1, v1 = b.get_state(1)
    assert np.abs(x0 - g["xN"]).max() < 1e-6 and np.abs(v0 - g["vN"]).max() < 1e-6
    assert np.array_equal(x1, x_alone) and np.array_equal(v1, v_alone)
    assert not np.array_equal(x0, x1)


@pytest.mark.parametrize("case", ["c0go", "c0x"])
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_continuation_calls_keep_the_list(case, prec, tmp_path, gpu_lib):
    """A run cut into continuation calls (awsem_run_window) is the run in one
    call: the list state carries over between the calls."""
    from awsemmd_b200.engine import AwsemSystem

    files, g = write_case(case, tmp_path)
    nsteps, kw = _kw(g)
    skin, delay, every, check = neigh_of(g)
    with AwsemSystem(files, precision=prec) as s:
        s.set_neighbor(skin, delay, every, check)
        s.set_state(g["x0"], g["v0"])
        rows_one = s.run(nsteps, thermo=True, **kw)
        x1, v1 = s.get_state()
    with AwsemSystem(files, precision=prec) as s:
        s.set_neighbor(skin, delay, every, check)
        s.set_state(g["x0"], g["v0"])
        r0 = s.run_window(0, (0, nsteps), False, thermo=True, **kw)
        r1 = s.run_window(7, (0, nsteps), True, thermo=True, **kw)
        r2 = s.run_window(nsteps - 7, (0, nsteps), True, thermo=True, **kw)
        x2, v2 = s.get_state()
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)
    assert np.array_equal(np.concatenate([r0, r1, r2]), rows_one)


@pytest.mark.parametrize("case", ["c0go", "c0x", "c0s", "c0v"])
def test_persistent_form_equals_kernel_chain(case, tmp_path, gpu_lib):
    """c0s, c0v: Shake, the membrane potential and vector fragment memory,
    whose pass the persistent kernel runs beside the pair passes."""
    from awsemmd_b200.engine import AwsemSystem

    files, g = write_case(case, tmp_path)
    nsteps, kw = _kw(g)
    out = {}
    for form in ["kernels", "persistent"]:
        with AwsemSystem(files, precision="fp64") as s:
            s.set_neighbor(*neigh_of(g))
            s.set_step_form(form)
            s.set_state(g["x0"], g["v0"])
            s.run(nsteps, **kw)
            out[form] = s.get_state() + (s.energies(),)
    for a, b in zip(out["kernels"], out["persistent"]):
        assert np.array_equal(a, b)
    assert np.abs(out["kernels"][0] - g["xN"]).max() < 1e-6


def test_neighbor_settings_are_checked(tmp_path, gpu_lib):
    from awsemmd_b200.engine import AwsemError, AwsemSystem

    files, g = write_case("r1r69go", tmp_path)
    with AwsemSystem(files, precision="fp64") as s:
        for bad in [(2.0, -1, 1, 1), (2.0, 0, 0, 1), (2.0, 0, 1, 2)]:
            with pytest.raises(AwsemError):
                s.set_neighbor(*bad)
