"""Failure paths, each made to happen without a GPU fault, trap or hang.

* A bounded device wait that runs out: awsem_set_wait_limits(hold) makes the
  conditions of one kind of wait unreachable (a fragment-memory copy stage expects bytes
  that never arrive; a grid barrier of the persistent step form one block
  more than the grid), so every wait gives up after its limit, the kernels
  end normally and the call reports AWSEM_ESTATE.
* A residue pair list that outgrows its capacity.
* Non-finite coordinates.

After each, the next call runs clean and gives the results of a handle that
never failed, bit for bit.  The reference stops the run on such errors
(error->all, e.g. src/fix_backbone.cpp:2938); here the handle survives.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHORT = 2_000_000  # SM clock cycles: about a millisecond


def c0_files(tmp_path):
    from awsemmd_b200 import synth

    return synth.write_system(synth.config_system(0), str(tmp_path / "c0"))


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_fragment_memory_wait_runs_out_then_next_call_is_clean(prec, tmp_path, gpu_lib):
    from awsemmd_b200.engine import AwsemError, AwsemSystem

    files = c0_files(tmp_path)
    with AwsemSystem(files, precision=prec) as s:
        x, _ = s.get_state()
        f0, e0 = s.compute(x)
        s.set_wait_limits(fm_cycles=SHORT, hold=1)
        with pytest.raises(AwsemError, match="fragment-memory stream"):
            s.compute(x)
        s.set_wait_limits()
        f1, e1 = s.compute(x)
    np.testing.assert_array_equal(f1, f0)
    np.testing.assert_array_equal(e1, e0)


def test_grid_barrier_wait_runs_out_then_next_call_is_clean(tmp_path, gpu_lib):
    from awsemmd_b200.engine import AwsemError, AwsemSystem

    files = c0_files(tmp_path)
    kw = dict(dt=2.0, langevin=False, thermo=True)
    with AwsemSystem(files, precision="mixed") as ref:
        ref.set_step_form("persistent")
        x0, v0 = ref.get_state()
        rows_ref = ref.run(10, **kw)
        x_ref, v_ref = ref.get_state()
    with AwsemSystem(files, precision="mixed") as s:
        s.set_step_form("persistent")
        s.set_wait_limits(barrier_cycles=SHORT, hold=2)
        with pytest.raises(AwsemError, match="grid barrier"):
            s.run(3, **kw)
        s.set_wait_limits()
        s.set_state(x0, v0)
        rows = s.run(10, **kw)
        x, v = s.get_state()
    np.testing.assert_array_equal(rows, rows_ref)
    np.testing.assert_array_equal(x, x_ref)
    np.testing.assert_array_equal(v, v_ref)


def test_pair_list_overflow(tmp_path, gpu_lib):
    """Configuration 1 (2,000 residues) squeezed to a fifth of its size needs
    some twenty times the pair-list room of its starting structure.
    awsem_compute grows the list and evaluates again; awsem_run reports the
    overflow (AWSEM_ESTATE), grows the list, and its next call runs clean."""
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemError, AwsemSystem

    files = synth.write_system(synth.config_system(1), str(tmp_path / "c1"))
    with AwsemSystem(files, precision="mixed") as s:
        x0, v0 = s.get_state()
        squeezed = x0.mean(axis=0) + 0.2 * (x0 - x0.mean(axis=0))
        f_ref, e_ref = s.compute(x0)
        f, e = s.compute(squeezed)  # grows the list and evaluates again
        assert np.isfinite(f).all() and np.isfinite(e).all()
        assert s.neighbor_stats()["overflow"] == 0
        with AwsemSystem(files, precision="mixed") as other:
            # another handle: the sums do not depend on the list's capacity or order
            other.compute(squeezed)
            fb, eb = other.compute(squeezed)
        np.testing.assert_array_equal(f, fb)
        np.testing.assert_array_equal(e, eb)
    with AwsemSystem(files, precision="mixed") as s:
        s.set_state(squeezed, v0)
        with pytest.raises(AwsemError, match="overflow"):
            s.run(1, dt=0.1, langevin=False)
        s.set_state(x0, v0)
        s.run(2, dt=2.0, langevin=False)
        f2, e2 = s.compute(x0)
    np.testing.assert_array_equal(f2, f_ref)
    np.testing.assert_array_equal(e2, e_ref)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_non_finite_coordinates(prec, tmp_path, gpu_lib):
    from awsemmd_b200.engine import AwsemError, AwsemSystem

    files = c0_files(tmp_path)
    with AwsemSystem(files, precision=prec) as s:
        x, _ = s.get_state()
        f0, e0 = s.compute(x)
        bad = x.copy()
        bad[37, 1] = np.nan
        with pytest.raises(AwsemError, match="non-finite"):
            s.compute(bad)
        bad[37, 1] = np.inf
        with pytest.raises(AwsemError, match="non-finite"):
            s.compute(bad)
        f1, e1 = s.compute(x)
    np.testing.assert_array_equal(f1, f0)
    np.testing.assert_array_equal(e1, e0)
