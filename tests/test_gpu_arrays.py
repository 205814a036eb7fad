"""Replicas described by arrays against the same chain given as files."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


# force tolerance (relative to the largest force) and per-term energy tolerance
@pytest.mark.parametrize("prec,tol,etol", [("fp64", 1e-9, 1e-6), ("mixed", 1e-4, 1e-5)])
def test_array_replica_matches_file_replica_and_oracle(prec, tol, etol, tmp_path, gpu_lib, oracle_built):
    import ref
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemBatch

    c = synth.chain_arrays(64, seed=3003, n_mem_per_window=4)
    files = synth.write_chain_arrays(c, str(tmp_path / "as_files"))
    ff = synth.forcefield_dir(str(tmp_path / "ff"))
    o = ref.OracleSystem(files)
    with AwsemBatch.from_arrays(ff, [c], precision=prec) as b:
        b.run(0, langevin=False)
        f, e = b.forces(0), b.energies(0)
        x, _ = b.get_state(0)
    np.testing.assert_array_equal(x, c["x"].reshape(-1, 3))
    fo, eo = o.compute(x)
    assert np.abs(f - fo).max() / np.abs(fo).max() < tol
    for k in range(20):
        assert abs(e[k] - eo[k]) <= etol * max(abs(eo[k]), 1e-2), (k, e[k], eo[k])
