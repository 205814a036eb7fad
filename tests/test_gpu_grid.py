"""Pair lists of large replicas come from a cell grid (replicas above 2,048
residues); the forces and energies must be those of the oracle, before and
after motion (several grid rebuilds)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_grid_list_matches_oracle(tmp_path, gpu_lib, oracle_built):
    import ref
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemBatch, AwsemError

    c = synth.packed_arrays([250] * 9, 150.0, 77, n_mem_per_window=1)
    assert c["n_res"] > 2048
    ff = synth.forcefield_dir(str(tmp_path / "ff"))
    files = synth.write_chain_arrays(c, str(tmp_path / "sys"))
    o = ref.OracleSystem(files)
    x0 = c["x"].reshape(-1, 3)
    with AwsemBatch.from_arrays(ff, [c], precision="fp64", seeds=[3]) as b:
        # the persistent step kernel builds no cell grids: refused on such handles
        with pytest.raises(AwsemError):
            b.set_step_form("persistent")
        for stage in range(2):
            x, _ = b.get_state(0)
            f, e = b.compute(x, step=b.step)
            fo, eo = o.compute(x)
            assert np.abs(f - fo).max() <= 1e-5 * np.abs(fo).max(), stage
            for k in range(19):
                assert abs(e[k] - eo[k]) <= 1e-6 * max(abs(eo[k]), 1.0), (stage, k, e[k], eo[k])
            b.run(120, skin=1.0, neigh_every=10)
            st = b.neighbor_stats()
            assert st["overflow"] == 0
        assert st["builds"] >= 10
        assert not np.array_equal(x0, b.get_state(0)[0])
