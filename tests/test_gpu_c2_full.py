"""Configuration 2 at its full size against the oracle: one system of 160
chains x 250 residues (40,000 residues) packed in a 320 A cube, whose pair
list comes from the cell grid.  The reference itself cannot run this size
(its n x n pair caches, src/smart_matrix_lib.h, need about 205 GB); the
oracle restatement, pinned to the reference on the golden cases and on
configuration 1, evaluates it directly (all-pairs loops, about two minutes
on one core).  One fragment memory per window keeps the oracle's input
parsing short; the pair terms, the list and the grid are those of the
benchmark's configuration 2."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2_case(tmp_path_factory, oracle_built):
    import ref
    from awsemmd_b200 import synth

    c = synth.packed_arrays([250] * 160, 320.0, 2000, n_mem_per_window=1)
    d = tmp_path_factory.mktemp("c2")
    files = synth.write_chain_arrays(c, str(d / "sys"))
    ff = synth.forcefield_dir(str(d / "ff"))
    x = c["x"].reshape(-1, 3)
    f_o, e_o = ref.OracleSystem(files).compute(x)
    return c, ff, x, f_o, e_o


@pytest.mark.parametrize("prec,ftol,etol", [("fp64", 1e-5, 1e-6), ("mixed", 1e-4, 1e-5)])
def test_config2_full_size_matches_oracle(prec, ftol, etol, c2_case, gpu_lib):
    from awsemmd_b200.engine import AwsemBatch

    c, ff, x, f_o, e_o = c2_case
    assert c["n_res"] == 40000
    with AwsemBatch.from_arrays(ff, [c], precision=prec, seeds=[1]) as b:
        f, e = b.compute(x, step=b.step)
        st = b.neighbor_stats()
    assert st["overflow"] == 0
    assert np.abs(f - f_o).max() <= ftol * np.abs(f_o).max()
    for k in range(19):
        assert abs(e[k] - e_o[k]) <= etol * max(abs(e_o[k]), 1.0), (k, e[k], e_o[k])
