"""Ragged batches with the shortest chains: replicas of 2, 3, 5 and 8
residues (too short for any 9-residue fragment-memory window, so no memory
records; the ends of a chain are its first and last residue at once for the
backbone terms), 9 and 10 residues (one and two windows) beside a 64-residue
chain, in one batch.  Every replica is compared with the FP64 oracle at the
starting coordinates and after 40 Langevin steps, where the replica's
positions come from the GPU run itself."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LENGTHS = [2, 3, 5, 8, 9, 10, 64]
TOL = {"fp64": (1e-6, 1e-5), "mixed": (1e-5, 1e-4)}


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_ragged_batch_of_short_chains_matches_oracle(prec, tmp_path, gpu_lib, oracle_built):
    import ref
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemBatch

    chains = [synth.chain_arrays(L, seed=500 + L, n_mem_per_window=2) for L in LENGTHS]
    ff = synth.forcefield_dir(str(tmp_path / "ff"))
    oracles = [ref.OracleSystem(synth.write_chain_arrays(c, str(tmp_path / f"r{k}"))) for k, c in enumerate(chains)]
    etol, ftol = TOL[prec]
    with AwsemBatch.from_arrays(ff, chains, precision=prec, seeds=list(range(1, len(chains) + 1))) as b:
        for stage in range(2):
            if stage:
                b.run(40, dt=2.0, langevin=True, seed=9)
            b.run(0, langevin=False)  # one evaluation at the current coordinates
            for r, o in enumerate(oracles):
                x, _ = b.get_state(r)
                f, e = b.forces(r), b.energies(r)
                fo, eo = o.compute(x)
                assert np.isfinite(f).all() and np.isfinite(e).all(), (stage, r)
                for k in range(20):
                    assert abs(e[k] - eo[k]) <= etol * max(abs(eo[k]), 1e-2), (stage, LENGTHS[r], k, e[k], eo[k])
                assert np.abs(f - fo).max() <= ftol * max(np.abs(fo).max(), 1e-6), (stage, LENGTHS[r])
    for o in oracles:
        o.close()


def test_empty_batch_is_refused(tmp_path, gpu_lib):
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemBatch, AwsemError

    ff = synth.forcefield_dir(str(tmp_path / "ff"))
    with pytest.raises(AwsemError, match="no replicas"):
        AwsemBatch.from_arrays(ff, [])
