"""Configuration 3 on a sample: eight of the batched workload's own replicas
(its longest, 500 residues, among them), each built from the seed the
benchmark gives it and carrying its own fragment-memory tables (20 memories
per 9-residue window), run as one batch and compared replica by replica with
the FP64 oracle.

Tolerances (relative per energy term with a 1e-2 kcal/mol floor; forces
relative to the largest force, max-norm):
  plain FP64 form: energies 1e-6, forces 1e-5
  mixed form:      energies 1e-5, forces 1e-4
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"fp64": (1e-6, 1e-5), "mixed": (1e-5, 1e-4)}


def sample():
    """(length, seed) of eight configuration-3 replicas: the longest and seven
    drawn with a fixed seed (seeds 3000 + replica index, as the benchmark)"""
    from awsemmd_b200 import synth

    lens = synth.replica_lengths(n=1024)
    pick = [int(np.argmax(lens))] + [int(k) for k in np.random.default_rng(31).choice(1024, 7, replace=False)]
    return [(lens[k], 3000 + k) for k in pick]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_config3_sample_matches_oracle(prec, tmp_path, gpu_lib, oracle_built):
    import ref
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemBatch

    picks = sample()
    assert max(L for L, _ in picks) == 500
    chains = [synth.chain_arrays(L, seed) for L, seed in picks]
    ff = synth.forcefield_dir(str(tmp_path / "ff"))
    etol, ftol = TOL[prec]
    with AwsemBatch.from_arrays(ff, chains, precision=prec, seeds=[s for _, s in picks]) as b:
        b.run(0, langevin=False)
        for r, c in enumerate(chains):
            f, e = b.forces(r), b.energies(r)
            x, _ = b.get_state(r)
            o = ref.OracleSystem(synth.write_chain_arrays(c, str(tmp_path / f"r{r}")))
            fo, eo = o.compute(x)
            o.close()
            for k in range(20):
                assert abs(e[k] - eo[k]) <= etol * max(abs(eo[k]), 1e-2), (r, k, e[k], eo[k])
            assert np.abs(f - fo).max() / np.abs(fo).max() < ftol, r
