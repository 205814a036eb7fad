"""Batched replicas: parity per replica, and results independent of the mix."""
import numpy as np
import pytest

from conftest import write_case

pytestmark = pytest.mark.gpu


def _extra_chain(tmp_path, L=57, seed=777):
    from awsemmd_b200 import synth

    s = synth.make_system([L], box=200.0, seed=seed)
    return synth.write_system(s, str(tmp_path / f"chain{L}_{seed}"))


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batch_replicas_match_golden(prec, tmp_path, gpu_lib):
    from awsemmd_b200.engine import AwsemBatch

    f0, g0 = write_case("c0", tmp_path)
    f1, g1 = write_case("sheet", tmp_path)
    f2 = _extra_chain(tmp_path)
    etol = 1e-6 if prec == "fp64" else 1e-5
    ftol = 1e-5 if prec == "fp64" else 1e-4
    with AwsemBatch([f0, f2, f1], precision=prec, seeds=[11, 12, 13]) as b:
        assert b.nreplicas == 3
        b.run(0, langevin=False)  # one evaluation at the loaded coordinates
        for r, g in [(0, g0), (2, g1)]:
            e = b.energies(r)
            f = b.forces(r)
            for k in range(20):
                assert abs(e[k] - g["e0"][k]) <= etol * max(abs(g["e0"][k]), 1e-3 * max(1.0, abs(g["e0"][0]) * 1e-6)), \
                    (r, k, e[k], g["e0"][k])
            assert np.abs(f - g["f0"]).max() / np.abs(g["f0"]).max() < ftol


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_replica_alone_equals_replica_in_the_mix(prec, tmp_path, gpu_lib):
    """Bitwise: a replica's trajectory does not depend on its batch mates."""
    from awsemmd_b200.engine import AwsemBatch

    f0, _ = write_case("c0", tmp_path)
    f1, _ = write_case("sheet", tmp_path)
    f2 = _extra_chain(tmp_path)
    kw = dict(dt=2.0, langevin=True, t_start=400.0, t_stop=300.0, damp=500.0, seed=5)
    with AwsemBatch([f2], precision=prec, seeds=[99]) as alone:
        alone.run(150, **kw)
        xa, va = alone.get_state(0)
        ea = alone.energies(0)
    with AwsemBatch([f0, f1, f2, f0], precision=prec, seeds=[1, 2, 99, 3]) as mix:
        mix.run(150, **kw)
        xm, vm = mix.get_state(2)
        em = mix.energies(2)
        x0, _ = mix.get_state(0)
        x3, _ = mix.get_state(3)
    assert np.array_equal(xa, xm) and np.array_equal(va, vm)
    np.testing.assert_allclose(em, ea, rtol=1e-12, atol=1e-9)
    # same input, different seeds: different trajectories
    assert not np.array_equal(x0, x3)


def test_batch_rejects_mismatched_force_fields(tmp_path, gpu_lib):
    from awsemmd_b200.engine import AwsemBatch, AwsemError

    f0, _ = write_case("c0", tmp_path)
    f1, _ = write_case("r1r69", tmp_path)  # different fragment-memory gamma classes
    with pytest.raises(AwsemError, match="share one force field"):
        AwsemBatch([f0, f1])


def test_whole_batch_state_transfer(tmp_path, gpu_lib):
    """awsem_batch_set_state / get_state move every replica in one call and
    agree with the per-replica calls (caller atom order, replicas concatenated)."""
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemBatch

    ff = synth.forcefield_dir(str(tmp_path / "ff"))
    chains = [synth.chain_arrays(L, seed=600 + k, n_mem_per_window=2) for k, L in enumerate([40, 77, 33])]
    with AwsemBatch.from_arrays(ff, chains, precision="mixed", seeds=[1, 2, 3]) as b:
        per = [b.get_state(r) for r in range(3)]
        x, v = b.get_state_all()
        assert np.array_equal(x, np.concatenate([p[0] for p in per]))
        assert np.array_equal(v, np.concatenate([p[1] for p in per]))
        rng = np.random.default_rng(5)
        x2 = x + rng.normal(0, 0.01, x.shape)
        v2 = rng.normal(0, 0.001, v.shape)
        b.set_state_all(x2, v2)
        off = 0
        for r, c in enumerate(chains):
            xr, vr = b.get_state(r)
            n = 3 * c["n_res"]
            assert np.array_equal(xr, x2[off:off + n]) and np.array_equal(vr, v2[off:off + n])
            off += n


def test_autotune_keeps_results(tmp_path, gpu_lib):
    """The autotuner changes launch shapes only: the state is restored and a
    run afterwards is bitwise the run without tuning."""
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemBatch

    ff = synth.forcefield_dir(str(tmp_path / "ff"))
    chains = [synth.chain_arrays(L, seed=650 + k, n_mem_per_window=3) for k, L in enumerate([90, 140, 60])]
    out = []
    for tune in (False, True):
        with AwsemBatch.from_arrays(ff, chains, precision="mixed", seeds=[4, 5, 6]) as b:
            if tune:
                shapes = b.autotune(2)
                assert shapes["fragmem_separations_per_warp"] >= 1 and shapes["pair_pass_blocks"] > 0
            b.run(30)
            out.append(b.get_state_all())
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
