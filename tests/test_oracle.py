"""The FP64 restatement (oracle) against the reference's golden vectors."""
import os

import numpy as np
import pytest

from conftest import REFERENCE_SRC, neigh_of, write_case

CASES = ["c0", "sheet", "r1r69", "r1r69tb", "r1r69go", "r1r69go2", "c0go", "c0x", "sheetx", "c0s", "sheets", "c0v"]
# configuration 1 (8 x 250 residues): single point only (the all-pairs oracle
# takes seconds per evaluation at 2,000 residues)
POINT_CASES = CASES + ["c1"]


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", POINT_CASES)
def test_oracle_forces_energies_match_reference(name, tmp_path, oracle_built):
    import ref

    files, g = write_case(name, tmp_path)
    o = ref.OracleSystem(files)
    o.set_neighbor(*neigh_of(g))
    f, e = o.compute(g["x0"])
    # the restatement follows the reference operation order: agreement is at
    # the last bits (energies) and 1e-13 of the largest force
    for k in range(20):
        assert abs(e[k] - g["e0"][k]) <= 1e-11 * max(abs(g["e0"][k]), 1e-3), (k, e[k], g["e0"][k])
    assert rel_err(f, g["f0"]) < 1e-12
    res = o.residue_arrays()
    np.testing.assert_allclose(res[:, :6], g["res0"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("name", CASES)
def test_oracle_trajectory_matches_reference(name, tmp_path, oracle_built):
    import ref

    files, g = write_case(name, tmp_path)
    o = ref.OracleSystem(files)
    o.set_neighbor(*neigh_of(g))
    nsteps, dt, t0, t1, damp, seed = g["run"]
    x, v, thermo = o.run(g["x0"], g["v0"], int(nsteps), dt=dt, langevin=True, t_start=t0, t_stop=t1, damp=damp,
                         seed=int(seed))
    assert np.abs(x - g["xN"]).max() < 1e-9
    assert np.abs(v - g["vN"]).max() < 1e-9
    np.testing.assert_allclose(thermo, g["thermo"], rtol=1e-9, atol=1e-9)


def test_terms_exercised():
    """The fixtures between them exercise every term on the path."""
    e = {n: np.load(os.path.join(os.path.dirname(__file__), "golden", f"{n}.npz"))["e0"] for n in CASES}
    for k, name in [(1, "chain"), (2, "shake"), (3, "chi"), (4, "rama"), (6, "dssp"), (7, "p_ap"), (8, "water"), (9, "burial"),
                    (10, "helix"), (11, "amh-go"), (12, "frag_mem"), (13, "vector frag_mem"), (14, "contact restraints"), (15, "membrane"), (16, "ssb"),
                    (17, "debye-hueckel"), (19, "bond")]:
        assert max(abs(e[c][k]) for c in CASES) > 1e-2, name
    assert max(abs(e[c][18]) for c in CASES) > 1.0  # vexcluded


@pytest.mark.parametrize("name", ["c0go", "c0x"])
def test_list_rule_is_pinned(name, tmp_path, oracle_built):
    """c0go's (AMH-Go) and c0x's (Debye-Hueckel on the CA pairs of the half
    list) trajectories depend on when LAMMPS rebuilds the fix's lists: the
    oracle run with another rebuild rule, or another skin, leaves the
    reference's final positions by more than the parity tolerance (1e-6 A)."""
    import ref

    files, g = write_case(name, tmp_path)
    nsteps, dt, t0, t1, damp, seed = g["run"]
    skin, delay, every, check = neigh_of(g)
    assert (delay, every, check) != (0, 1, 1)
    wrongs = [(skin, 0, 1, 0), (2.0, delay, every, check)]
    if name == "c0go":
        wrongs.append((skin, delay, every, 0))
    for wrong in wrongs:
        o = ref.OracleSystem(files)
        o.set_neighbor(*wrong)
        x, _, _ = o.run(g["x0"], g["v0"], int(nsteps), dt=dt, langevin=True, t_start=t0, t_stop=t1, damp=damp,
                        seed=int(seed))
        o.close()
        assert np.abs(x - g["xN"]).max() > 2e-6, wrong


def test_langevin_stream_shared(oracle_built):
    import ref

    o = ref._load_oracle()

    def mix(z):
        z = (z + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        return z ^ (z >> 31)

    for seed, step, tag, comp in [(1, 0, 1, 0), (12345, 17, 300, 2), (2 ** 40 + 3, 99999, 7, 1)]:
        key = mix(seed ^ mix(step))
        u = (mix(key ^ (tag * 4 + comp)) >> 11) * (1.0 / 9007199254740992.0)
        assert o.oracle_uniform(seed, step, tag, comp) == u


@pytest.mark.skipif(not os.path.isdir(REFERENCE_SRC), reason="reference tree not present")
def test_oracle_matches_reference_on_multichain(tmp_path, oracle_built):
    """Eight 60-residue chains packed in a 60 A cube (inter-chain terms)."""
    import ref
    from awsemmd_b200 import synth

    s = synth.make_system([60] * 8, box=60.0, seed=4242)
    files = synth.write_system(s, str(tmp_path / "mc"))
    r = ref.RefSystem(files)
    fr = r.compute(0)
    er = r.energies()
    o = ref.OracleSystem(files)
    fo, eo = o.compute(r.get("x"))
    for k in range(20):
        assert abs(eo[k] - er[k]) <= 1e-11 * max(abs(er[k]), 1e-3), k
    assert rel_err(fo, fr) < 1e-12


def test_oracle_nve_drift_matches_reference(tmp_path, oracle_built):
    """1,000 constant-energy steps of configuration 0: the restated
    integrator follows the reference's trajectory and energy drift."""
    import numpy as np
    import ref

    files, g = write_case("c0", tmp_path)
    nve = np.load(os.path.join(os.path.dirname(__file__), "golden", "c0_nve.npz"))
    assert str(nve["inputs_sha256"]) == str(g["inputs_sha256"])
    o = ref.OracleSystem(files)
    _, _, rows = o.run(g["x0"], g["v0"], 1000, dt=2.0, langevin=False)
    e, er = rows.sum(axis=1), nve["thermo"].sum(axis=1)
    assert np.abs(e[:200] - er[:200]).max() < 1e-9 * abs(er[0])
    d, dr = np.abs(e - e[0]).max(), np.abs(er - er[0]).max()
    assert abs(d - dr) <= 0.05 * dr, (d, dr)


@pytest.mark.parametrize("name", ["r1r69", "c0"])
def test_oracle_q_matches_reference(name, tmp_path, oracle_built):
    """compute qwolynes / qonuchic in all four types: the restatement against
    the reference computes (compiled in the shim) at the start and the end of
    the 20-step run."""
    import make_golden
    import ref

    files = make_golden.write_q_case(name, str(tmp_path / name))
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", f"q_{name}.npz"))
    assert make_golden.dir_hash(files["workdir"]) == str(g["inputs_sha256"])
    x0 = np.load(os.path.join(os.path.dirname(__file__), "golden", f"{name}.npz"))["x0"]
    o = ref.OracleSystem(files)
    cwd = os.getcwd()
    os.chdir(files["workdir"])
    try:
        for k, words in enumerate(g["words"]):
            for x, want in ((x0, g["q0"][k]), (g["xN"], g["qN"][k])):
                got = o.q(x, str(words))
                assert abs(got - want) <= 1e-12 * max(abs(want), 1e-3), (str(words), got, want)
    finally:
        os.chdir(cwd)


@pytest.mark.skipif(not os.path.isdir(REFERENCE_SRC), reason="reference tree not present")
@pytest.mark.parametrize("L", [2, 3, 5, 8, 9, 10])
def test_oracle_matches_reference_on_short_chains(L, tmp_path, oracle_built):
    """Chains of 2 to 10 residues (no fragment-memory window below 9
    residues): the edge cases of the ragged GPU batch
    (tests/test_gpu_ragged.py), pinned to the reference here."""
    import ref
    from awsemmd_b200 import synth

    c = synth.chain_arrays(L, seed=500 + L, n_mem_per_window=2)
    files = synth.write_chain_arrays(c, str(tmp_path / f"s{L}"))
    r = ref.RefSystem(files)
    fr = r.compute(0)
    er = r.energies()
    o = ref.OracleSystem(files)
    x = r.get("x")
    fo, eo = o.compute(x)
    for k in range(20):
        assert abs(eo[k] - er[k]) <= 1e-11 * max(abs(er[k]), 1e-3), (k, eo[k], er[k])
    assert rel_err(fo, fr) < 1e-12
    assert np.array_equal(np.sort(r.touches()), np.sort(o.selections(x, "touch")))


@pytest.mark.skipif(not os.path.isdir(REFERENCE_SRC), reason="reference tree not present")
def test_oracle_matches_reference_on_longest_config3_replica(tmp_path, oracle_built):
    """The benchmark workload's longest replica (500 residues, 20 memories
    per 9-residue window, the seed the benchmark gives it): the oracle that
    the GPU's configuration-3 sample is compared with
    (tests/test_gpu_c3_sample.py) equals the compiled reference on it --
    energies, forces and the reference's cache entries (selections)."""
    import ref
    from awsemmd_b200 import synth

    lens = synth.replica_lengths(n=1024)
    k = int(np.argmax(lens))
    assert lens[k] == 500
    c = synth.chain_arrays(lens[k], 3000 + k)
    files = synth.write_chain_arrays(c, str(tmp_path / "r"))
    r = ref.RefSystem(files)
    fr = r.compute(0)
    er = r.energies()
    o = ref.OracleSystem(files)
    x = r.get("x")
    fo, eo = o.compute(x)
    for i in range(20):
        assert abs(eo[i] - er[i]) <= 1e-11 * max(abs(er[i]), 1e-3), (i, eo[i], er[i])
    assert rel_err(fo, fr) < 1e-12
    assert np.array_equal(np.sort(r.touches()), np.sort(o.selections(x, "touch")))
