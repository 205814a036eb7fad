"""GPU engine against the reference golden vectors and the FP64 oracle.

Tolerances (per term, relative to the term's magnitude with an absolute
floor for terms that are ~0 on a given input):
  plain FP64 form: energies 1e-6, forces 1e-5 of the largest force (max-norm)
  mixed form:      energies 1e-5, forces 1e-4
"""
import numpy as np
import pytest

from conftest import neigh_of, write_case

pytestmark = pytest.mark.gpu

# c1: configuration 1 (8 x 250 residues), made by the compiled reference like the others
CASES = ["c0", "sheet", "r1r69", "r1r69tb", "r1r69go", "r1r69go2", "c0go", "c0x", "sheetx", "c0s", "sheets", "c0v",
         "c1"]
TOL = {"fp64": (1e-6, 1e-5), "mixed": (1e-5, 1e-4)}


def energy_ok(e, ref, tol, floor):
    bad = []
    for k in range(21):
        if k == 20:
            continue
        scale = max(abs(ref[k]), floor)
        if abs(e[k] - ref[k]) > tol * scale:
            bad.append((k, e[k], ref[k]))
    return bad


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", CASES)
def test_single_point_matches_reference(name, prec, tmp_path, gpu_lib):
    from awsemmd_b200.engine import AwsemSystem

    files, g = write_case(name, tmp_path)
    etol, ftol = TOL[prec]
    with AwsemSystem(files, precision=prec) as s:
        s.set_neighbor(*neigh_of(g))
        f, e = s.compute(g["x0"], step=0)
        # energy floor: a term that is ~0 must stay ~0 relative to the total
        floor = 1e-3 * max(1.0, abs(g["e0"][0]) * 1e-6)
        assert not energy_ok(e, g["e0"], etol, floor), energy_ok(e, g["e0"], etol, floor)
        err = np.abs(f - g["f0"]).max() / np.abs(g["f0"]).max()
        assert err < ftol, err
        if prec == "fp64":
            res = s.residue_arrays()
            np.testing.assert_allclose(res[:, :6], g["res0"], rtol=1e-9, atol=1e-10)


@pytest.mark.parametrize("name", CASES)
def test_term_groups_partition_the_forces(name, tmp_path, gpu_lib):
    from awsemmd_b200.engine import AwsemSystem, TERMS_BOND, TERMS_FIX, TERMS_PAIR

    files, g = write_case(name, tmp_path)
    with AwsemSystem(files, precision="fp64") as s:
        s.set_neighbor(*neigh_of(g))
        fa, ea = s.compute(g["x0"])
        f1, e1 = s.compute(g["x0"], terms=TERMS_FIX)
        f2, e2 = s.compute(g["x0"], terms=TERMS_PAIR)
        f3, e3 = s.compute(g["x0"], terms=TERMS_BOND)
    np.testing.assert_allclose(f1 + f2 + f3, fa, rtol=0, atol=1e-8)
    assert abs(e1[0] - ea[0]) < 1e-9 * abs(ea[0])
    assert e1[18] == 0 and e2[0] == 0 and abs(e2[18] - ea[18]) < 1e-9 * max(1, abs(ea[18]))
    assert abs(e3[19] - ea[19]) < 1e-9 * max(1, abs(ea[19]))


@pytest.mark.parametrize("name", CASES)
def test_trajectory_matches_reference(name, tmp_path, gpu_lib):
    from awsemmd_b200.engine import AwsemSystem

    files, g = write_case(name, tmp_path)
    nsteps, dt, t0, t1, damp, seed = g["run"]
    skin, delay, every, check = neigh_of(g)
    with AwsemSystem(files, precision="fp64") as s:
        s.set_neighbor(skin, delay, every, check)
        s.set_state(g["x0"], g["v0"])
        rows = s.run(int(nsteps), dt=dt, langevin=True, t_start=t0, t_stop=t1, damp=damp, seed=int(seed),
                     skin=skin, thermo=True)
        x, v = s.get_state()
    assert np.abs(x - g["xN"]).max() < 1e-6
    assert np.abs(v - g["vN"]).max() < 1e-6
    np.testing.assert_allclose(rows, g["thermo"], rtol=1e-6, atol=1e-6)


def test_multichain_matches_oracle(tmp_path, gpu_lib, oracle_built):
    """Configuration 1 (8 x 250 residues) against the FP64 restatement."""
    import ref
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemSystem

    files = synth.write_system(synth.config_system(1), str(tmp_path / "c1"))
    o = ref.OracleSystem(files)
    with AwsemSystem(files, precision="fp64") as s:
        x, _ = s.get_state()
        fo, eo = o.compute(x)
        f, e = s.compute(x)
        floor = 1e-3
        assert not energy_ok(e, eo, 1e-6, floor), energy_ok(e, eo, 1e-6, floor)
        assert np.abs(f - fo).max() / np.abs(fo).max() < 1e-5
        np.testing.assert_allclose(s.residue_arrays()[:, :6], o.residue_arrays()[:, :6], rtol=1e-9, atol=1e-10)
    with AwsemSystem(files, precision="mixed") as s:
        f, e = s.compute(x)
        assert not energy_ok(e, eo, 1e-5, floor), energy_ok(e, eo, 1e-5, floor)
        assert np.abs(f - fo).max() / np.abs(fo).max() < 1e-4


def test_pair_list_survives_motion(tmp_path, gpu_lib, oracle_built):
    """After 200 Langevin steps (several list rebuilds) forces still match the oracle."""
    import ref
    from awsemmd_b200.engine import AwsemSystem

    files, g = write_case("c0", tmp_path)
    o = ref.OracleSystem(files)
    with AwsemSystem(files, precision="fp64") as s:
        s.set_state(g["x0"], g["v0"])
        s.run(200, dt=2.0, langevin=True, seed=3, skin=1.0)
        st = s.neighbor_stats()
        x, _ = s.get_state()
        f, e = s.compute(x, step=s.step)
    assert st["builds"] >= 2 and st["overflow"] == 0
    fo, eo = o.compute(x)
    assert np.abs(f - fo).max() / np.abs(fo).max() < 1e-5
    assert abs(e[0] - eo[0]) < 1e-6 * abs(eo[0])


def test_nve_energy_drift_matches_reference(tmp_path, gpu_lib):
    """Plain FP64 form, 1,000 constant-energy steps of configuration 0: the
    total energy follows the reference's step by step at first and drifts
    by the reference's amount over the run (golden c0_nve.npz)."""
    import os

    from awsemmd_b200.engine import AwsemSystem

    files, g = write_case("c0", tmp_path)
    nve = np.load(os.path.join(os.path.dirname(__file__), "golden", "c0_nve.npz"))
    with AwsemSystem(files, precision="fp64") as s:
        s.set_state(g["x0"], g["v0"])
        rows = s.run(1000, dt=2.0, langevin=False, thermo=True)
    e, er = rows.sum(axis=1), nve["thermo"].sum(axis=1)
    assert np.abs(e[:200] - er[:200]).max() < 1e-9 * abs(er[0])
    d, dr = np.abs(e - e[0]).max(), np.abs(er - er[0]).max()
    assert abs(d - dr) <= 0.05 * dr, (d, dr)
