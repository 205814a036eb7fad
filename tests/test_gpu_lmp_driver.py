"""Input-script driver on the GPU: a LAMMPS deck in the style of the
reference's examples (folding.in) run on the reference's own 1R69 inputs
must reproduce the reference's 20-step Langevin run (the golden vectors made
by the shim-hosted reference, tests/golden/make_golden.py) at every output
step; and a run cut into calls at the output steps (awsem_run_window) must be
the run in one call bit for bit."""
import os

import numpy as np
import pytest

from conftest import neigh_of, write_case

pytestmark = pytest.mark.gpu

DECK = """
units real
timestep {dt}
dimension 3
boundary s s s
neighbor {skin} bin
neigh_modify delay {delay} every {every} check {check}
atom_modify sort 0 0.0
special_bonds fene
atom_style awsemmd
bond_style harmonic
pair_style vexcluded 2 3.5 3.5
read_data {data}
pair_coeff * * 0.0
pair_coeff 1 1 20.0 3.5 4.5
pair_coeff 1 4 20.0 3.5 4.5
pair_coeff 4 4 20.0 3.5 4.5
pair_coeff 3 3 20.0 3.5 3.5
group alpha_carbons type 1
group beta_atoms type 4 5
group oxygens type 3
fix 1 all nve
fix 11 all langevin {t0} {t1} {damp} {seed}
fix 2 alpha_carbons backbone beta_atoms oxygens fix_backbone_coeff.data {seq}
thermo {thermo}
dump 1 all atom 10 run.dump
dump_modify 1 sort id
variable E_chain equal f_2[1]
variable E_pot equal pe
variable E_kin equal ke
variable Step equal step
fix energy all print 5 "${{Step}} ${{E_pot}} ${{E_kin}} ${{E_chain}}" file energy screen no
reset_timestep 0
run {nsteps}
write_restart restart.end
"""


def run_deck(files, g, thermo):
    from awsemmd_b200 import lmp

    workdir = files["workdir"]
    nsteps, dt, t0, t1, damp, seed = g["run"]
    skin, delay, every, check = neigh_of(g)
    deck = DECK.format(dt=dt, t0=t0, t1=t1, damp=damp, seed=int(seed), nsteps=int(nsteps), thermo=thermo,
                       skin=skin, delay=delay, every=every, check="yes" if check else "no", data=files["data"],
                       seq=files["seq"])
    cwd = os.getcwd()
    os.chdir(workdir)
    try:
        d = lmp.Driver(precision="fp64", screen=None, logfile="log.test")
        try:
            d.lines(deck.split("\n"))
        finally:
            d.close()
    finally:
        os.chdir(cwd)


@pytest.mark.parametrize("case", ["r1r69", "r1r69tb", "r1r69go", "c0go", "c0x"])
def test_deck_reproduces_the_reference_run(case, tmp_path, gpu_lib):
    """r1r69tb: fragment memory in the table form, as the shipped 1R69 decks
    use it; r1r69go and c0go: [AMH-Go], c0go with neighbor 0.6 and
    neigh_modify delay 3 every 2 (the deck's settings decide when the list
    AMH-Go reads is rebuilt)."""
    from awsemmd_b200 import lmp

    files, g = write_case(case, tmp_path)
    wd = files["workdir"]
    run_deck(files, g, thermo=5)
    rows = g["thermo"]  # per step: fix total, vexcluded, bonds, kinetic (reference, 20 Langevin steps)
    pe_ref, ke_ref = rows[:, 0] + rows[:, 1] + rows[:, 2], rows[:, 3]
    # fix print at steps 0, 5, 10, 15, 20
    out = np.array([[float(t) for t in l.split()] for l in open(os.path.join(wd, "energy")).read().splitlines()[1:]])
    assert list(out[:, 0]) == [0, 5, 10, 15, 20]
    steps = out[:, 0].astype(int)
    np.testing.assert_allclose(out[:, 1], pe_ref[steps], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(out[:, 2], ke_ref[steps], rtol=1e-6, atol=1e-6)
    assert abs(out[0, 3] - g["e0"][1]) <= 1e-6 * abs(g["e0"][1])
    # energy.log of fix backbone at the thermo steps: step 0 is the reference's energy vector
    log = open(os.path.join(wd, "energy.log")).read().splitlines()
    assert log[0].startswith("Step") and [int(l.split()[0]) for l in log[1:]] == [0, 5, 10, 15, 20]
    e0 = [float(t) for t in log[1].split()[1:]]
    for k in range(1, 18):
        assert abs(e0[k - 1] - g["e0"][k]) <= 1e-6 * max(abs(g["e0"][k]), 1.0), k
    assert abs(e0[17] - g["e0"][0]) <= 1e-6 * abs(g["e0"][0])
    # the final state (restart file) is the reference's after 20 steps
    r = lmp.read_data(os.path.join(wd, "restart.end"))
    assert r.timestep == 20
    assert np.abs(r.x - g["xN"]).max() < 1e-6 and np.abs(r.v - g["vN"]).max() < 1e-6
    # dump frames at 0, 10, 20
    assert open(os.path.join(wd, "run.dump")).read().count("ITEM: TIMESTEP") == 3


def test_output_cadence_does_not_change_the_trajectory(tmp_path, gpu_lib):
    """thermo 1 (a call per step) and thermo 20 (calls at 5, 10, 15, 20 only for
    fix print and dumps): the restart files are identical."""
    files, g = write_case("r1r69", tmp_path)
    texts = []
    for thermo in (1, 20):
        run_deck(files, g, thermo=thermo)
        texts.append(open(os.path.join(files["workdir"], "restart.end")).read())
    assert texts[0] == texts[1]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_run_window_parts_equal_one_call(prec, tmp_path, gpu_lib):
    from awsemmd_b200.engine import AwsemError, AwsemSystem

    files, g = write_case("c0", tmp_path)
    kw = dict(dt=2.0, langevin=True, t_start=450.0, t_stop=250.0, damp=500.0, seed=99, neigh_every=10)
    with AwsemSystem(files, precision=prec) as s:
        s.set_state(g["x0"], g["v0"])
        rows_one = s.run(30, thermo=True, **kw)
        x1, v1 = s.get_state()
        e1 = s.energies()
    with AwsemSystem(files, precision=prec) as s:
        s.set_state(g["x0"], g["v0"])
        r0 = s.run_window(0, (0, 30), False, thermo=True, **kw)
        e_setup = s.energies()
        r1 = s.run_window(7, (0, 30), True, thermo=True, **kw)
        r2 = s.run_window(23, (0, 30), True, thermo=True, **kw)
        x2, v2 = s.get_state()
        e2 = s.energies()
        with pytest.raises(AwsemError):  # the window has ended
            s.run_window(1, (0, 30), True, **kw)
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)
    assert np.array_equal(e1, e2)
    assert np.array_equal(np.concatenate([r0, r1, r2]), rows_one)
    # the setup call leaves the energies of step 0 (thermo row 0: fix total, vexcluded, bonds, kinetic)
    np.testing.assert_allclose([e_setup[0], e_setup[18], e_setup[19], e_setup[20]], rows_one[0], rtol=1e-12, atol=1e-9)
    # a state change ends the possibility to continue
    with AwsemSystem(files, precision=prec) as s:
        s.run_window(3, (0, 10), False, **kw)
        s.set_state(g["x0"], g["v0"])
        with pytest.raises(AwsemError):
            s.run_window(3, (0, 10), True, **kw)


def test_deck_q_computes_match_the_reference(tmp_path, gpu_lib):
    """compute qwolynes / qonuchic (all four types) in a deck on the 1R69
    inputs: the values fix print writes at steps 0 and 20 of the reference's
    20-step run are the reference computes' (tests/golden/q_r1r69.npz)."""
    import make_golden

    files = make_golden.write_q_case("r1r69", str(tmp_path / "r1r69"))
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "r1r69.npz"))
    q = np.load(os.path.join(os.path.dirname(__file__), "golden", "q_r1r69.npz"))
    nsteps, dt, t0, t1, damp, seed = g["run"]
    deck = DECK.format(dt=dt, t0=t0, t1=t1, damp=damp, seed=int(seed), nsteps=int(nsteps), thermo=20, skin=2.0,
                       delay=0, every=1, check="yes", data=files["data"], seq=files["seq"])
    comp = "\n".join(f"compute {w}" for w in q["words"])
    qv = "\n".join(f"variable Q{k + 1} equal c_q{k + 1}" for k in range(len(q["words"])))
    line = " ".join(f"${{Q{k + 1}}}" for k in range(len(q["words"])))
    deck = deck.replace("reset_timestep 0", f"{comp}\n{qv}\nfix qprint all print 20 \"{line}\" file qvals screen no\n"
                                            "reset_timestep 0")
    from awsemmd_b200 import lmp

    cwd = os.getcwd()
    os.chdir(files["workdir"])
    try:
        d = lmp.Driver(precision="fp64", screen=None, logfile=None)
        try:
            d.lines(deck.split("\n"))
        finally:
            d.close()
        rows = [[float(t) for t in l.split()] for l in open("qvals").read().splitlines()[1:]]
    finally:
        os.chdir(cwd)
    assert len(rows) == 2
    np.testing.assert_allclose(rows[0], q["q0"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(rows[1], q["qN"], rtol=1e-5, atol=1e-6)
