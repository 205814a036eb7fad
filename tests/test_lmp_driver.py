"""Input-script driver (awsemmd_b200/lmp.py) on the CPU: command parsing,
variable substitution and formulas, data and restart files, groups, and the
way a `run` is cut into engine calls at the output steps, with a fake engine
in place of the GPU handle."""
import io
import os

import numpy as np
import pytest

from awsemmd_b200 import lmp
from ref import REFERENCE_DIR  # oracle/ref.py (on the path via conftest)

DATA = """LAMMPS data file for a test

6 atoms
4 bonds

5 atom types
3 bond types

-50.0 50.0 xlo xhi
-50.0 50.0 ylo yhi
-50.0 50.0 zlo zhi

Masses

1 27.0
2 14.0
3 28.0
4 60.0
5 2.0

Bond Coeffs

1 60.0 3.816
2 60.0 2.40
3 60.0 1.53

Atoms

1 1 1 1 0.0 0.0 0.0 0.0
2 1 1 3 0.0 1.0 1.0 0.0
3 1 1 4 0.0 -1.0 0.5 0.0
4 1 2 1 0.0 3.8 0.0 0.0
5 1 2 3 0.0 4.8 1.0 0.0
6 1 2 5 0.0 2.8 -0.5 0.0

Bonds

1 1 1 4
2 2 1 2
3 3 1 3
4 3 4 6
"""


class FakeEngine:
    """Records the engine calls; energies are a function of the step."""

    def __init__(self, **kw):
        self.kw = kw
        self.calls = []
        self._step = 0
        self.n = len(kw["role"])
        self.x = np.array(kw["x"], dtype=float)
        self.v = np.zeros_like(self.x)

    @property
    def step(self):
        return self._step

    def compute(self, x, step=0, **kw):
        self.calls.append(("compute", step))
        self._step = step

    def set_state(self, x, v):
        self.x, self.v = np.array(x, dtype=float), np.array(v, dtype=float)

    def set_neighbor(self, skin, delay, every, check):
        self.calls.append(("neighbor", skin, delay, every, check))

    def q_create(self, words):
        self.calls.append(("q_create", words))
        return 0

    def q_value(self, qid):
        return 0.5 + 0.01 * self._step

    def get_state(self):
        return self.x.copy(), self.v.copy()

    def run_window(self, n, window, cont, **kw):
        self.calls.append(("run", n, tuple(window), cont, kw["t_start"], kw["t_stop"], kw["langevin"]))
        self._step += n
        self.x = self.x + 0.001 * n

    def energies(self):
        e = np.zeros(21)
        e[1:18] = np.arange(1, 18) * (1 + self._step)
        e[0] = e[1:18].sum()
        e[18], e[19], e[20] = 0.5, 2.0, 3.0 + self._step
        return e

    def close(self):
        pass


DECK = """
# a deck in the style of the reference's examples
units real
timestep 2
dimension 3
boundary s s s
neighbor 5 bin
neigh_modify delay 5
atom_modify sort 0 0.0
special_bonds fene
atom_style awsemmd
bond_style harmonic
pair_style vexcluded 2 3.5 3.5
read_data data.test
pair_coeff * * 0.0
pair_coeff 1 1 20.0 3.5 4.5
group alpha_carbons id 1 4
group beta_atoms type 4 5
group oxygens id 2:5:3
fix 1 all nve
fix 11 all langevin 500.0 300.0 1000 3456
fix 2 alpha_carbons backbone beta_atoms oxygens coeff.data test.seq
thermo 5
thermo_style custom step pe ke etotal emol epair f_2 v_E_P
dump 1 all atom 10 out.dump
dump_modify 1 sort id
variable E_chain equal f_2[1]
variable E_bond equal emol
variable E_P equal v_E_chain+v_E_bond
variable E_P equal v_E_chain+v_E_bond+f_2[17]
variable Step equal step
fix energy all print 5 "${Step} ${E_chain} ${E_P}" file energy screen no
reset_timestep 0
run 12
write_restart restart.end
"""


def run_deck(tmp_path, deck=DECK, **kw):
    """Runs a deck in tmp_path (decks name their files relative to the working directory)."""
    (tmp_path / "data.test").write_text(DATA)
    engines = []

    def make(**k):
        engines.append(FakeEngine(**k))
        return engines[-1]

    screen = io.StringIO()
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        d = lmp.Driver(screen=screen, logfile=None, make_engine=make, **kw)
        try:
            d.lines(deck.split("\n"))
        finally:
            d.close()
    finally:
        os.chdir(cwd)
    return d, engines, screen.getvalue()


def test_run_is_cut_at_output_steps(tmp_path):
    d, engines, screen = run_deck(tmp_path)
    (eng,) = engines
    runs = [c for c in eng.calls if c[0] == "run"]
    # setup evaluation, then continuation calls up to each output step (thermo 5, dump 10, print 5) and the end
    assert [(c[1], c[2], c[3]) for c in runs] == [(0, (0, 12), False), (5, (0, 12), True), (5, (0, 12), True),
                                                   (2, (0, 12), True)]
    assert all(c[4:] == (500.0, 300.0, True) for c in runs)  # the ramp spans the whole run
    # `neigh_modify delay 5` reaches the engine with LAMMPS's defaults for the rest
    assert ("neighbor", 5.0, 5, 1, True) in eng.calls
    # roles from the fix's groups, bonds as 0-based indices with the Bond Coeffs
    assert list(eng.kw["role"]) == [0, 2, 1, 0, 2, 1]
    assert list(eng.kw["bonds"][0]) == [0, 0, 0, 3] and list(eng.kw["bonds"][1]) == [3, 1, 2, 5]
    assert list(eng.kw["bonds"][3]) == [3.816, 2.40, 1.53, 1.53]
    assert eng.kw["pair_style"] == "2 3.5 3.5" and eng.kw["pair_coeffs"] == "* * 0.0;1 1 20.0 3.5 4.5"


def test_output_files(tmp_path):
    run_deck(tmp_path)
    # fix print: steps 0, 5, 10 with the formulas evaluated at each
    lines = (tmp_path / "energy").read_text().splitlines()
    assert lines[0] == "# Fix print output for fix energy"
    vals = [[float(t) for t in l.split()] for l in lines[1:]]
    assert [v[0] for v in vals] == [0, 5, 10]
    for s, chain, ep in vals:
        assert chain == 1 * (1 + s) and ep == chain + 2.0 + 17 * (1 + s)
    # energy.log of fix backbone: header and the thermo steps
    log = (tmp_path / "energy.log").read_text().splitlines()
    assert log[0].startswith("Step   \tChain   \tShake")
    rows = [l.split() for l in log[1:]]
    assert [int(r[0]) for r in rows] == [0, 5, 10]
    assert len(rows[0]) == 19 and float(rows[1][1]) == 6.0 and float(rows[1][-1]) == sum(range(1, 18)) * 6
    # dump frames at 0 and 10 in LAMMPS's atom format
    dump = (tmp_path / "out.dump").read_text().splitlines()
    assert dump[:4] == ["ITEM: TIMESTEP", "0", "ITEM: NUMBER OF ATOMS", "6"]
    assert dump[4] == "ITEM: BOX BOUNDS ss ss ss" and dump[8] == "ITEM: ATOMS id type xs ys zs"
    assert dump[9].split()[:2] == ["1", "1"] and dump.count("ITEM: TIMESTEP") == 2
    xs = np.array([[float(t) for t in l.split()[2:]] for l in dump[9:15]])
    assert xs.min() >= 0.0 and xs.max() <= 1.0
    # restart at the end: step 12 with the state the engine returned
    r = lmp.read_data(str(tmp_path / "restart.end"))
    assert r.timestep == 12 and np.allclose(r.x[0], [0.012, 0.012, 0.012])


def test_thermo_keywords(tmp_path):
    d, engines, screen = run_deck(tmp_path)
    out = [l.split() for l in screen.splitlines() if l.strip() and l.split()[0].isdigit()]
    steps = [int(r[0]) for r in out]
    assert steps == [0, 5, 10, 12]  # setup, every 5, the last step
    s, pe, ke, etotal, emol, epair, f2, vep = [float(t) for t in out[-1]]
    e = engines[0].energies()
    assert pe == pytest.approx(e[0] + 0.5 + 2.0) and ke == 15.0 and etotal == pytest.approx(pe + ke)
    assert emol == 2.0 and epair == 0.5 and f2 == pytest.approx(e[0])


def test_restart_round_trip_and_upto(tmp_path):
    run_deck(tmp_path)
    deck = DECK.replace("read_data data.test", "read_restart restart.end").replace("reset_timestep 0\n", "") \
        .replace("run 12", "run 20 upto").replace("write_restart restart.end", "")
    d, engines, _ = run_deck(tmp_path, deck)
    runs = [c for c in engines[0].calls if c[0] == "run"]
    assert runs[0][1:4] == (0, (12, 20), False) and sum(c[1] for c in runs) == 8
    assert ("compute", 12) in engines[0].calls  # the engine's counter moved to the restart's step


def test_formulas_and_substitution():
    d = lmp.Driver(screen=None, logfile=None, make_engine=None, variables={"T": "350"})
    d.lines(["variable a equal 2", "variable b equal v_a^2+3*(1-v_a)/2", "variable c string hello",
             "variable T index 300", "variable n loop 3"])
    assert d.keyword("v_b") == pytest.approx(4 - 1.5)
    assert d.substitute("x ${a} $a $(v_a*3) ${c} ${T} \"${a}\"") == "x 2 2 6 hello 350 \"${a}\""
    assert lmp.Expr("2^3^2", d.keyword).value() == 2 ** 9
    assert lmp.Expr("-2^2", d.keyword).value() == -4
    assert lmp.Expr("(1 < 2) && !(3 == 4)", d.keyword).value() == 1.0
    assert lmp.Expr("sqrt(16)+exp(0)+ln(1)", d.keyword).value() == 5.0
    with pytest.raises(lmp.LammpsError):
        lmp.Expr("1/0", d.keyword).value()
    with pytest.raises(lmp.LammpsError):
        d.var_text("undefined")


def test_groups(tmp_path):
    (tmp_path / "d").write_text(DATA)
    data = lmp.read_data(str(tmp_path / "d"))
    g = {"all": np.ones(6, dtype=bool)}
    assert list(lmp.group_select(data, "id", ["1:6:2"], g).nonzero()[0]) == [0, 2, 4]
    assert list(lmp.group_select(data, "type", ["<>", "3", "4"], g).nonzero()[0]) == [1, 2, 4]
    assert list(lmp.group_select(data, "id", ["<=", "2"], g).nonzero()[0]) == [0, 1]
    g["a"] = lmp.group_select(data, "id", ["1", "2"], g)
    g["b"] = lmp.group_select(data, "id", ["2", "3"], g)
    assert list(lmp.group_select(data, "subtract", ["a", "b"], g).nonzero()[0]) == [0]
    assert list(lmp.group_select(data, "union", ["a", "b"], g).nonzero()[0]) == [0, 1, 2]


@pytest.mark.parametrize("line,msg", [("boundary p p p", "periodic"), ("units lj", "real"),
                                      ("fix 9 all nvt temp 300 300 100", "not supported"),
                                      ("minimize 1e-4 1e-6 100 1000", "Unknown command"),
                                      ("pair_style lj/cut 10", "vexcluded")])
def test_errors(tmp_path, line, msg):
    deck = DECK.replace("units real", "units real\n" + line) if not line.startswith("fix") else \
        DECK.replace("fix 1 all nve", line)
    with pytest.raises(lmp.LammpsError, match=msg):
        run_deck(tmp_path, deck)


REF_EXAMPLE = os.path.join(REFERENCE_DIR, "examples", "examples_new", "1R69_single_memory")


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLE), reason="the reference's example decks are not present")
@pytest.mark.parametrize("deck", ["folding.in", "extended.in", "unfolding.in"])
def test_shipped_decks_parse_and_run(deck, tmp_path):
    """The reference's own 1R69 decks, unmodified, through every command of the
    driver (the fake engine stands in for the GPU; run lengths as shipped)."""
    import shutil

    for f in os.listdir(REF_EXAMPLE):
        p = os.path.join(REF_EXAMPLE, f)
        if os.path.isfile(p) and os.path.getsize(p) < 5_000_000:
            shutil.copy(p, tmp_path / f)
    engines = []

    def make(**k):
        engines.append(FakeEngine(**k))
        return engines[-1]

    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        d = lmp.Driver(screen=None, logfile=None, make_engine=make)
        try:
            d.file(deck)
        finally:
            d.close()
    finally:
        os.chdir(cwd)
    (eng,) = engines
    runs = [c for c in eng.calls if c[0] == "run"]
    assert runs[0][3] is False and all(c[3] for c in runs[1:])
    assert sorted(set(eng.kw["role"])) == [0, 1, 2]
    assert (tmp_path / "energy.log").exists()


def test_q_compute_in_thermo_and_print(tmp_path):
    """compute qwolynes on the CA group: c_ID in thermo columns and fix print
    formulas is the engine's Q at each output step; the definition is made
    once per engine; another group or style is refused."""
    deck = DECK.replace("thermo_style custom step pe ke etotal emol epair f_2 v_E_P",
                        "compute qw alpha_carbons qwolynes rnative.dat 2 0.15\n"
                        "thermo_style custom step pe c_qw") \
               .replace('"${Step} ${E_chain} ${E_P}"', '"${Step} ${Q}"') \
               .replace("variable Step equal step", "variable Step equal step\nvariable Q equal c_qw")
    d, engines, screen = run_deck(tmp_path, deck)
    (eng,) = engines
    assert [c for c in eng.calls if c[0] == "q_create"] == [("q_create", "qw alpha_carbons qwolynes rnative.dat 2 0.15")]
    rows = [l.split() for l in screen.splitlines() if l.strip() and l.split()[0].isdigit()]
    assert [(int(r[0]), float(r[2])) for r in rows] == [(s, 0.5 + 0.01 * s) for s in (0, 5, 10, 12)]
    lines = (tmp_path / "energy").read_text().splitlines()[1:]
    assert [[float(t) for t in l.split()] for l in lines] == [[s, 0.5 + 0.01 * s] for s in (0, 5, 10)]
    for bad, msg in [("compute qw oxygens qwolynes rnative.dat 2 0.15", "CA group"),
                     ("compute qw alpha_carbons rg", "not supported")]:
        with pytest.raises(lmp.LammpsError, match=msg):
            run_deck(tmp_path, deck.replace("compute qw alpha_carbons qwolynes rnative.dat 2 0.15", bad))
