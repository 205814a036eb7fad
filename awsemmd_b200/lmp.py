"""LAMMPS input-script driver for the AWSEM step on the GPU.

The reference runs inside LAMMPS: a user writes an input deck (for example
examples/examples_new/1R69_single_memory/folding.in:1-80 of the reference)
that reads an atom_style awsemmd data file, sets pair_style vexcluded and
bond_style harmonic, adds `fix nve`, `fix langevin` and `fix backbone`, and
asks for thermo output, dumps, `fix print` files and restarts.  This module
runs such decks unmodified on this package's engine and writes the same
files: thermo output (screen and log), `dump ... atom` files in LAMMPS's
format, `fix print` files, the `energy.log` that FixBackbone writes itself
(src/fix_backbone.cpp:101-106, 7661-7672), and restart files.

Command subset (what the reference's example decks use around the fix):
units real; dimension 3; boundary (non-periodic styles s, f, m); atom_style
awsemmd; atom_modify / comm_modify / thermo_modify / processors / newton /
timer (accepted, no effect); timestep; neighbor <skin> bin|nsq;
neigh_modify every/delay/check; special_bonds fene; bond_style harmonic;
bond_coeff; pair_style vexcluded|excluded_volume <p> <cut_short>
<cut_long>; pair_coeff; read_data; read_restart / write_restart / restart
(restart files are this driver's own: a data file carrying the timestep);
velocity <group> create|set|zero|scale (all atoms); group (id, type,
molecule: lists, ranges a:b[:c], `<>`, `<`, `>` ... ; union, subtract,
intersect, delete); fix nve / langevin / backbone / print; unfix; thermo;
thermo_style custom; dump atom; dump_modify sort id; undump; variable
equal|string|index|loop; print; reset_timestep; run N [upto]; log; echo;
compute qwolynes / qonuchic on the fix's CA group, c_ID in formulas and
thermo columns (awsem_q_create / awsem_q_value); uncompute.
Anything else (clear, minimize, fix nvt, other computes, ...) is an error
naming the command.

Differences from LAMMPS, by design of the engine: the Langevin noise is the
engine's counter-based stream keyed by (seed, step, atom id) instead of
LAMMPS's RanMars sequence, and `velocity create` draws from numpy's
generator seeded with the command's seed, so trajectories are not LAMMPS's
bit for bit (energies and forces at given coordinates are the reference's);
shrink-wrapped box bounds written to dumps are the atoms' extent at that
step.
"""
from __future__ import annotations

import math
import re
import shlex
import sys

import numpy as np

MVV2E = 48.88821291 * 48.88821291  # units real: (g/mol)(A/fs)^2 -> kcal/mol
BOLTZ = 0.0019872067               # kcal/mol/K
THERMO_DEFAULT = ["step", "temp", "epair", "emol", "etotal", "press"]
E_FIX_TOTAL, E_VEXCL, E_BOND, E_KIN = 0, 18, 19, 20


class LammpsError(Exception):
    pass


# ---------------------------------------------------------------------------
# data files (atom_style awsemmd: atom-ID molecule-ID residue-ID type q x y z [ix iy iz])

class Data:
    def __init__(self):
        self.box = np.array([[-0.5, 0.5]] * 3)
        self.ntypes = 0
        self.nbondtypes = 0
        self.mass = {}
        self.ids = np.zeros(0, dtype=np.int64)
        self.mol = self.res = self.type = np.zeros(0, dtype=np.int64)
        self.q = np.zeros(0)
        self.x = np.zeros((0, 3))
        self.v = np.zeros((0, 3))
        self.bonds = np.zeros((0, 3), dtype=np.int64)  # type, atom id a, atom id b
        self.bond_coeff = {}
        self.timestep = 0


SECTION_NAMES = ("Masses", "Atoms", "Velocities", "Bonds", "Bond Coeffs", "Pair Coeffs", "PairIJ Coeffs", "Angles",
                 "Dihedrals", "Impropers", "Angle Coeffs", "Dihedral Coeffs", "Improper Coeffs")


def read_data(path: str) -> Data:
    d = Data()
    with open(path) as f:
        lines = f.read().split("\n")
    first = lines[0]
    m = re.search(r"timestep\s*=\s*(\d+)", first)
    if m:
        d.timestep = int(m.group(1))
    i = 1
    natoms = nbonds = 0
    while i < len(lines):
        t = lines[i].split("#")[0].strip()
        if t in SECTION_NAMES or any(t.startswith(s + " ") for s in SECTION_NAMES):
            break
        w = t.split()
        if len(w) >= 2 and w[-1] == "atoms":
            natoms = int(w[0])
        elif len(w) >= 2 and w[-1] == "bonds":
            nbonds = int(w[0])
        elif len(w) >= 3 and w[-2:] == ["atom", "types"]:
            d.ntypes = int(w[0])
        elif len(w) >= 3 and w[-2:] == ["bond", "types"]:
            d.nbondtypes = int(w[0])
        elif len(w) == 4 and w[2:] in (["xlo", "xhi"], ["ylo", "yhi"], ["zlo", "zhi"]):
            d.box["xyz".index(w[2][0])] = [float(w[0]), float(w[1])]
        elif len(w) >= 3 and w[-2:] in (["angle", "types"], ["dihedral", "types"], ["improper", "types"]):
            pass
        elif len(w) >= 2 and w[-1] in ("angles", "dihedrals", "impropers") and int(w[0]) != 0:
            raise LammpsError(f"data file {path}: {w[-1]} are not supported (bond_style harmonic only)")
        i += 1
    atoms, vel, bonds = {}, {}, []
    # a section is its keyword line, a blank line, then as many lines as the
    # header counts for it (LAMMPS's read_data reads counted lines)
    counts = {"Masses": d.ntypes, "Atoms": natoms, "Velocities": natoms, "Bonds": nbonds,
              "Bond Coeffs": d.nbondtypes, "Pair Coeffs": d.ntypes, "PairIJ Coeffs": d.ntypes * (d.ntypes + 1) // 2}
    while i < len(lines):
        head = lines[i].split("#")[0].strip()
        i += 1
        if not head:
            continue
        name = next((s for s in SECTION_NAMES if head == s or head.startswith(s + " ")), None)
        if name is None:
            raise LammpsError(f"data file {path}: unknown section '{head}'")
        if name not in counts:
            raise LammpsError(f"data file {path}: {name} are not supported (bond_style harmonic only)")
        while i < len(lines) and not lines[i].split("#")[0].strip():
            i += 1
        body = []
        while len(body) < counts[name]:
            if i >= len(lines):
                raise LammpsError(f"data file {path}: unexpected end of file in section {name}")
            t = lines[i].split("#")[0].split()
            i += 1
            if t:
                body.append(t)
        if name == "Masses":
            for w in body:
                d.mass[int(w[0])] = float(w[1])
        elif name == "Atoms":
            for w in body:
                if len(w) < 8:
                    raise LammpsError(f"data file {path}: Atoms line needs 8 columns for atom_style awsemmd")
                atoms[int(w[0])] = (int(w[1]), int(w[2]), int(w[3]), float(w[4]), float(w[5]), float(w[6]),
                                    float(w[7]))
        elif name == "Velocities":
            for w in body:
                vel[int(w[0])] = (float(w[1]), float(w[2]), float(w[3]))
        elif name == "Bonds":
            for w in body:
                bonds.append((int(w[1]), int(w[2]), int(w[3])))
        elif name == "Bond Coeffs":
            for w in body:
                d.bond_coeff[int(w[0])] = (float(w[1]), float(w[2]))
    if len(atoms) != natoms:
        raise LammpsError(f"data file {path}: {len(atoms)} atoms listed, header says {natoms}")
    if len(bonds) != nbonds:
        raise LammpsError(f"data file {path}: {len(bonds)} bonds listed, header says {nbonds}")
    ids = np.array(sorted(atoms), dtype=np.int64)
    a = np.array([atoms[k] for k in ids], dtype=np.float64).reshape(-1, 7)
    d.ids = ids
    d.mol, d.res, d.type = (a[:, 0].astype(np.int64), a[:, 1].astype(np.int64), a[:, 2].astype(np.int64))
    d.q = a[:, 3]
    d.x = a[:, 4:7].copy()
    d.v = np.array([vel.get(k, (0.0, 0.0, 0.0)) for k in ids], dtype=np.float64).reshape(-1, 3)
    d.bonds = np.array(bonds, dtype=np.int64).reshape(-1, 3)
    return d


def write_data(path: str, d: Data, x: np.ndarray, v: np.ndarray, step: int, bond_coeff: dict):
    """An atom_style awsemmd data file with velocities: this driver's restart format."""
    def r(val):  # shortest text that reads back to the same double
        return repr(float(val))

    out = [f"LAMMPS data file written by the awsemmd_b200 driver, timestep = {step}", "",
           f"{len(d.ids)} atoms", f"{len(d.bonds)} bonds", "", f"{d.ntypes} atom types",
           f"{d.nbondtypes} bond types", ""]
    for k, ax in enumerate("xyz"):
        out.append(f"{r(d.box[k][0])} {r(d.box[k][1])} {ax}lo {ax}hi")
    out += ["", "Masses", ""] + [f"{t} {r(d.mass[t])}" for t in sorted(d.mass)]
    if bond_coeff:
        out += ["", "Bond Coeffs", ""] + [f"{t} {r(bond_coeff[t][0])} {r(bond_coeff[t][1])}" for t in sorted(bond_coeff)]
    out += ["", "Atoms", ""]
    for k in range(len(d.ids)):
        out.append(f"{d.ids[k]} {d.mol[k]} {d.res[k]} {d.type[k]} {r(d.q[k])} {r(x[k, 0])} {r(x[k, 1])} {r(x[k, 2])}")
    out += ["", "Velocities", ""] + [f"{d.ids[k]} {r(v[k, 0])} {r(v[k, 1])} {r(v[k, 2])}" for k in range(len(d.ids))]
    if len(d.bonds):
        out += ["", "Bonds", ""] + [f"{b + 1} {t} {i} {j}" for b, (t, i, j) in enumerate(d.bonds)]
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


# ---------------------------------------------------------------------------
# equal-style expressions

class Expr:
    """Recursive-descent evaluator of LAMMPS equal-style formulas: numbers,
    thermo keywords, v_name, f_ID / f_ID[k], + - * / ^, unary minus,
    parentheses, comparison and logical operators, and the math functions."""

    FUNCS = {"sqrt": math.sqrt, "exp": math.exp, "ln": math.log, "log": math.log10, "abs": abs, "sin": math.sin,
             "cos": math.cos, "tan": math.tan, "asin": math.asin, "acos": math.acos, "atan": math.atan,
             "ceil": math.ceil, "floor": math.floor, "round": round}
    TOK = re.compile(r"\s*(?:(\d+\.?\d*(?:[eE][-+]?\d+)?|\.\d+(?:[eE][-+]?\d+)?)|([A-Za-z_][\w]*(?:\[\d+\])?)"
                     r"|(==|!=|<=|>=|&&|\|\||[-+*/^()<>!,%]))")

    def __init__(self, text: str, lookup):
        self.toks = []
        pos = 0
        text = text.strip()
        while pos < len(text):
            m = self.TOK.match(text, pos)
            if not m or m.end() == pos:
                raise LammpsError(f"invalid syntax in variable formula '{text}'")
            self.toks.append(m.group(1) or m.group(2) or m.group(3))
            pos = m.end()
        self.i = 0
        self.lookup = lookup

    def peek(self):
        return self.toks[self.i] if self.i < len(self.toks) else None

    def take(self):
        t = self.peek()
        self.i += 1
        return t

    def value(self) -> float:
        v = self.logic()
        if self.peek() is not None:
            raise LammpsError(f"invalid syntax near '{self.peek()}' in variable formula")
        return v

    def logic(self):
        v = self.comparison()
        while self.peek() in ("&&", "||"):
            op, w = self.take(), self.comparison()
            v = float(bool(v) and bool(w)) if op == "&&" else float(bool(v) or bool(w))
        return v

    def comparison(self):
        v = self.sum()
        while self.peek() in ("==", "!=", "<", "<=", ">", ">="):
            op, w = self.take(), self.sum()
            v = float({"==": v == w, "!=": v != w, "<": v < w, "<=": v <= w, ">": v > w, ">=": v >= w}[op])
        return v

    def sum(self):
        v = self.product()
        while self.peek() in ("+", "-"):
            v = v + self.product() if self.take() == "+" else v - self.product()
        return v

    def product(self):
        v = self.unary()
        while self.peek() in ("*", "/", "%"):
            op, w = self.take(), self.unary()
            if op == "/" and w == 0:
                raise LammpsError("divide by 0 in variable formula")
            v = v * w if op == "*" else v / w if op == "/" else math.fmod(v, w)
        return v

    def unary(self):
        if self.peek() == "-":
            self.take()
            return -self.unary()
        if self.peek() == "!":
            self.take()
            return float(not self.unary())
        return self.power()

    def power(self):
        v = self.atom()
        if self.peek() == "^":
            self.take()
            return v ** self.unary()
        return v

    def atom(self):
        t = self.take()
        if t is None:
            raise LammpsError("incomplete variable formula")
        if t == "(":
            v = self.logic()
            if self.take() != ")":
                raise LammpsError("missing ')' in variable formula")
            return v
        if re.match(r"^[\d.]", t):
            return float(t)
        if t in self.FUNCS and self.peek() == "(":
            self.take()
            args = [self.logic()]
            while self.peek() == ",":
                self.take()
                args.append(self.logic())
            if self.take() != ")":
                raise LammpsError(f"missing ')' after {t}(")
            return float(self.FUNCS[t](*args))
        return float(self.lookup(t))


# ---------------------------------------------------------------------------
# groups

def group_select(d: Data, style: str, args: list, groups: dict) -> np.ndarray:
    if style in ("union", "subtract", "intersect"):
        masks = [groups[g] for g in args if g in groups]
        if len(masks) != len(args):
            raise LammpsError(f"group {style}: unknown group among {args}")
        m = masks[0].copy()
        for k in masks[1:]:
            m = m | k if style == "union" else m & ~k if style == "subtract" else m & k
        return m
    col = {"id": d.ids, "type": d.type, "molecule": d.mol}.get(style)
    if col is None:
        raise LammpsError(f"group style '{style}' is not supported")
    ops = {"<": np.less, ">": np.greater, "<=": np.less_equal, ">=": np.greater_equal, "==": np.equal,
           "!=": np.not_equal}
    if args and args[0] in ops:
        return ops[args[0]](col, int(args[1]))
    if args and args[0] == "<>":
        return (col >= int(args[1])) & (col <= int(args[2]))
    m = np.zeros(len(col), dtype=bool)
    for a in args:
        p = a.split(":")
        if len(p) == 1:
            m |= col == int(p[0])
        else:
            lo, hi = int(p[0]), int(p[1])
            step = int(p[2]) if len(p) > 2 else 1
            m |= (col >= lo) & (col <= hi) & ((col - lo) % step == 0)
    return m


# ---------------------------------------------------------------------------

class Driver:
    """Executes input-script commands.  `make_engine(**kw)` builds the GPU
    handle (AwsemSystem.from_atoms by default; the CPU tests pass a fake)."""

    def __init__(self, precision: str = "fp64", device: int = 0, screen=sys.stdout, logfile: str | None = "log.lammps",
                 variables: dict | None = None, make_engine=None):
        self.precision, self.device = precision, device
        self.screen = screen
        self.log = open(logfile, "w") if logfile else None
        self.make_engine = make_engine or self._default_engine
        self.vars = {}
        for k, v in (variables or {}).items():
            self.vars[k] = ("index", [str(v)], 0)
        self.units = None
        self.boundary = ["p", "p", "p"]
        self.dt = None
        self.skin, self.neigh_every = 2.0, 0
        self.neigh = {"delay": 0, "every": 1, "check": True}  # LAMMPS's neigh_modify defaults
        self.special_fene = False
        self.atom_style = None
        self.bond_style = None
        self.bond_coeff_cmd = {}
        self.pair_style = None
        self.pair_coeffs = []
        self.data = None
        self.groups = {}
        self.fixes = {}       # ID -> (style, group, args)
        self.fix_order = []
        self.thermo_every = 0
        self.thermo_keys = list(THERMO_DEFAULT)
        self.dumps = {}       # ID -> dict(group, every, file, sort, last)
        self.restart_every, self.restart_files = 0, []
        self.step = 0
        self.eng = None
        self.eng_key = None
        self.computes = {}   # ID -> the words after `compute`
        self.qids = {}       # ID -> (engine, Q definition id)
        self.x = self.v = None   # host state (between runs)
        self.energies = None
        self.energy_log = None
        self.print_files = {}

    # -- output ------------------------------------------------------------
    def out(self, text: str):
        if self.screen:
            self.screen.write(text + "\n")
            self.screen.flush()
        if self.log:
            self.log.write(text + "\n")
            self.log.flush()

    def close(self):
        for f in list(self.print_files.values()) + [self.energy_log, self.log]:
            if f:
                f.close()
        self.print_files, self.energy_log, self.log = {}, None, None
        if self.eng is not None:
            self.eng.close()
            self.eng = None

    # -- input -------------------------------------------------------------
    def file(self, path: str):
        with open(path) as f:
            self.lines(f.read().split("\n"))

    def lines(self, lines):
        buf = ""
        for raw in lines:
            line = raw.rstrip("\n")
            if line.rstrip().endswith("&"):
                buf += line.rstrip()[:-1] + " "
                continue
            self.command(buf + line)
            buf = ""
        if buf:
            self.command(buf)

    @staticmethod
    def strip_comment(line: str) -> str:
        q = None
        for k, ch in enumerate(line):
            if ch in "\"'" and q is None:
                q = ch
            elif ch == q:
                q = None
            elif ch == "#" and q is None:
                return line[:k]
        return line

    def substitute(self, line: str) -> str:
        """$x, ${name} and $(formula) outside quotes, as the LAMMPS input reader does."""
        out, k, q = [], 0, None
        while k < len(line):
            ch = line[k]
            if ch in "\"'" and q is None:
                q = ch
            elif ch == q:
                q = None
            if ch == "$" and q is None and k + 1 < len(line):
                if line[k + 1] == "{":
                    e = line.index("}", k)
                    out.append(self.var_text(line[k + 2:e]))
                    k = e + 1
                    continue
                if line[k + 1] == "(":
                    depth, e = 0, k + 1
                    while e < len(line):
                        depth += line[e] == "("
                        depth -= line[e] == ")"
                        if depth == 0:
                            break
                        e += 1
                    out.append(f"{Expr(line[k + 2:e], self.keyword).value():.15g}")
                    k = e + 1
                    continue
                out.append(self.var_text(line[k + 1]))
                k += 2
                continue
            out.append(ch)
            k += 1
        return "".join(out)

    def text_subst(self, text: str) -> str:
        """Variable substitution of a stored string (fix print, print)."""
        out = re.sub(r"\$\{(\w+)\}", lambda m: self.var_text(m.group(1)), text)
        return re.sub(r"\$(\w)", lambda m: self.var_text(m.group(1)), out)

    def var_text(self, name: str) -> str:
        if name not in self.vars:
            raise LammpsError(f"substitution for illegal variable {name}")
        style, val, idx = self.vars[name]
        if style == "equal":
            return f"{Expr(val, self.keyword).value():.15g}"
        return str(val[idx])

    def command(self, line: str):
        line = self.strip_comment(line).strip()
        if not line:
            return
        line = self.substitute(line)
        try:
            words = shlex.split(line, posix=True)
        except ValueError as e:
            raise LammpsError(f"unbalanced quotes in '{line}': {e}")
        if not words:
            return
        cmd, args = words[0], words[1:]
        handler = getattr(self, "c_" + cmd.replace("/", "_"), None)
        if handler is None:
            raise LammpsError(f"Unknown command: {line}")
        handler(args)

    # -- settings ----------------------------------------------------------
    def c_units(self, a):
        if a != ["real"]:
            raise LammpsError("units: only 'units real' is supported (the fix's parameters are in real units)")
        self.units = "real"

    def c_dimension(self, a):
        if a != ["3"]:
            raise LammpsError("dimension: only 3 is supported")

    def c_boundary(self, a):
        if len(a) != 3:
            raise LammpsError("boundary needs 3 styles")
        for s in a:
            if "p" in s:
                raise LammpsError("boundary: periodic boundaries are not supported by this engine (use s, f or m)")
            if any(c not in "sfm" for c in s):
                raise LammpsError(f"boundary: unknown style '{s}'")
        self.boundary = a

    def c_atom_style(self, a):
        if a[:1] != ["awsemmd"]:
            raise LammpsError("atom_style: only awsemmd is supported")
        self.atom_style = "awsemmd"

    def _accept(self, a):
        pass

    c_atom_modify = c_comm_modify = c_thermo_modify = c_processors = c_newton = c_timer = _accept

    def c_echo(self, a):
        pass

    def c_log(self, a):
        if self.log:
            self.log.close()
        self.log = None if a[0] == "none" else open(a[0], "a" if "append" in a[1:] else "w")

    def c_timestep(self, a):
        self.dt = float(a[0])

    def c_neighbor(self, a):
        self.skin = float(a[0])
        if a[1:] and a[1] not in ("bin", "nsq", "multi"):
            raise LammpsError(f"neighbor: unknown style {a[1]}")

    def c_neigh_modify(self, a):
        # keywords not given keep their values, as in LAMMPS
        k = 0
        while k < len(a):
            if a[k] in ("every", "delay", "check", "once", "page", "one", "binsize", "cluster", "include", "exclude"):
                if a[k] in ("every", "delay"):
                    v = int(a[k + 1])
                    if v < (1 if a[k] == "every" else 0):
                        raise LammpsError(f"neigh_modify: illegal {a[k]} {a[k + 1]}")
                    self.neigh[a[k]] = v
                elif a[k] == "check":
                    if a[k + 1] not in ("yes", "no"):
                        raise LammpsError(f"neigh_modify: check {a[k + 1]}")
                    self.neigh["check"] = a[k + 1] == "yes"
                elif a[k] == "once" and a[k + 1] == "yes":
                    raise LammpsError("neigh_modify once yes is not supported")
                elif a[k] == "exclude":
                    raise LammpsError("neigh_modify exclude is not supported")
                k += 2
            else:
                raise LammpsError(f"neigh_modify: unknown keyword {a[k]}")
        # the engine's own pair list is rebuilt whenever its displacement check
        # fails; `check no` asks for a rebuild every `every` steps on top of it.
        # The list [AMH-Go] reads follows delay/every/check exactly.
        self.neigh_every = 0 if self.neigh["check"] else self.neigh["every"]

    def c_special_bonds(self, a):
        if a == ["fene"] or a == ["lj", "0.0", "1.0", "1.0"] or a == ["lj/coul", "0.0", "1.0", "1.0"]:
            self.special_fene = True
        else:
            raise LammpsError("special_bonds: only fene (1-2 pairs excluded, 1-3 and 1-4 included) is supported")

    def c_bond_style(self, a):
        if a != ["harmonic"]:
            raise LammpsError("bond_style: only harmonic is supported")
        self.bond_style = "harmonic"

    def c_bond_coeff(self, a):
        types = self._type_range(a[0], self.data.nbondtypes if self.data else 100)
        for t in types:
            self.bond_coeff_cmd[t] = (float(a[1]), float(a[2]))
        self.eng_key = None

    def c_pair_style(self, a):
        if a[:1] not in (["vexcluded"], ["excluded_volume"]) or len(a) != 4:
            raise LammpsError("pair_style: only 'vexcluded <p> <cut_short> <cut_long>' is supported")
        self.pair_style = " ".join(a[1:])
        self.pair_coeffs = []
        self.eng_key = None

    def c_pair_coeff(self, a):
        if self.pair_style is None:
            raise LammpsError("pair_coeff command before pair_style is defined")
        self.pair_coeffs.append(" ".join(a))
        self.eng_key = None

    @staticmethod
    def _type_range(s: str, n: int):
        if s == "*":
            return list(range(1, n + 1))
        if "*" in s:
            lo, hi = s.split("*")
            return list(range(int(lo) if lo else 1, (int(hi) if hi else n) + 1))
        return [int(s)]

    # -- atoms ---------------------------------------------------------------
    def c_read_data(self, a):
        if self.atom_style != "awsemmd":
            raise LammpsError("read_data: atom_style awsemmd must be set first")
        if self.data is not None:
            raise LammpsError("read_data: the system is already defined")
        self._load(read_data(a[0]))

    def c_read_restart(self, a):
        if self.data is not None:
            raise LammpsError("read_restart: the system is already defined")
        d = read_data(a[0])
        self._load(d)
        self.step = d.timestep

    def _load(self, d: Data):
        self.data = d
        self.x, self.v = d.x.copy(), d.v.copy()
        self.groups = {"all": np.ones(len(d.ids), dtype=bool)}
        self.eng_key = None

    def c_write_restart(self, a):
        self._need_data("write_restart")
        self._write_restart(a[0])

    def c_restart(self, a):
        self.restart_every = int(a[0])
        self.restart_files = a[1:3] if self.restart_every else []

    def _write_restart(self, name: str):
        write_data(name.replace("*", str(self.step)), self.data, self.x, self.v, self.step, self._bond_coeffs())

    def _need_data(self, what: str):
        if self.data is None:
            raise LammpsError(f"{what} command before simulation box is defined")

    def c_group(self, a):
        self._need_data("group")
        name, style = a[0], a[1]
        if style == "delete":
            self.groups.pop(name, None)
            return
        m = group_select(self.data, style, a[2:], self.groups)
        self.groups[name] = self.groups.get(name, np.zeros_like(m)) | m
        self.eng_key = None

    def c_velocity(self, a):
        self._need_data("velocity")
        g, style = a[0], a[1]
        if g != "all":
            raise LammpsError("velocity: only group all is supported")
        m = self._masses()
        if style == "create":
            temp, seed = float(a[2]), int(a[3])
            kw = dict(zip(a[4::2], a[5::2]))
            rng = np.random.default_rng(seed)
            if kw.get("dist", "uniform") == "gaussian":
                v = rng.standard_normal(self.v.shape)
            else:
                v = rng.uniform(-0.5, 0.5, self.v.shape)
            v = v / np.sqrt(m)[:, None]
            if kw.get("mom", "yes") == "yes":
                v -= (m[:, None] * v).sum(0) / m.sum()
            if kw.get("rot", "no") == "yes":
                raise LammpsError("velocity create rot yes is not supported")
            self.v = v * math.sqrt(temp / self._temp(v))
        elif style == "set":
            for k in range(3):
                if a[2 + k] != "NULL":
                    self.v[:, k] = float(a[2 + k])
        elif style == "zero":
            if a[2] != "linear":
                raise LammpsError("velocity zero: only linear is supported")
            self.v -= (m[:, None] * self.v).sum(0) / m.sum()
        elif style == "scale":
            self.v *= math.sqrt(float(a[2]) / self._temp(self.v))
        else:
            raise LammpsError(f"velocity style {style} is not supported")

    def _masses(self):
        return np.array([self.data.mass[int(t)] for t in self.data.type])

    def _dof(self):
        return 3 * len(self.data.ids) - 3

    def _temp(self, v):
        ke = 0.5 * MVV2E * (self._masses()[:, None] * v * v).sum()
        return 2.0 * ke / (self._dof() * BOLTZ)

    # -- fixes, output -------------------------------------------------------
    def c_compute(self, a):
        if len(a) < 3:
            raise LammpsError("Illegal compute command")
        if a[2] not in ("qwolynes", "qonuchic"):
            raise LammpsError(f"compute style {a[2]} is not supported by this driver")
        if a[1] not in self.groups:
            raise LammpsError(f"Could not find compute group ID {a[1]}")
        self.computes[a[0]] = " ".join(a)
        self.qids.pop(a[0], None)

    def c_uncompute(self, a):
        if a[0] not in self.computes:
            raise LammpsError(f"Could not find uncompute ID {a[0]}")
        del self.computes[a[0]]
        self.qids.pop(a[0], None)

    def _compute_value(self, cid: str) -> float:
        """c_ID of a Q compute on the engine's current positions"""
        if cid not in self.computes:
            raise LammpsError(f"Invalid compute ID c_{cid} in variable formula")
        if self.eng is None:
            raise LammpsError(f"compute {cid} used before the first run")
        words = self.computes[cid]
        fb = [f for f in self.fixes.values() if f[0] == "backbone"]
        if not fb or words.split()[1] != fb[0][1]:
            raise LammpsError(f"compute {cid}: its group must be the CA group of fix backbone")
        held = self.qids.get(cid)
        if held is None or held[0] is not self.eng:
            held = (self.eng, self.eng.q_create(words))
            self.qids[cid] = held
        return float(self.eng.q_value(held[1]))

    def c_fix(self, a):
        fid, group, style, rest = a[0], a[1], a[2], a[3:]
        if group not in self.groups:
            raise LammpsError(f"fix {fid}: could not find fix group ID {group}")
        if style == "nve":
            if group != "all":
                raise LammpsError("fix nve: only group all is supported")
        elif style == "langevin":
            if group != "all":
                raise LammpsError("fix langevin: only group all is supported")
            t0, t1, damp, seed = float(rest[0]), float(rest[1]), float(rest[2]), int(rest[3])
            kw = dict(zip(rest[4::2], rest[5::2]))
            if any(k not in ("zero", "tally") or (k == "zero" and v == "yes") for k, v in kw.items()):
                raise LammpsError(f"fix langevin: keywords {kw} are not supported")
            rest = [t0, t1, damp, seed]
        elif style == "backbone":
            if len(rest) < 4:
                raise LammpsError("fix backbone: needs <CB group> <O group> <coeff file> <sequence file>")
            for gname in rest[:2]:
                if gname not in self.groups:
                    raise LammpsError(f"fix backbone: could not find group {gname}")
            self.eng_key = None
        elif style == "print":
            every, text = int(rest[0]), rest[1]
            kw, k = {"screen": "yes", "file": None, "append": None, "title": f"# Fix print output for fix {fid}"}, 2
            while k < len(rest):
                kw[rest[k]] = rest[k + 1]
                k += 2
            path = kw["file"] or kw["append"]
            if path:
                f = open(path, "a" if kw["append"] else "w")
                if kw["file"]:
                    f.write(kw["title"] + "\n")
                self.print_files[fid] = f
            rest = [every, text, kw["screen"] == "yes"]
        else:
            raise LammpsError(f"fix style {style} is not supported by this driver")
        if fid not in self.fixes:
            self.fix_order.append(fid)
        self.fixes[fid] = (style, group, rest)

    def c_unfix(self, a):
        if a[0] not in self.fixes:
            raise LammpsError(f"could not find fix ID {a[0]} to delete")
        if self.fixes[a[0]][0] == "backbone":
            self.eng_key = None
        del self.fixes[a[0]]
        self.fix_order.remove(a[0])
        f = self.print_files.pop(a[0], None)
        if f:
            f.close()

    def c_thermo(self, a):
        self.thermo_every = int(a[0])

    def c_thermo_style(self, a):
        if a[0] == "one":
            self.thermo_keys = ["step", "temp", "epair", "emol", "etotal", "press"]
        elif a[0] == "custom":
            self.thermo_keys = a[1:]
        else:
            raise LammpsError(f"thermo_style {a[0]} is not supported")

    def c_dump(self, a):
        did, group, style, every, path = a[0], a[1], a[2], int(a[3]), a[4]
        if style != "atom":
            raise LammpsError(f"dump style {style} is not supported (atom only)")
        if group not in self.groups:
            raise LammpsError(f"dump {did}: could not find group {group}")
        self.dumps[did] = {"group": group, "every": every, "file": open(path, "w"), "last": None}

    def c_dump_modify(self, a):
        if a[0] not in self.dumps:
            raise LammpsError(f"dump_modify: could not find dump ID {a[0]}")
        k = 1
        while k < len(a):
            if a[k] == "sort" and a[k + 1] in ("id", "off"):
                k += 2
            elif a[k] in ("flush", "append") and k + 1 < len(a):
                k += 2
            else:
                raise LammpsError(f"dump_modify {a[k]} is not supported")

    def c_undump(self, a):
        d = self.dumps.pop(a[0], None)
        if d is None:
            raise LammpsError(f"could not find undump ID {a[0]}")
        d["file"].close()

    def c_variable(self, a):
        name, style = a[0], a[1]
        if style == "delete":
            self.vars.pop(name, None)
            return
        if style in ("index", "loop") and name in self.vars:
            return  # an existing index variable keeps its value (LAMMPS -var overrides)
        if style == "equal":
            self.vars[name] = ("equal", " ".join(a[2:]), 0)
        elif style == "string":
            self.vars[name] = ("string", [" ".join(a[2:])], 0)
        elif style == "index":
            self.vars[name] = ("index", a[2:], 0)
        elif style == "loop":
            n = int(a[2])
            self.vars[name] = ("loop", [str(k) for k in range(1, n + 1)], 0)
        else:
            raise LammpsError(f"variable style {style} is not supported")

    def c_print(self, a):
        self.out(self.text_subst(a[0]) if a else "")

    def c_reset_timestep(self, a):
        self.step = int(a[0])

    # -- thermo keywords ----------------------------------------------------
    def keyword(self, name: str) -> float:
        if name.startswith("v_"):
            v = self.vars.get(name[2:])
            if v is None:
                raise LammpsError(f"variable {name[2:]} is not defined")
            return Expr(v[1], self.keyword).value() if v[0] == "equal" else float(v[1][v[2]])
        if name == "step":
            return float(self.step)
        if name in ("dt",):
            return float(self.dt or 1.0)
        if name == "time":
            return self.step * float(self.dt or 1.0)
        if name == "atoms":
            return float(len(self.data.ids))
        if name.startswith("c_"):
            return self._compute_value(name[2:])
        e = self.energies
        if e is None:
            raise LammpsError(f"energy keyword {name} used before the first run")
        if name.startswith("f_"):
            m = re.match(r"f_(\w+?)(?:\[(\d+)\])?$", name)
            fid, k = m.group(1), m.group(2)
            if fid not in self.fixes or self.fixes[fid][0] != "backbone":
                raise LammpsError(f"fix {fid} in a formula is not a fix backbone")
            if k is None:
                return float(e[E_FIX_TOTAL])
            k = int(k)
            if not 1 <= k <= 17:
                raise LammpsError(f"fix {fid} vector is accessed out-of-range ([{k}], 17 values)")
            return float(e[k])
        fix_total = float(e[E_FIX_TOTAL]) if any(s[0] == "backbone" for s in self.fixes.values()) else 0.0
        pe = fix_total + float(e[E_VEXCL]) + float(e[E_BOND])
        ke = float(e[E_KIN])
        table = {"pe": pe, "ke": ke, "etotal": pe + ke, "emol": float(e[E_BOND]), "ebond": float(e[E_BOND]),
                 "epair": float(e[E_VEXCL]), "evdwl": float(e[E_VEXCL]), "ecoul": 0.0, "elong": 0.0,
                 "eangle": 0.0, "edihed": 0.0, "eimp": 0.0, "temp": 2.0 * ke / (self._dof() * BOLTZ)}
        if name not in table:
            raise LammpsError(f"thermo keyword {name} is not supported by this driver")
        return table[name]

    # -- the engine ------------------------------------------------------------
    def _bond_coeffs(self) -> dict:
        c = dict(self.data.bond_coeff)
        c.update(self.bond_coeff_cmd)
        return c

    def _default_engine(self, **kw):
        from .engine import AwsemSystem

        return AwsemSystem.from_atoms(**kw)

    def _engine(self):
        key = (id(self.data), tuple(sorted(self.fixes)), tuple(self.pair_coeffs), self.pair_style,
               tuple(sorted(self._bond_coeffs().items())))
        if self.eng is not None and self.eng_key == key:
            return self.eng
        fb = [(fid, f) for fid, f in self.fixes.items() if f[0] == "backbone"]
        if len(fb) != 1:
            raise LammpsError("this driver runs exactly one fix backbone")
        fid, (_, ca_group, (cb_group, o_group, coeff, seq, *_)) = fb[0]
        if not self.special_fene:
            raise LammpsError("special_bonds fene is required (the fix's bonded exclusions)")
        if self.pair_style is None or self.bond_style is None:
            raise LammpsError("pair_style vexcluded and bond_style harmonic are required")
        d = self.data
        role = np.full(len(d.ids), -1, dtype=np.int32)
        role[self.groups[ca_group]] = 0
        role[self.groups[cb_group]] = 1
        role[self.groups[o_group]] = 2
        if (role < 0).any():
            raise LammpsError("every atom must be in the fix backbone's CA, CB or O group")
        if (d.ids != np.arange(1, len(d.ids) + 1)).any():
            raise LammpsError("atom ids must be 1..N")
        coeffs = self._bond_coeffs()
        if len(d.bonds) and any(int(t) not in coeffs for t in d.bonds[:, 0]):
            raise LammpsError("all bond coeffs are not set")
        bk = np.array([coeffs[int(t)][0] for t in d.bonds[:, 0]])
        br = np.array([coeffs[int(t)][1] for t in d.bonds[:, 0]])
        mass = np.zeros(max(d.mass) + 1)
        for t, m in d.mass.items():
            mass[t] = m
        if self.eng is not None:
            self.eng.close()
        self.eng = self.make_engine(workdir=".", coeff=coeff, seq=seq, role=role, residue=d.res, molecule=d.mol,
                                    atom_type=d.type, tag=d.ids, mass_by_type=mass, x=self.x,
                                    bonds=(d.bonds[:, 1] - 1, d.bonds[:, 2] - 1, bk, br),
                                    pair_style=self.pair_style, pair_coeffs=";".join(self.pair_coeffs),
                                    precision=self.precision, device=self.device)
        self.eng_key = key
        self.fix_id = fid
        if self.energy_log is None:
            # FixBackbone writes energy.log in the working directory (src/fix_backbone.cpp:101-106)
            self.energy_log = open("energy.log", "w")
            self.energy_log.write("Step   \tChain   \tShake   \tChi     \tRama    \tExcluded\tDSSP    \tP_AP    \t"
                                  "Water   \tBurial  \tHelix   \tAMH-Go  \tFrag_Mem\tVec_FM  \t"
                                  "Contact_Restraints  \tMembrane\tSSB     \tElectro.\tVTotal\n")
        return self.eng

    # -- run -------------------------------------------------------------------
    def c_run(self, a):
        self._need_data("run")
        n = int(a[0])
        if "upto" in a[1:]:
            n = n - self.step
        if n < 0:
            raise LammpsError("run: invalid number of steps")
        if any(k not in ("upto",) for k in a[1:]):
            raise LammpsError(f"run keywords {a[1:]} are not supported")
        if self.dt is None:
            self.dt = 1.0  # LAMMPS's default for units real
        if not any(f[0] == "nve" for f in self.fixes.values()):
            raise LammpsError("this driver integrates with fix nve (+ fix langevin): fix nve is missing")
        lang = [f[2] for f in self.fixes.values() if f[0] == "langevin"]
        eng = self._engine()
        eng.set_neighbor(self.skin, **self.neigh)
        eng.set_state(self.x, self.v)
        if eng.step != self.step:
            eng.compute(self.x, step=self.step)  # moves the engine's step counter (reset_timestep, read_restart)
        t0, t1, damp, seed = lang[0] if lang else (0.0, 0.0, 100.0, 1)
        kw = dict(dt=self.dt, langevin=bool(lang), t_start=t0, t_stop=t1, damp=damp, seed=seed, skin=self.skin,
                  neigh_every=self.neigh_every)
        s0 = self.step
        window = (s0, s0 + n)
        self.out(f"Setting up run: {n} steps, timestep {self.dt} fs, engine {self.precision} on device {self.device}")
        self.thermo_header()
        eng.run_window(0, window, False, **kw)   # the setup evaluation at s0
        self.after_step(eng, setup=True, last=(n == 0))
        cur = s0
        while cur < s0 + n:
            nxt = self.next_output(cur, s0 + n)
            eng.run_window(nxt - cur, window, True, **kw)
            cur = nxt
            self.step = cur
            self.after_step(eng, setup=False, last=(cur == s0 + n))
        self.out(f"Loop time: {n} steps of {len(self.data.ids)} atoms")

    def next_output(self, cur: int, end: int) -> int:
        cands = [end]
        for every in [self.thermo_every, self.restart_every] + [d["every"] for d in self.dumps.values()] + \
                [f[2][0] for f in self.fixes.values() if f[0] == "print"]:
            if every > 0:
                cands.append((cur // every + 1) * every)
        return min(c for c in cands if c > cur)

    def after_step(self, eng, setup: bool, last: bool):
        x, v = eng.get_state()
        self.x, self.v = x, v
        self.energies = eng.energies()
        s = self.step
        te = self.thermo_every
        if te > 0 and s % te == 0:
            e = self.energies
            self.energy_log.write(f"{s} " + "".join(f"\t{e[k]:8.6f}" for k in range(1, 18)) +
                                  f"\t{e[E_FIX_TOTAL]:8.6f}\n")
            self.energy_log.flush()
        if setup or last or (te > 0 and s % te == 0):
            self.thermo_row()
        for did, d in self.dumps.items():
            if d["every"] > 0 and s % d["every"] == 0 and d["last"] != s:
                self.write_dump(d)
                d["last"] = s
        for fid in self.fix_order:
            style, _, rest = self.fixes[fid]
            if style == "print" and rest[0] > 0 and s % rest[0] == 0:
                text = self.text_subst(rest[1])
                if fid in self.print_files:
                    self.print_files[fid].write(text + "\n")
                    self.print_files[fid].flush()
                if rest[2]:
                    self.out(text)
        if not setup and self.restart_every > 0 and s % self.restart_every == 0:
            names = self.restart_files
            name = names[0] if len(names) == 1 or (s // self.restart_every) % 2 else names[-1]
            self._write_restart(name if "*" in name or len(names) == 2 else name + f".{s}")

    def thermo_header(self):
        self.out(" ".join(f"{k:>14s}" for k in self.thermo_keys))

    def thermo_row(self):
        vals = []
        for k in self.thermo_keys:
            if k == "press" or k == "vol" or (k.startswith("c_") and k[2:] not in self.computes):
                vals.append(f"{'n/a':>14s}")
            elif k == "step":
                vals.append(f"{self.step:>14d}")
            else:
                vals.append(f"{self.keyword(k):>14.8g}")
        self.out(" ".join(vals))

    def write_dump(self, d):
        m = self.groups[d["group"]]
        x = self.x[m]
        ids, types = self.data.ids[m], self.data.type[m]
        lo, hi = self.data.box[:, 0].copy(), self.data.box[:, 1].copy()
        for k, b in enumerate(self.boundary):
            if b[0] == "s" or b[0] == "m":
                ext_lo, ext_hi = self.x[:, k].min(), self.x[:, k].max()
                lo[k] = ext_lo if b[0] == "s" else min(lo[k], ext_lo)
                hi[k] = ext_hi if b[0] == "s" else max(hi[k], ext_hi)
        span = np.where(hi > lo, hi - lo, 1.0)
        f = d["file"]
        f.write(f"ITEM: TIMESTEP\n{self.step}\nITEM: NUMBER OF ATOMS\n{len(ids)}\n")
        f.write("ITEM: BOX BOUNDS " + " ".join(b if len(b) == 2 else b * 2 for b in self.boundary) + "\n")
        for k in range(3):
            f.write(f"{lo[k]:-1.16e} {hi[k]:-1.16e}\n")
        f.write("ITEM: ATOMS id type xs ys zs\n")
        xs = (x - lo) / span
        for k in range(len(ids)):
            f.write(f"{ids[k]} {types[k]} {xs[k, 0]:g} {xs[k, 1]:g} {xs[k, 2]:g}\n")
        f.flush()


def main(argv=None):
    import argparse

    ap = argparse.ArgumentParser(description="Run a LAMMPS input deck of the AWSEM model on the GPU engine")
    ap.add_argument("-in", dest="infile", required=True, help="input script")
    ap.add_argument("-var", nargs="+", action="append", default=[], metavar=("NAME", "VALUE"),
                    help="index-style variable, as LAMMPS's -var")
    ap.add_argument("-log", default="log.lammps")
    ap.add_argument("-screen", default=None, help="'none' to silence the screen")
    ap.add_argument("-precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("-device", type=int, default=0)
    a = ap.parse_args(argv)
    variables = {v[0]: v[1] if len(v) > 1 else "" for v in a.var}
    drv = Driver(precision=a.precision, device=a.device, screen=None if a.screen == "none" else sys.stdout,
                 logfile=None if a.log == "none" else a.log, variables=variables)
    try:
        drv.file(a.infile)
    except LammpsError as e:
        drv.out(f"ERROR: {e}")
        drv.close()
        return 1
    drv.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
