"""Seeded synthetic AWSEM systems (the workloads the engine is measured on).

A chain is built the way the benchmark configurations describe it:

* sequence i.i.d. uniform over the 20 amino acids;
* C-alpha trace: self-avoiding random walk with 3.8 A virtual bonds,
  CA-CA-CA angles ~ N(110 deg, 10 deg), dihedrals uniform in [-180, 180) deg,
  rejection of any non-bonded CA pair (|i-j| >= 2) closer than 4 A;
* CB (H-beta for glycine, 1.09 A) and O from local ideal geometry
  (CA-CB 1.53 A, CA-O 2.40 A, O-CA(i+1) 2.76 A), CB on the side that gives
  the L-chirality sign of the reference chi term (chi0 < 0);
* secondary structure: random H/E/C segments of length 4-12, written as the
  two ssweight columns (H -> 1 0, E -> 0 1, C -> 0 0);
* fragment memories: for every 9-residue window, 20 memories that are copies
  of the chain's own window with N(0, 1 A) noise on every CA/CB coordinate,
  weight 1, gamma from ``uniform.gamma``.

Systems are written in the reference's input formats: a LAMMPS data file for
``atom_style awsemmd`` (``id molecule residue type q x y z``, types 1 CA,
3 O, 4 CB, 5 H-beta; masses 27/14/28/60/2; harmonic bonds CA-CA 3.816,
CA-O 2.40, O-CA 2.76, CA-CB 1.53, CA-HB 1.09 with K = 60), the sequence file,
``ssweight``, a ``.mem`` list with ``.gro`` memory structures (nm), the
parameter tables, and a ``fix_backbone_coeff.data`` that is the default
parameter file with a ``[Fragment_Memory]`` section enabled.

Seeds: configuration index * 1000 + replica id.
"""
from __future__ import annotations

import math
import os
import shutil
from dataclasses import dataclass, field

import numpy as np

AA = "ARNDCQEGHILKMFPSTWYV"
THREE = {
    "A": "ALA", "R": "ARG", "N": "ASN", "D": "ASP", "C": "CYS", "Q": "GLN", "E": "GLU",
    "G": "GLY", "H": "HIS", "I": "ILE", "L": "LEU", "K": "LYS", "M": "MET", "F": "PHE",
    "P": "PRO", "S": "SER", "T": "THR", "W": "TRP", "Y": "TYR", "V": "VAL",
}
MASSES = {1: 27.0, 2: 14.0, 3: 28.0, 4: 60.0, 5: 2.0}
BOND_COEFFS = {1: (60.0, 3.816), 2: (60.0, 2.40), 3: (60.0, 2.76), 4: (60.0, 1.53), 5: (60.0, 1.09)}
# pair_style vexcluded 2 3.5 3.5 and the pair_coeff lines of the shipped examples
PAIR_STYLE = "2 3.5 3.5"
PAIR_COEFFS = ["* * 0.0", "1 1 20.0 3.5 4.5", "1 4 20.0 3.5 4.5", "4 4 20.0 3.5 4.5", "3 3 20.0 3.5 3.5"]

BOLTZ_REAL = 0.0019872067
MVV2E_REAL = 48.88821291 * 48.88821291

PARAM_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "params")
PARAM_TABLES = ["anti_HB", "anti_NHB", "anti_one", "para_HB", "para_one", "gamma.dat",
                "burial_gamma.dat", "uniform.gamma"]

WINDOW = 9
MEMS_PER_WINDOW = 20


@dataclass
class Chain:
    seq: str
    ca: np.ndarray          # (L,3)
    cb: np.ndarray          # (L,3) H-beta position for glycine
    o: np.ndarray           # (L,3)
    ss: str                 # 'H','E','C' per residue
    # memories: (W, MEMS_PER_WINDOW, WINDOW, 3) in A, already rounded to the
    # .gro text precision; NaN for the CB of glycine
    mem_ca: np.ndarray | None = None
    mem_cb: np.ndarray | None = None
    mem_text: list | None = None  # per window: list of per-memory per-residue (ca_txt, cb_txt)

    @property
    def length(self) -> int:
        return len(self.seq)


@dataclass
class System:
    chains: list
    box: float
    periodic: bool = False
    velocities: np.ndarray | None = None   # (natoms,3) in A/fs, data-file atom order
    temperature: float = 300.0
    seed: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def n_res(self) -> int:
        return sum(c.length for c in self.chains)

    @property
    def n_atoms(self) -> int:
        return 3 * self.n_res


# --------------------------------------------------------------------------
# geometry

def _nerf(a, b, c, bond, angle, torsion):
    bc = c - b
    bc /= np.linalg.norm(bc)
    n = np.cross(b - a, bc)
    nn = np.linalg.norm(n)
    if nn < 1e-8:
        n = np.cross(bc, np.array([1.0, 0.0, 0.0]) if abs(bc[0]) < 0.9 else np.array([0.0, 1.0, 0.0]))
        nn = np.linalg.norm(n)
    n /= nn
    m = np.cross(n, bc)
    d2 = np.array([-bond * math.cos(angle), bond * math.sin(angle) * math.cos(torsion),
                   bond * math.sin(angle) * math.sin(torsion)])
    return c + d2[0] * bc + d2[1] * m + d2[2] * n


def ca_trace(L: int, rng: np.random.Generator, bond=3.8, min_dist=4.0) -> np.ndarray:
    """Self-avoiding CA walk (non-bonded CA pairs >= min_dist)."""
    ca = np.zeros((max(L, 3), 3))
    ca[1] = [bond, 0.0, 0.0]
    th = math.radians(rng.normal(110.0, 10.0))
    ca[2] = ca[1] + bond * np.array([-math.cos(th), math.sin(th), 0.0])
    k = 3
    fails = 0
    while k < L:
        ok = False
        for _ in range(60):
            th = math.radians(rng.normal(110.0, 10.0))
            tor = rng.uniform(-math.pi, math.pi)
            p = _nerf(ca[k - 3], ca[k - 2], ca[k - 1], bond, th, tor)
            d = np.linalg.norm(ca[: k - 1] - p, axis=1)
            if d.min() >= min_dist:
                ok = True
                break
        if ok:
            ca[k] = p
            k += 1
            fails = 0
        else:
            fails += 1
            k = max(3, k - 3 * fails)
    return ca[:L].copy()


def _local_frame(ca, i):
    L = len(ca)
    prev = ca[i - 1] if i > 0 else 2 * ca[0] - ca[1]
    nxt = ca[i + 1] if i < L - 1 else 2 * ca[L - 1] - ca[L - 2]
    b1 = ca[i] - prev
    b2 = nxt - ca[i]
    e1 = b1 / np.linalg.norm(b1)
    e2 = b2 / np.linalg.norm(b2)
    u = e1 - e2
    nu = np.linalg.norm(u)
    u = u / nu if nu > 1e-8 else np.cross(e1, [0.0, 0.0, 1.0])
    n = np.cross(b1, b2)
    nn = np.linalg.norm(n)
    if nn < 1e-8:
        n = np.cross(e1, [1.0, 0.0, 0.0] if abs(e1[0]) < 0.9 else [0.0, 1.0, 0.0])
        nn = np.linalg.norm(n)
    n = n / nn
    return u, n, e2, nxt


def place_beads(ca: np.ndarray, seq: str):
    """CB/HB and O from local ideal geometry around the CA trace."""
    L = len(ca)
    cb = np.zeros_like(ca)
    o = np.zeros_like(ca)
    # O_i in the triangle CA_i, CA_{i+1}: |CA_i O| = 2.40, |O CA_{i+1}| = 2.76
    d = 3.8
    along = (2.40 ** 2 - 2.76 ** 2 + d ** 2) / (2 * d)
    perp = math.sqrt(max(2.40 ** 2 - along ** 2, 0.0))
    alpha = math.radians(52.0)
    for i in range(L):
        u, n, e2, nxt = _local_frame(ca, i)
        sgn = 1.0 if i % 2 == 0 else -1.0
        o[i] = ca[i] + along * e2 + perp * sgn * n
        r = 1.09 if seq[i] == "G" else 1.53
        cb[i] = ca[i] + r * (math.cos(alpha) * u - math.sin(alpha) * n)
    return cb, o


def _chi_sign_fix(ca, cb, o, seq):
    """Flip CB across the CA plane where that brings chi (the reference chi
    term's triple product) to the L side (negative)."""
    an, bn, cn = 0.483, 0.703, -0.186
    ap, bp, cp = 0.444, 0.235, 0.321
    L = len(ca)
    for i in range(1, L - 1):
        n_i = an * ca[i - 1] + bn * ca[i] + cn * o[i - 1]
        cp_i = ap * ca[i] + bp * ca[i + 1] + cp * o[i]
        a = cp_i - ca[i]
        b = ca[i] - n_i
        c = ca[i] - cb[i]
        chi = np.dot(np.cross(a, b), c) / (np.linalg.norm(a) * np.linalg.norm(b) * np.linalg.norm(c))
        if chi > 0:
            _, n, _, _ = _local_frame(ca, i)
            v = cb[i] - ca[i]
            cb[i] = ca[i] + v - 2.0 * np.dot(v, n) * n
    return cb


def ss_segments(L: int, rng: np.random.Generator) -> str:
    out = []
    while len(out) < L:
        kind = "HEC"[rng.integers(0, 3)]
        out.extend(kind * int(rng.integers(4, 13)))
    return "".join(out[:L])


def _fmt_nm(x_a: float) -> str:
    return f"{x_a / 10.0:.5f}"


def build_memories(ch: Chain, rng: np.random.Generator, n_per=MEMS_PER_WINDOW, win=WINDOW, sigma=1.0):
    """Noisy copies of every window.  Coordinates are rounded to the .gro text
    that gets written (nm, 5 decimals) and read back as float(text) * 10, the
    same arithmetic the reference's .gro reader applies."""
    L = ch.length
    W = max(L - win + 1, 0)
    mem_ca = np.zeros((W, n_per, win, 3))
    mem_cb = np.full((W, n_per, win, 3), np.nan)
    text = []
    for w in range(W):
        wt = []
        for m in range(n_per):
            noise_ca = rng.normal(0.0, sigma, size=(win, 3))
            noise_cb = rng.normal(0.0, sigma, size=(win, 3))
            rows = []
            for r in range(win):
                i = w + r
                ca_txt = [_fmt_nm(v) for v in ch.ca[i] + noise_ca[r]]
                mem_ca[w, m, r] = [float(t) * 10 for t in ca_txt]
                cb_txt = None
                if ch.seq[i] != "G":
                    cb_txt = [_fmt_nm(v) for v in ch.cb[i] + noise_cb[r]]
                    mem_cb[w, m, r] = [float(t) * 10 for t in cb_txt]
                rows.append((ca_txt, cb_txt))
            wt.append(rows)
        text.append(wt)
    ch.mem_ca, ch.mem_cb, ch.mem_text = mem_ca, mem_cb, text


def make_chain(L: int, rng: np.random.Generator, memories=True) -> Chain:
    seq = "".join(AA[k] for k in rng.integers(0, 20, size=L))
    ca = ca_trace(L, rng)
    cb, o = place_beads(ca, seq)
    cb = _chi_sign_fix(ca, cb, o, seq)
    ss = ss_segments(L, rng)
    ch = Chain(seq=seq, ca=ca, cb=cb, o=o, ss=ss)
    if memories:
        build_memories(ch, rng)
    return ch


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([
        [a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
        [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
        [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d],
    ])


def pack_chains(chains, box: float, rng: np.random.Generator, min_dist=4.0, tries=200):
    """Random rotation + translation of each chain, rejecting placements with
    an inter-chain CA pair closer than min_dist."""
    from scipy.spatial import cKDTree

    placed = []
    tree_pts = np.zeros((0, 3))
    for ch in chains:
        com = ch.ca.mean(axis=0)
        for attempt in range(tries):
            R = _random_rotation(rng)
            shift = rng.uniform(-box / 2, box / 2, size=3)
            new_ca = (ch.ca - com) @ R.T + shift
            if len(tree_pts) == 0:
                ok = True
            else:
                d, _ = cKDTree(tree_pts).query(new_ca, k=1)
                ok = d.min() >= min_dist
            if ok:
                break
        else:
            raise RuntimeError("could not place chain without overlap")
        for name in ("ca", "cb", "o"):
            setattr(ch, name, (getattr(ch, name) - com) @ R.T + shift)
        if ch.mem_ca is not None:
            pass  # memories are internal distances only; orientation does not matter
        tree_pts = np.vstack([tree_pts, ch.ca])
        placed.append(ch)
    return placed


def atom_arrays(sys_: System):
    """Data-file order: per residue CA, O, CB/HB.  Returns (x, type, mol, res)."""
    xs, types, mols, ress = [], [], [], []
    r = 0
    for ci, ch in enumerate(sys_.chains):
        for i in range(ch.length):
            r += 1
            xs += [ch.ca[i], ch.o[i], ch.cb[i]]
            types += [1, 3, 5 if ch.seq[i] == "G" else 4]
            mols += [ci + 1] * 3
            ress += [r] * 3
    return np.array(xs, dtype=np.float64), np.array(types, np.int32), np.array(mols, np.int32), np.array(ress, np.int32)


def write_native_gro(sys_: System, path: str, scale: float = 1.0) -> None:
    """A native structure for [AMH-Go] (amh-go.gro): the system's CA and CB
    atoms (no CB for glycine), residues numbered 1..n over all chains,
    coordinates scaled by `scale` about the CA centroid (scale < 1 makes the
    native structure more compact than the system), in nm."""
    ca = np.concatenate([ch.ca for ch in sys_.chains])
    c0 = ca.mean(axis=0)
    lines, r, k = [], 0, 0
    for ch in sys_.chains:
        for i in range(ch.length):
            r += 1
            beads = [("CA", ch.ca[i])] + ([] if ch.seq[i] == "G" else [("CB", ch.cb[i])])
            for name, x in beads:
                k += 1
                y = c0 + scale * (np.asarray(x) - c0)
                lines.append(f"{r:5d}{THREE[ch.seq[i]]:>5s}{name:>5s}{k:5d} "
                             + " ".join(_fmt_nm(float(v)) for v in y))
    with open(path, "w") as f:
        f.write(f"native structure (synthetic, scale {scale})\n{len(lines)}\n" + "\n".join(lines) + "\n   0.0 0.0 0.0\n")


# [Solvent_Barrier] settings of the synthetic pair-term cases: well 1 (barrier)
# and well 2 strengths and ranges (A), kappa, minimum same-chain separation,
# radius correction on, and per residue type radius shifts (A)
SSB_PARAMS = (0.35, 6.0, 7.0, -0.2, 7.5, 9.0, 5.0, 10, 1,
              (0.00, 0.20, 0.06, 0.06, 0.04, 0.11, 0.12, -0.15, 0.09, 0.07,
               0.08, 0.15, 0.10, 0.10, -0.01, 0.03, 0.04, 0.12, 0.12, 0.04))
# [DebyeHuckel]: strengths ++, --, +- (strong, so that which pairs the fix's list holds
# shows in a short trajectory); screening constant; screening length (A); minimum separation
DH_PARAMS = (40.0, 40.0, 40.0, 1.0, 5.0, 10)


def pair_terms_text(k_cont_rest=1.0, cr_sigma=1.0, cr_file="contact_restraints.dat") -> str:
    """[Solvent_Barrier], [DebyeHuckel] and [Contact_Restraints] sections."""
    k1, a1, b1, k2, a2, b2, kap, sep, cor, shifts = SSB_PARAMS
    kpp, kmm, kpm, ks, L, msep = DH_PARAMS
    return (f"\n[Solvent_Barrier]\n{k1}\n{a1} {b1}\n{k2}\n{a2} {b2}\n{kap}\n{sep}\n{cor}\n"
            + " ".join(str(v) for v in shifts) + "\n"
            + f"\n[DebyeHuckel]\n{kpp} {kmm} {kpm}\n{ks}\n{L}\n{msep}\n"
            + f"\n[Contact_Restraints]\n{k_cont_rest}\n{cr_sigma}\n{cr_file}\n")


def residue_terms_text(sys_: System, phosph=None) -> str:
    """[Shake] (the reference examples' lengths), [Membrane] centred on the
    system's CA centroid (30 A slab, distorted pore, per-zone gammas) and
    [Phosphorylation] of the given residue numbers (hypercharge 1.2)."""
    ca = np.concatenate([ch.ca for ch in sys_.chains])
    c = ca.mean(axis=0)
    gm = ((1.0, 0.8, 1.2, 0.5), (0.7, 0.9, 1.1, 0.6), (0.4, 1.3, 0.9, 0.8))
    text = "\n[Shake]\n10.0 3.83 2.36 2.71\n"
    text += (f"\n[Membrane]\n1.0\n0.5\n{c[0]:.3f} {c[1]:.3f} {c[2]:.3f}\n0\n30.0\n5.0\n0.3\n"
             + "".join(" ".join(str(v) for v in row) + "\n" for row in gm))
    if phosph:
        text += f"\n[Phosphorylation]\n1.2\n{len(phosph)}\n" + " ".join(str(r) for r in phosph) + "\n"
    return text


def write_zim(sys_: System, path: str, seed: int = 11) -> None:
    """zim: a membrane zone (1, 2 or 3) per residue, seeded."""
    n = sum(ch.length for ch in sys_.chains)
    z = np.random.default_rng(seed).integers(1, 4, size=n)
    with open(path, "w") as f:
        f.write("\n".join(str(int(v)) for v in z) + "\n")


def write_q_files(ca_native: np.ndarray, outdir: str, r_contact: float = 9.5) -> None:
    """Inputs of the Q order parameters for a native CA trace [n][3] (A):
    rnative.dat (compute qwolynes: the n x n CA-CA distance matrix),
    native_ca.dat (compute qonuchic cutoff: the count, then CA coordinates)
    and shadow.dat (compute qonuchic shadow: "i j r" for the native pairs
    with |i - j| > 3 closer than r_contact)."""
    ca = np.asarray(ca_native, dtype=np.float64)
    n = len(ca)
    d = np.linalg.norm(ca[:, None, :] - ca[None, :, :], axis=-1)
    with open(os.path.join(outdir, "rnative.dat"), "w") as f:
        for i in range(n):
            f.write(" ".join(f"{float(v):.6f}" for v in d[i]) + "\n")
    with open(os.path.join(outdir, "native_ca.dat"), "w") as f:
        f.write(f"{n}\n" + "".join(f"{float(p[0]):.6f} {float(p[1]):.6f} {float(p[2]):.6f}\n" for p in ca))
    with open(os.path.join(outdir, "shadow.dat"), "w") as f:
        for i in range(n):
            for j in range(i + 4, n):
                if d[i, j] < r_contact:
                    f.write(f"{i + 1} {j + 1} {float(d[i, j]):.6f}\n")


def write_charges(sys_: System, path: str) -> None:
    """charge_on_residues.dat: +1 on K and R, -1 on D and E (residues numbered over all chains)."""
    seq = "".join(ch.seq for ch in sys_.chains)
    rec = [(k + 1, 1.0 if a in "KR" else -1.0) for k, a in enumerate(seq) if a in "KRDE"]
    with open(path, "w") as f:
        f.write(f"{len(rec)}\n" + "".join(f"{r} {q}\n" for r, q in rec))


def write_contact_restraints(sys_: System, path: str, n: int = 24, seed: int = 5) -> None:
    """Restraints "i j w r0" on residue pairs whose contact beads are within
    12 A (separation > 2), r0 the current distance shifted by up to 2 A; plus
    a pair listed twice (the first record counts) and an adjacent pair (never
    evaluated: the fix skips |i - j| <= 1 on one chain)."""
    rng = np.random.default_rng(seed)
    beads = np.concatenate([np.where(np.array([a == "G" for a in ch.seq])[:, None], ch.ca, ch.cb)
                            for ch in sys_.chains])
    nres = len(beads)
    d = np.linalg.norm(beads[:, None, :] - beads[None, :, :], axis=-1)
    cand = [(i, j) for i in range(nres) for j in range(i + 3, nres) if d[i, j] < 12.0]
    pick = rng.choice(len(cand), size=min(n, len(cand)), replace=False)
    lines = []
    for k in pick:
        i, j = cand[k]
        w = round(float(rng.uniform(1.0, 2.0)), 3)
        r0 = round(float(max(3.5, d[i, j] + rng.uniform(-2.0, 2.0))), 3)
        lines.append(f"{j + 1} {i + 1} {w} {r0}" if rng.random() < 0.3 else f"{i + 1} {j + 1} {w} {r0}")
    i, j = cand[pick[0]]
    lines.append(f"{i + 1} {j + 1} 5.0 {round(float(d[i, j]), 3)}")  # duplicate: ignored
    lines.append(f"4 5 3.0 {round(float(d[3, 4]), 3)}")  # adjacent: ignored
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def bond_list(sys_: System):
    """(type, atom_i, atom_j) with 0-based atom indices in data-file order."""
    bonds = []
    base = 0
    for ch in sys_.chains:
        L = ch.length
        for i in range(L):
            a_ca, a_o, a_cb = base + 3 * i, base + 3 * i + 1, base + 3 * i + 2
            bonds.append((2, a_ca, a_o))
            bonds.append((5 if ch.seq[i] == "G" else 4, a_ca, a_cb))
            if i < L - 1:
                bonds.append((1, a_ca, base + 3 * (i + 1)))
                bonds.append((3, a_o, base + 3 * (i + 1)))
        base += 3 * L
    return bonds


def maxwell_velocities(types: np.ndarray, T: float, rng: np.random.Generator) -> np.ndarray:
    """Gaussian velocities (A/fs), zero total momentum, scaled to T exactly
    with 3N-3 degrees of freedom (LAMMPS compute temp)."""
    m = np.array([MASSES[int(t)] for t in types])
    v = rng.normal(size=(len(types), 3)) / np.sqrt(m)[:, None]
    p = (m[:, None] * v).sum(axis=0) / m.sum()
    v -= p
    ke2 = (m[:, None] * v * v).sum() * MVV2E_REAL
    dof = 3 * len(types) - 3
    t_now = ke2 / (dof * BOLTZ_REAL)
    return v * math.sqrt(T / t_now)


def make_system(chain_lengths, box: float, seed: int, T=300.0, memories=True) -> System:
    rng = np.random.default_rng(seed)
    chains = [make_chain(L, rng, memories=memories) for L in chain_lengths]
    if len(chains) > 1:
        chains = pack_chains(chains, box, rng)
    else:
        com = chains[0].ca.mean(axis=0)
        for name in ("ca", "cb", "o"):
            setattr(chains[0], name, getattr(chains[0], name) - com)
    s = System(chains=chains, box=box, temperature=T, seed=seed)
    _, types, _, _ = atom_arrays(s)
    s.velocities = maxwell_velocities(types, T, rng)
    return s


# --------------------------------------------------------------------------
# benchmark configurations

CONFIGS = {
    0: dict(name="c0_1x100", chains=[100], box=300.0, steps=1000, T=300.0, dt=2.0, damp=500.0),
    1: dict(name="c1_8x250", chains=[250] * 8, box=150.0, steps=1000, T=300.0, dt=2.0, damp=500.0),
    2: dict(name="c2_160x250", chains=[250] * 160, box=320.0, steps=500, T=300.0, dt=2.0, damp=500.0,
            skin=2.0, every=10),
}


def config_system(k: int, replica: int = 0, memories=True) -> System:
    c = CONFIGS[k]
    return make_system(c["chains"], c["box"], seed=k * 1000 + replica, T=c["T"], memories=memories)


def replica_lengths(n=1024, lo=40, hi=500, seed=3000):
    """Chain lengths of the batched-replica workload: uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    return [int(x) for x in rng.integers(lo, hi + 1, size=n)]


# --------------------------------------------------------------------------
# writers (the reference's input formats)

def coeff_text(k_fm=1.0, mem_file="frags.mem", gamma_file="uniform.gamma", table=None, amh_go=None) -> str:
    """The repository's parameter file plus a [Fragment_Memory] section, or with
    table = (rmin, rmax, dr, well_width, use_table_files, sigma_exp) a
    [Fragment_Memory_Table] section instead; amh_go = (k, p, rc, censoring)
    adds an [AMH-Go] section (inputs amh-go.gro and amh-go.gamma)."""
    with open(os.path.join(PARAM_DIR, "fix_backbone_coeff.data")) as f:
        base = f.read()
    if table is None:
        text = base.rstrip("\n") + f"\n\n[Fragment_Memory]\n{k_fm}\n{mem_file}\n{gamma_file}\n"
    else:
        rmin, rmax, dr, width, use, sexp = table
        text = base.rstrip("\n") + (f"\n\n[Fragment_Memory_Table]\n{k_fm}\n{mem_file}\n{gamma_file}\n"
                                     f"{rmin} {rmax} {dr}\n{width}\n{use}\n{sexp}\n")
    if amh_go is not None:
        k, pw, rc, cens = amh_go
        text += f"\n[AMH-Go]\n{k}\n{pw}\n{rc}\n{cens}\n"
    return text


def write_system(sys_: System, outdir: str, with_fm=True) -> dict:
    os.makedirs(outdir, exist_ok=True)
    x, types, mols, ress = atom_arrays(sys_)
    bonds = bond_list(sys_)
    h = sys_.box / 2
    lines = ["LAMMPS data file (synthetic AWSEM system)", "",
             f"{len(x)} atoms", f"{len(bonds)} bonds", "0 angles", "0 dihedrals", "0 impropers", "",
             "5 atom types", "5 bond types", "0 angle types", "0 dihedral types", "0 improper types", "",
             f"{-h:.1f} {h:.1f} xlo xhi", f"{-h:.1f} {h:.1f} ylo yhi", f"{-h:.1f} {h:.1f} zlo zhi", "",
             "Masses", ""]
    lines += [f"{t} {MASSES[t]}" for t in range(1, 6)]
    lines += ["", "Atoms", ""]
    for i in range(len(x)):
        lines.append(f"{i + 1} {mols[i]} {ress[i]} {types[i]} 0.0 {float(x[i, 0])!r} {float(x[i, 1])!r} {float(x[i, 2])!r}")
    if sys_.velocities is not None:
        lines += ["", "Velocities", ""]
        v = sys_.velocities
        for i in range(len(x)):
            lines.append(f"{i + 1} {float(v[i, 0])!r} {float(v[i, 1])!r} {float(v[i, 2])!r}")
    lines += ["", "Bond Coeffs", ""]
    lines += [f"{t} {BOND_COEFFS[t][0]} {BOND_COEFFS[t][1]}" for t in range(1, 6)]
    lines += ["", "Bonds", ""]
    for b, (t, i, j) in enumerate(bonds):
        lines.append(f"{b + 1} {t} {i + 1} {j + 1}")
    with open(os.path.join(outdir, "data.awsem"), "w") as f:
        f.write("\n".join(lines) + "\n")
    with open(os.path.join(outdir, "protein.seq"), "w") as f:
        f.write("\n".join(c.seq for c in sys_.chains) + "\n")
    with open(os.path.join(outdir, "ssweight"), "w") as f:
        for c in sys_.chains:
            for s in c.ss:
                f.write({"H": "1.0 0.0\n", "E": "0.0 1.0\n", "C": "0.0 0.0\n"}[s])
    for t in PARAM_TABLES:
        shutil.copy(os.path.join(PARAM_DIR, t), os.path.join(outdir, t))
    with open(os.path.join(outdir, "fix_backbone_coeff.data"), "w") as f:
        if with_fm:
            f.write(coeff_text())
        else:
            with open(os.path.join(PARAM_DIR, "fix_backbone_coeff.data")) as g:
                f.write(g.read())
    if with_fm:
        _write_memories(sys_, outdir)
    return {"workdir": outdir, "data": "data.awsem", "coeff": "fix_backbone_coeff.data",
            "seq": "protein.seq", "pair_style": PAIR_STYLE, "pair_coeffs": ";".join(PAIR_COEFFS)}


def _write_memories(sys_: System, outdir: str):
    memdir = os.path.join(outdir, "mems")
    os.makedirs(memdir, exist_ok=True)
    mem_lines = ["[Target]", "query", "", "[Memories]"]
    res0 = 0
    for ci, ch in enumerate(sys_.chains):
        for w, wt in enumerate(ch.mem_text):
            fname = f"mems/c{ci + 1:03d}_w{w + 1:04d}.gro"
            rows = []
            atom = 0
            for m, mem in enumerate(wt):
                for r, (ca_txt, cb_txt) in enumerate(mem):
                    resnum = m * WINDOW + r + 1
                    rn = THREE[ch.seq[w + r]]
                    atom += 1
                    rows.append(f"{resnum} {rn} CA {atom} {ca_txt[0]} {ca_txt[1]} {ca_txt[2]}")
                    if cb_txt is not None:
                        atom += 1
                        rows.append(f"{resnum} {rn} CB {atom} {cb_txt[0]} {cb_txt[1]} {cb_txt[2]}")
            with open(os.path.join(outdir, fname), "w") as f:
                f.write(f"memory window {w + 1} of chain {ci + 1}\n{len(rows)}\n" + "\n".join(rows) + "\n0.0 0.0 0.0\n")
            for m in range(len(wt)):
                mem_lines.append(f"{fname} {res0 + w + 1} {m * WINDOW + 1} {WINDOW} 1")
        res0 += ch.length
    with open(os.path.join(outdir, "frags.mem"), "w") as f:
        f.write("\n".join(mem_lines) + "\n")


# --------------------------------------------------------------------------
# beta-sheet test system: exercises the hydrogen-bond (all separation
# classes below 45), P_AP (medium, long, parallel, inter-chain) and burial
# branches that random-coil chains barely reach

def _arc(p, q, n_inner: int, step: float, bulge: np.ndarray) -> np.ndarray:
    """n_inner points on a circular arc from p to q (exclusive) with spacing
    close to `step`, bulging towards `bulge`."""
    c = np.linalg.norm(q - p)
    s = (n_inner + 1) * step
    # solve 2 R sin(t/2) = c, R t = s for t in (0, 2 pi)
    lo, hi = 1e-6, 2 * math.pi - 1e-6
    for _ in range(200):
        t = 0.5 * (lo + hi)
        if 2 * (s / t) * math.sin(t / 2) > c:
            lo = t
        else:
            hi = t
    R = s / t
    e = (q - p) / c
    b = bulge - np.dot(bulge, e) * e
    b /= np.linalg.norm(b)
    mid = 0.5 * (p + q)
    h = R * math.cos(t / 2)
    center = mid - h * b
    u0 = (p - center) / R
    w = np.cross(u0, (q - center) / R)
    w /= np.linalg.norm(w)
    v0 = np.cross(w, u0)
    return np.array([center + R * (math.cos(a) * u0 + math.sin(a) * v0)
                     for a in np.linspace(0, t, n_inner + 2)[1:-1]])


def sheet_system(seed=7, T=300.0) -> System:
    rng = np.random.default_rng(seed)
    rise, gap, pleat = 3.3, 4.8, 0.9

    def strand(n, x0, y, direction, z0=0.0):
        return np.array([[x0 + direction * rise * k, y, z0 + pleat * (1 if k % 2 == 0 else -1)] for k in range(n)])

    chains = []
    # chain 1: strand(12) - turn(4) - strand(12) - loop(6) - strand(10), a three-stranded sheet
    s1 = strand(12, 0.0, 0.0, +1)
    s2 = strand(12, s1[-1, 0], gap, -1)
    turn = _arc(s1[-1], s2[0], 4, 3.8, np.array([1.0, 0.0, 0.0]))
    s3 = strand(10, s2[-1, 0] + 0.0, 2 * gap, +1)
    loop = _arc(s2[-1], s3[0], 6, 3.8, np.array([-1.0, 0.0, 0.6]))
    ca1 = np.vstack([s1, turn, s2, loop, s3])
    # chain 2: strand parallel to s1 on the other side, plus a short tail
    s4 = strand(12, 0.0, -gap, +1)
    # chain 3: a strand antiparallel to s3 beyond it
    s5 = strand(10, s3[-1, 0], 3 * gap, -1)
    for ca in (ca1, s4, s5):
        L = len(ca)
        seq = "".join(AA[k] for k in rng.integers(0, 20, size=L))
        seq = seq.replace("P", "V")  # keep prolines out of the sheet
        cb, o = place_beads(ca, seq)
        cb = _chi_sign_fix(ca, cb, o, seq)
        ss = "".join("E" for _ in range(L))
        ch = Chain(seq=seq, ca=ca, cb=cb, o=o, ss=ss)
        build_memories(ch, rng)
        chains.append(ch)
    s = System(chains=chains, box=200.0, temperature=T, seed=seed)
    _, types, _, _ = atom_arrays(s)
    s.velocities = maxwell_velocities(types, T, rng)
    return s


# --------------------------------------------------------------------------
# array form of a chain (no files): what the batched engine takes for the
# 1,024-replica and served workloads

def chain_arrays(L: int, seed: int, n_mem_per_window=MEMS_PER_WINDOW, win=WINDOW, sigma=1.0, T=300.0) -> dict:
    """One chain built as in configuration 0 from its own seed, returned as
    the arrays of an awsem_replica_desc (atoms in data-file order CA, O, CB)."""
    rng = np.random.default_rng(seed)
    seq = "".join(AA[k] for k in rng.integers(0, 20, size=L))
    ca = ca_trace(L, rng)
    cb, o = place_beads(ca, seq)
    cb = _chi_sign_fix(ca, cb, o, seq)
    com = ca.mean(axis=0)
    ca, cb, o = ca - com, cb - com, o - com
    ss = ss_segments(L, rng)
    x = np.stack([ca, o, cb], axis=1)  # [L][CA, O, CB][3]
    types = np.array([[1, 3, 5 if s == "G" else 4] for s in seq]).reshape(-1)
    v = maxwell_velocities(types, T, rng).reshape(L, 3, 3)
    ssw = np.array([{"H": (1.0, 0.0), "E": (0.0, 1.0), "C": (0.0, 0.0)}[s] for s in ss])
    W = max(L - win + 1, 0)
    idx = np.arange(W)[:, None] + np.arange(win)[None, :]            # [W][win]
    noise_ca = rng.normal(0.0, sigma, size=(W, n_mem_per_window, win, 3))
    noise_cb = rng.normal(0.0, sigma, size=(W, n_mem_per_window, win, 3))
    mem_ca = ca[idx][:, None, :, :] + noise_ca                        # [W][m][win][3]
    mem_cb = cb[idx][:, None, :, :] + noise_cb
    # the .gro precision (nm, 5 decimals)
    mem_ca = np.round(mem_ca / 10.0, 5) * 10.0
    mem_cb = np.round(mem_cb / 10.0, 5) * 10.0
    n_mem = W * n_mem_per_window
    seq_b = np.frombuffer(seq.encode(), dtype=np.uint8)
    mem_seq = np.repeat(seq_b[idx][:, None, :], n_mem_per_window, axis=1).reshape(-1)
    return {
        "n_res": L, "chain_len": np.array([L], dtype=np.int32), "seq": seq.encode(),
        "ssweight": np.ascontiguousarray(ssw, dtype=np.float64),
        "x": np.ascontiguousarray(x, dtype=np.float64), "v": np.ascontiguousarray(v, dtype=np.float64),
        "n_mem": n_mem, "mem_pos": np.repeat(np.arange(W, dtype=np.int32), n_mem_per_window),
        "mem_len": np.full(n_mem, win, dtype=np.int32), "mem_weight": np.ones(n_mem),
        "mem_seq": mem_seq.tobytes(),
        "mem_ca": np.ascontiguousarray(mem_ca.reshape(-1, 3)), "mem_cb": np.ascontiguousarray(mem_cb.reshape(-1, 3)),
    }


def forcefield_dir(outdir: str) -> dict:
    """A run directory holding only the shared force field (default
    parameters + fragment memory with uniform.gamma)."""
    os.makedirs(outdir, exist_ok=True)
    for t in PARAM_TABLES:
        shutil.copy(os.path.join(PARAM_DIR, t), os.path.join(outdir, t))
    with open(os.path.join(outdir, "fix_backbone_coeff.data"), "w") as f:
        f.write(coeff_text(mem_file="none.mem"))
    return {"workdir": outdir, "coeff": "fix_backbone_coeff.data", "pair_style": PAIR_STYLE,
            "pair_coeffs": ";".join(PAIR_COEFFS)}


def write_chain_arrays(c: dict, outdir: str) -> dict:
    """The run directory (reference input formats) of a chain given in array
    form, e.g. to check the array path against the file path or the oracle."""
    os.makedirs(outdir, exist_ok=True)
    L = int(c["n_res"])
    seq = c["seq"].decode()
    x = c["x"].reshape(L * 3, 3)
    v = c["v"].reshape(L * 3, 3)
    clen = [int(n) for n in c["chain_len"]]
    mol = np.repeat(np.arange(1, len(clen) + 1), clen)
    last = set(np.cumsum(clen) - 1)
    lines = ["LAMMPS data file (synthetic AWSEM chain)", "", f"{3 * L} atoms", f"{4 * L - 2 * len(clen)} bonds",
             "5 atom types", "5 bond types", "", "-500.0 500.0 xlo xhi", "-500.0 500.0 ylo yhi",
             "-500.0 500.0 zlo zhi", "", "Masses", ""]
    lines += [f"{t} {MASSES[t]}" for t in range(1, 6)]
    lines += ["", "Atoms", ""]
    for r in range(L):
        for k, t in enumerate([1, 3, 5 if seq[r] == "G" else 4]):
            a = 3 * r + k
            lines.append(f"{a + 1} {mol[r]} {r + 1} {t} 0.0 {float(x[a, 0])!r} {float(x[a, 1])!r} "
                         f"{float(x[a, 2])!r}")
    lines += ["", "Velocities", ""]
    for a in range(3 * L):
        lines.append(f"{a + 1} {float(v[a, 0])!r} {float(v[a, 1])!r} {float(v[a, 2])!r}")
    lines += ["", "Bond Coeffs", ""] + [f"{t} {BOND_COEFFS[t][0]} {BOND_COEFFS[t][1]}" for t in range(1, 6)]
    lines += ["", "Bonds", ""]
    b = 0
    for r in range(L):
        pairs = [(2, 3 * r, 3 * r + 1), (5 if seq[r] == "G" else 4, 3 * r, 3 * r + 2)]
        if r not in last:
            pairs += [(1, 3 * r, 3 * r + 3), (3, 3 * r + 1, 3 * r + 3)]
        for t, i, j in pairs:
            b += 1
            lines.append(f"{b} {t} {i + 1} {j + 1}")
    with open(os.path.join(outdir, "data.awsem"), "w") as f:
        f.write("\n".join(lines) + "\n")
    with open(os.path.join(outdir, "protein.seq"), "w") as f:
        starts = np.concatenate([[0], np.cumsum(clen)])
        f.write("\n".join(seq[starts[k]:starts[k + 1]] for k in range(len(clen))) + "\n")
    with open(os.path.join(outdir, "ssweight"), "w") as f:
        for row in c["ssweight"]:
            f.write(f"{float(row[0])!r} {float(row[1])!r}\n")
    for t in PARAM_TABLES:
        shutil.copy(os.path.join(PARAM_DIR, t), os.path.join(outdir, t))
    with open(os.path.join(outdir, "fix_backbone_coeff.data"), "w") as f:
        f.write(coeff_text())
    # memories: one .gro per memory window group, coordinates written so
    # that float(text) * 10 reproduces the array values to the last bits
    # memories starting at the same residue share one .gro file (stacked)
    os.makedirs(os.path.join(outdir, "mems"), exist_ok=True)
    mem_lines = ["[Target]", "query", "", "[Memories]"]
    off = 0
    mseq = c["mem_seq"].decode()
    groups = {}
    for m in range(int(c["n_mem"])):
        n = int(c["mem_len"][m])
        groups.setdefault(int(c["mem_pos"][m]), []).append((m, off, n))
        off += n
    for pos, members in groups.items():
        fname = f"mems/p{pos:05d}.gro"
        rows = []
        atom = 0
        base = 0
        for m, off, n in members:
            for r in range(n):
                rn = THREE[mseq[off + r]]
                atom += 1
                p = c["mem_ca"][off + r]
                rows.append(f"{base + r + 1} {rn} CA {atom} " + " ".join(repr(float(q) / 10.0) for q in p))
                if mseq[off + r] != "G":
                    atom += 1
                    p = c["mem_cb"][off + r]
                    rows.append(f"{base + r + 1} {rn} CB {atom} " + " ".join(repr(float(q) / 10.0) for q in p))
            mem_lines.append(f"{fname} {pos + 1} {base + 1} {n} {float(c['mem_weight'][m])!r}")
            base += n
        with open(os.path.join(outdir, fname), "w") as f:
            f.write(f"memories at residue {pos + 1}\n{len(rows)}\n" + "\n".join(rows) + "\n0 0 0\n")
    with open(os.path.join(outdir, "frags.mem"), "w") as f:
        f.write("\n".join(mem_lines) + "\n")
    return {"workdir": outdir, "data": "data.awsem", "coeff": "fix_backbone_coeff.data", "seq": "protein.seq",
            "pair_style": PAIR_STYLE, "pair_coeffs": ";".join(PAIR_COEFFS)}


def packed_arrays(chain_lengths, box: float, seed: int, n_mem_per_window=MEMS_PER_WINDOW, min_dist=4.0,
                  tries=5000) -> dict:
    """One system of several chains, each built as in configuration 0 (see
    chain_arrays, chain k from seed * 100003 + k), placed by a random rotation
    and a translation uniform in the box with rejection of any inter-chain CA
    pair closer than min_dist; returned as the arrays of one awsem_replica_desc.
    Memories are internal distances, unchanged by the placement."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    parts, placed = [], np.zeros((0, 3))
    for k, L in enumerate(chain_lengths):
        c = chain_arrays(int(L), seed * 100003 + k, n_mem_per_window=n_mem_per_window)
        x = c["x"].reshape(-1, 3)
        ca = c["x"][:, 0, :]
        tree = cKDTree(placed) if len(placed) else None
        for _ in range(tries):
            R = _random_rotation(rng)
            shift = rng.uniform(-box / 2, box / 2, size=3)
            new_ca = ca @ R.T + shift
            if tree is None or tree.query(new_ca, k=1, distance_upper_bound=min_dist)[0].min() >= min_dist:
                break
        else:
            raise RuntimeError("could not place chain without overlap")
        c["x"] = np.ascontiguousarray((x @ R.T + shift).reshape(-1, 3, 3))
        c["v"] = np.ascontiguousarray((c["v"].reshape(-1, 3) @ R.T).reshape(-1, 3, 3))
        placed = np.vstack([placed, new_ca])
        parts.append(c)
    offs = np.cumsum([0] + [p["n_res"] for p in parts])
    return {
        "n_res": int(offs[-1]), "chain_len": np.array([p["n_res"] for p in parts], dtype=np.int32),
        "seq": b"".join(p["seq"] for p in parts),
        "ssweight": np.ascontiguousarray(np.concatenate([p["ssweight"] for p in parts])),
        "x": np.ascontiguousarray(np.concatenate([p["x"] for p in parts])),
        "v": np.ascontiguousarray(np.concatenate([p["v"] for p in parts])),
        "n_mem": int(sum(p["n_mem"] for p in parts)),
        "mem_pos": np.concatenate([p["mem_pos"] + o for p, o in zip(parts, offs)]).astype(np.int32),
        "mem_len": np.concatenate([p["mem_len"] for p in parts]).astype(np.int32),
        "mem_weight": np.concatenate([p["mem_weight"] for p in parts]),
        "mem_seq": b"".join(p["mem_seq"] for p in parts),
        "mem_ca": np.ascontiguousarray(np.concatenate([p["mem_ca"] for p in parts])),
        "mem_cb": np.ascontiguousarray(np.concatenate([p["mem_cb"] for p in parts])),
    }
