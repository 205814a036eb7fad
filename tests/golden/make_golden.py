"""Regenerate the golden vectors of tests/golden/*.npz from the reference.

The reference FixBackbone / PairExcludedVolume sources are compiled in place
against the LAMMPS-API shim (``make -C oracle ref``) and run on four inputs:

* ``c0``    -- the 100-residue random-coil chain of benchmark configuration 0
               (generated by awsemmd_b200.synth, seed 0);
* ``sheet`` -- a three-chain beta-sheet system that exercises the hydrogen-
               bond, P_AP and burial branches (synth.sheet_system, seed 7);
* ``r1r69`` -- the reference's own 1R69 example inputs (63 residues, native
               coordinates, one 63-residue fragment memory), copied verbatim
               into tests/golden/r1r69 from
               examples/examples_new/1R69_single_memory, with the default
               parameter set plus a [Fragment_Memory] section;
* ``r1r69tb`` -- the same inputs with fragment memory in its table form
               ([Fragment_Memory_Table] with that example's settings: k 0.2,
               grid 0-50 A by 0.01 A, well width 0.1, sigma exponent 0.15);
* ``r1r69go`` -- the r1r69 inputs plus an [AMH-Go] section with the settings
               of the reference's 1R69_AMH-Go example (k 1, p 1, rc 8 A,
               no censoring) and that example's amh-go.gro native structure
               and amh-go.gamma, copied verbatim into tests/golden/r1r69go
               from examples/examples_new/1R69_AMH-Go;
* ``r1r69go2`` -- the same with k 1.5, p 2, rc 9 A and censoring 1 (four
               native residue pairs listed in frustration_censored_contacts.dat);
* ``c0x``     -- ``c0`` with [Solvent_Barrier], [DebyeHuckel] (charges +1 on
               K/R, -1 on D/E) and [Contact_Restraints] (synth.pair_terms_text,
               write_charges, write_contact_restraints), run with neighbor 0.6
               and neigh_modify delay 3 every 2: the barrier and Debye-Hueckel
               sum over the CA pairs of the fix's half list as last built;
* ``sheetx``  -- ``sheet`` (three chains) with the same three sections;
* ``c0s``     -- ``c0`` with [Shake], [Membrane] (zones from a seeded zim)
               and [Phosphorylation] of two serines and one other residue
               (synth.residue_terms_text, write_zim);
* ``sheets``  -- ``sheet`` with the same sections, its serines phosphorylated
               (water contacts of phosphorylated residues);
* ``c0v``     -- ``c0`` with [Vector_Fragment_Memory] (k 1, sigma 0.3 rad)
               over its fragment memories;
* ``c1``      -- benchmark configuration 1: 8 chains x 250 residues (2,000
               residues) at seeded non-overlapping positions in a 150 A cube
               (synth.config_system(1)), all terms of the default parameter
               set plus fragment memory;
* ``c0go``    -- ``c0`` with [AMH-Go] (k 200, p 2, rc 10 A) towards a native
               structure 0.6 times as large as the starting chain
               (synth.write_native_gro), run with neighbor skin 0.6 A and
               neigh_modify delay 3 every 2 check yes: the fix's full list is
               rebuilt during the run and native contacts cross its reach, so
               the trajectory depends on LAMMPS's rebuild rule.

``q_r1r69.npz`` and ``q_c0.npz`` hold the reference's Q order parameters
(compute qwolynes, compute qonuchic in its four types; Q_DEFS) at the start
and the end of the 20-step run, with the inputs of synth.write_q_files: the
native CA trace of r1r69 is its own (crystal) coordinates, that of c0 its
chain shrunk to 0.8 times its size.

For each it stores the inputs' hash, the step-0 forces and energies, the
per-residue pair-pass intermediates and a 20-step Langevin trajectory
(x, v and per-step thermo rows).  ``c0_nve.npz`` holds the thermo rows of a
1,000-step constant-energy run (fix nve only, dt 2 fs) of ``c0``: the energy
drift of the reference.  Run from the repository root with the reference tree
present:  python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import hashlib
import os
import shutil
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from awsemmd_b200 import synth  # noqa: E402

GOLDEN = os.path.dirname(os.path.abspath(__file__))
RUN = dict(nsteps=20, dt=2.0, t_start=300.0, t_stop=300.0, damp=500.0, seed=12345)
NVE = dict(nsteps=1000, dt=2.0)


def dir_hash(d: str) -> str:
    h = hashlib.sha256()
    for root, _, files in sorted(os.walk(d)):
        for f in sorted(files):
            if f in ("energy.log", "timer.log"):
                continue
            p = os.path.join(root, f)
            h.update(os.path.relpath(p, d).encode())
            with open(p, "rb") as fh:
                h.update(fh.read())
    return h.hexdigest()


def write_case(name: str, outdir: str) -> dict:
    if name == "c0":
        return synth.write_system(synth.config_system(0), outdir)
    if name == "c1":
        return synth.write_system(synth.config_system(1), outdir)
    if name in ("c0x", "sheetx"):
        sys_ = synth.config_system(0) if name == "c0x" else synth.sheet_system()
        files = synth.write_system(sys_, outdir)
        with open(os.path.join(outdir, files["coeff"]), "w") as fh:
            fh.write(synth.coeff_text() + synth.pair_terms_text())
        synth.write_charges(sys_, os.path.join(outdir, "charge_on_residues.dat"))
        synth.write_contact_restraints(sys_, os.path.join(outdir, "contact_restraints.dat"))
        return files
    if name in ("c0s", "sheets"):
        sys_ = synth.config_system(0) if name == "c0s" else synth.sheet_system()
        files = synth.write_system(sys_, outdir)
        seq = "".join(ch.seq for ch in sys_.chains)
        if name == "c0s":
            phosph = [k + 1 for k, a in enumerate(seq) if a == "S"][:2] + [next(k + 1 for k, a in enumerate(seq) if a not in "SG")]
        else:
            phosph = ([k + 1 for k, a in enumerate(seq) if a == "S"] + [k + 1 for k, a in enumerate(seq) if a == "T"])[:20]
        with open(os.path.join(outdir, files["coeff"]), "w") as fh:
            fh.write(synth.coeff_text() + synth.residue_terms_text(sys_, phosph))
        synth.write_zim(sys_, os.path.join(outdir, "zim"))
        return files
    if name == "c0v":
        files = synth.write_system(synth.config_system(0), outdir)
        with open(os.path.join(outdir, files["coeff"]), "a") as fh:
            fh.write("\n[Vector_Fragment_Memory]\n1.0\n0.3\n")
        return files
    if name == "c0go":
        sys_ = synth.config_system(0)
        files = synth.write_system(sys_, outdir)
        with open(os.path.join(outdir, files["coeff"]), "w") as fh:
            fh.write(synth.coeff_text(amh_go=(200.0, 2, 10.0, 0)))
        synth.write_native_gro(sys_, os.path.join(outdir, "amh-go.gro"), scale=0.6)
        shutil.copy(os.path.join(GOLDEN, "r1r69go", "amh-go.gamma"), os.path.join(outdir, "amh-go.gamma"))
        os.chmod(os.path.join(outdir, "amh-go.gamma"), 0o644)
        return files
    if name == "sheet":
        return synth.write_system(synth.sheet_system(), outdir)
    if name in ("r1r69", "r1r69tb", "r1r69go", "r1r69go2"):
        os.makedirs(outdir, exist_ok=True)
        for d in ("r1r69", "r1r69go") if name.startswith("r1r69go") else ("r1r69",):
            src = os.path.join(GOLDEN, d)
            for f in os.listdir(src):
                shutil.copy(os.path.join(src, f), os.path.join(outdir, f))
                os.chmod(os.path.join(outdir, f), 0o644)
        for t in synth.PARAM_TABLES:
            shutil.copy(os.path.join(synth.PARAM_DIR, t), os.path.join(outdir, t))
        with open(os.path.join(outdir, "fix_backbone_coeff.data"), "w") as fh:
            if name == "r1r69":
                fh.write(synth.coeff_text(mem_file="fragsLAMW.mem.single", gamma_file="seq.gamma"))
            elif name == "r1r69go":
                fh.write(synth.coeff_text(mem_file="fragsLAMW.mem.single", gamma_file="seq.gamma",
                                          amh_go=(1.0, 1, 8.0, 0)))
            elif name == "r1r69go2":
                fh.write(synth.coeff_text(mem_file="fragsLAMW.mem.single", gamma_file="seq.gamma",
                                          amh_go=(1.5, 2, 9.0, 1)))
                with open(os.path.join(outdir, "frustration_censored_contacts.dat"), "w") as cf:
                    cf.write("3 35\n26 21\n33 39\n49 56\n")
            else:  # the table form and settings of the reference's 1R69 example coefficient file
                fh.write(synth.coeff_text(k_fm=0.2, mem_file="fragsLAMW.mem.single", gamma_file="seq.gamma",
                                          table=(0, 50, 0.01, 0.1, 0, 0.15)))
        return {"workdir": outdir, "data": "data.1r69", "coeff": "fix_backbone_coeff.data", "seq": "extended.seq",
                "pair_style": synth.PAIR_STYLE, "pair_coeffs": ";".join(synth.PAIR_COEFFS)}
    raise KeyError(name)


CASES = ["c0", "sheet", "r1r69", "r1r69tb", "r1r69go", "r1r69go2", "c0go", "c0x", "sheetx", "c0s", "sheets", "c0v",
         "c1"]
# LAMMPS neighbor skin and neigh_modify delay / every / check of a case's runs
# (the others: 2.0, 0, 1, yes -- LAMMPS's defaults)
NEIGH = {"c0go": (0.6, 3, 2, 1), "c0x": (0.6, 3, 2, 1)}


Q_DEFS = [
    "q1 alpha_carbons qwolynes rnative.dat 2 0.15",
    "q2 alpha_carbons qwolynes rnative.dat 3 0.3",
    "q3 alpha_carbons qonuchic cutoff 9.5 native_ca.dat 1.2",
    "q4 alpha_carbons qonuchic cutoff/gauss 9.5 native_ca.dat",
    "q5 alpha_carbons qonuchic shadow shadow.dat 1.2",
    "q6 alpha_carbons qonuchic shadow/gauss shadow.dat",
]
Q_CASES = ["r1r69", "c0"]


def write_q_case(name: str, outdir: str) -> dict:
    """A case's inputs plus the Q inputs (synth.write_q_files) of its native CA trace."""
    files = write_case(name, outdir)
    x0 = read_data_x(os.path.join(outdir, files["data"]))
    ca = x0[::3]  # data files list CA, O, CB per residue
    if name == "c0":
        ca = ca.mean(axis=0) + 0.8 * (ca - ca.mean(axis=0))
    synth.write_q_files(ca, outdir)
    return files


def read_data_x(path: str) -> np.ndarray:
    """Atom coordinates of a data file in atom-id order."""
    lines = open(path).read().splitlines()
    k = next(i for i, l in enumerate(lines) if l.strip().startswith("Atoms"))
    rows = {}
    for l in lines[k + 1:]:
        t = l.split()
        if not t:
            if rows:
                break
            continue
        rows[int(t[0])] = [float(v) for v in t[5:8]]
    return np.array([rows[i] for i in sorted(rows)])


def main_q(cases=None):
    import ref

    for name in cases or Q_CASES:
        with tempfile.TemporaryDirectory() as tmp:
            files = write_q_case(name, os.path.join(tmp, name))
            h = dir_hash(files["workdir"])
            r = ref.RefSystem(files)
            q0 = [r.compute_q(w) for w in Q_DEFS]
            r.run(RUN["nsteps"], dt=RUN["dt"], langevin=True, t_start=RUN["t_start"], t_stop=RUN["t_stop"],
                  damp=RUN["damp"], seed=RUN["seed"])
            qN = [r.compute_q(w) for w in Q_DEFS]
            xN = r.get("x")
            r.close()
            np.savez_compressed(os.path.join(GOLDEN, f"q_{name}.npz"), inputs_sha256=np.array(h),
                                words=np.array(Q_DEFS), q0=np.array(q0), qN=np.array(qN), xN=xN)
            print("q", name, np.round(q0, 4), np.round(qN, 4))


def main(cases=None):
    import ref

    for name in cases or CASES:
        with tempfile.TemporaryDirectory() as tmp:
            files = write_case(name, os.path.join(tmp, name))
            h = dir_hash(files["workdir"])
            skin, delay, every, check = NEIGH.get(name, (2.0, 0, 1, 1))
            r = ref.RefSystem(files, skin=skin, every=every, delay=delay, check=check)
            x0, v0 = r.get("x"), r.get("v")
            f0 = r.compute(0)
            e0 = r.energies()
            nres = int(open(os.path.join(files["workdir"], files["seq"])).read().replace("\n", "").__len__())
            res0 = r.residue_arrays(nres)
            thermo = r.run(RUN["nsteps"], dt=RUN["dt"], langevin=True, t_start=RUN["t_start"], t_stop=RUN["t_stop"],
                           damp=RUN["damp"], seed=RUN["seed"])
            xN, vN = r.get("x"), r.get("v")
            builds = r.nbuilds()
            r.close()
            np.savez_compressed(os.path.join(GOLDEN, f"{name}.npz"), inputs_sha256=np.array(h), x0=x0, v0=v0,
                                f0=f0, e0=e0, res0=res0, thermo=thermo, xN=xN, vN=vN,
                                run=np.array([RUN["nsteps"], RUN["dt"], RUN["t_start"], RUN["t_stop"], RUN["damp"],
                                              RUN["seed"]], dtype=np.float64),
                                neigh=np.array([skin, delay, every, check], dtype=np.float64))
            print(name, "natoms", len(x0), "E_total", e0[0], "list builds", builds, "hash", h[:12])
            if name == "c0":
                r = ref.RefSystem(files)
                rows = r.run(NVE["nsteps"], dt=NVE["dt"], langevin=False)
                r.close()
                np.savez_compressed(os.path.join(GOLDEN, "c0_nve.npz"), inputs_sha256=np.array(h), thermo=rows,
                                    run=np.array([NVE["nsteps"], NVE["dt"]], dtype=np.float64))
                e = rows.sum(axis=1)
                print("c0 nve: max |E(t) - E(0)| over", NVE["nsteps"], "steps:", np.abs(e - e[0]).max())


if __name__ == "__main__":
    args = sys.argv[1:]
    if args and args[0] == "q":
        main_q(args[1:] or None)
    else:
        main(args or None)
