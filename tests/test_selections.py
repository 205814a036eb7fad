"""The oracle's discrete decisions against the compiled reference's own.

The reference caches per residue pair what its pair passes evaluate: cWell
(water and helix wells), cR (r_NO, r_HO) and cP_AP (nu), each entry tagged
with the timestep that filled it (src/smart_matrix_lib.h:82-652).  After one
reference evaluation, the entries tagged with its timestep are exactly the
well windows, hydrogen-bond candidates and gates, and P_AP pairs the
reference selected (src/fix_backbone.cpp:7728-8135, :2902-3060, :3279-3383,
:3706-3740).  ``RefSystem.touches`` reads them from the reference compiled
unmodified (oracle/ref_host.cpp); the oracle emulates the same entries from
its own selections.  Equal sets pin the oracle's selections to the
reference's, so that the GPU selection test (tests/test_gpu_selections.py),
which compares the GPU with the oracle, reaches the reference.
"""
import os

import numpy as np
import pytest

from conftest import REFERENCE_SRC, neigh_of, write_case

CASES = ["c0", "sheet", "r1r69", "r1r69tb", "r1r69go", "r1r69go2", "c0go", "c0x", "sheetx", "c0s", "sheets", "c0v"]

needs_ref = pytest.mark.skipif(not os.path.isdir(REFERENCE_SRC), reason="reference tree not present")


def kinds(keys):
    return np.bincount((np.asarray(keys, dtype=np.uint64) >> np.uint64(56)).astype(np.int64), minlength=40)


def same_touches(r, o, x):
    tr = r.touches()
    to = o.selections(x, "touch")
    assert len(tr) > 0
    missing, extra = np.setdiff1d(tr, to), np.setdiff1d(to, tr)
    assert len(missing) == 0 and len(extra) == 0, (kinds(missing)[32:37], kinds(extra)[32:37])
    return tr


@needs_ref
@pytest.mark.parametrize("name", CASES)
def test_oracle_selections_match_reference_caches(name, tmp_path, oracle_built):
    import ref

    files, g = write_case(name, tmp_path)
    skin, delay, every, check = neigh_of(g)
    r = ref.RefSystem(files, skin=skin, every=every, delay=delay, check=check)
    x0 = r.get("x")
    r.compute(0)
    o = ref.OracleSystem(files)
    o.set_neighbor(skin, delay, every, check)
    t = same_touches(r, o, x0)
    # every cache the fixtures can exercise is exercised
    k = kinds(t)
    assert k[32] > 0 and k[33] > 0 and k[34] > 0 and k[35] > 0 and k[36] > 0


@needs_ref
def test_oracle_selections_match_reference_caches_config1(tmp_path, oracle_built):
    """Configuration 1 (8 x 250 residues, inter-chain contacts) at its
    starting coordinates and after 200 Langevin steps of the reference."""
    import ref
    from awsemmd_b200 import synth

    files = synth.write_system(synth.config_system(1), str(tmp_path / "c1"))
    r = ref.RefSystem(files)
    o = ref.OracleSystem(files)
    x0 = r.get("x")
    r.compute(0)
    same_touches(r, o, x0)
    r.run(200, dt=2.0, langevin=True, seed=5)
    x = r.get("x")
    r.compute(200)
    same_touches(r, o, x)


def test_selection_records_cover_every_kind(tmp_path, oracle_built):
    """The golden inputs between them produce every selection kind."""
    import ref

    seen = np.zeros(40, dtype=np.int64)
    for name in ["c0", "sheet", "r1r69"]:
        files, g = write_case(name, tmp_path)
        seen += kinds(ref.OracleSystem(files).selections(g["x0"]))
    assert (seen[1:11] > 0).all(), seen[1:11]
