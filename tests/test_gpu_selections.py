"""Discrete decisions of the GPU pair passes against the oracle's.

The plain FP64 form must take the reference's selections bit for bit:
density-well windows, water wells, xi and helix-force gates, helical
(i, i+4) pairs, DSSP candidates and their gates, P_AP pairs and classes,
and excluded-volume bead pairs (AWSEM_SEL_* records of
awsem_debug_selections, include/awsem_gpu.h).  The oracle's selections are
pinned to the compiled reference's own cache entries by
tests/test_selections.py.  The mixed form may decide a distance predicate
differently only within 2e-6 (relative) of its threshold; its differences
are counted and reported.
"""
import json

import numpy as np
import pytest

from conftest import neigh_of, write_case

pytestmark = pytest.mark.gpu

CASES = ["c0", "sheet", "r1r69", "r1r69tb", "r1r69go", "r1r69go2", "c0go", "c0x", "sheetx", "c0s", "sheets", "c0v"]


def assert_identical(got, want):
    import ref

    if not np.array_equal(got, want):
        raise AssertionError(json.dumps({k: v for k, v in ref.compare_selections(got, want).items()
                                         if v["cand"] or v["gate"]}))


@pytest.mark.parametrize("name", CASES)
def test_fp64_selections_are_the_oracles(name, tmp_path, gpu_lib, oracle_built):
    import ref
    from awsemmd_b200.engine import AwsemSystem

    files, g = write_case(name, tmp_path)
    o = ref.OracleSystem(files)
    o.set_neighbor(*neigh_of(g))
    want = o.selections(g["x0"])
    with AwsemSystem(files, precision="fp64") as s:
        s.set_neighbor(*neigh_of(g))
        got = s.selections(g["x0"])
    assert len(want) > 100
    assert_identical(got, want)


@pytest.mark.parametrize("case", ["c0", "c1"])
def test_fp64_selections_after_motion(case, tmp_path, gpu_lib, oracle_built):
    """Starting coordinates and after 200 Langevin steps (the pair list
    rebuilt on the way) of the 100-residue chain and of configuration 1
    (8 x 250 residues)."""
    import ref
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemSystem

    files = synth.write_system(synth.config_system(0 if case == "c0" else 1), str(tmp_path / case))
    o = ref.OracleSystem(files)
    with AwsemSystem(files, precision="fp64") as s:
        x0, _ = s.get_state()
        assert_identical(s.selections(x0), o.selections(x0))
        s.run(200, dt=2.0, langevin=True, seed=11, skin=1.0)
        assert s.neighbor_stats()["builds"] >= 2
        x, _ = s.get_state()
        assert_identical(s.selections(x, step=s.step), o.selections(x))


@pytest.mark.parametrize("case", ["c0", "sheet", "r1r69", "c1"])
def test_mixed_selections_differ_only_near_thresholds(case, tmp_path, gpu_lib, oracle_built):
    import ref
    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemSystem

    if case == "c1":
        files = synth.write_system(synth.config_system(1), str(tmp_path / case))
        x = None
    else:
        files, g = write_case(case, tmp_path)
        x = g["x0"]
    o = ref.OracleSystem(files)
    with AwsemSystem(files, precision="mixed") as s:
        if x is None:
            x, _ = s.get_state()
        got = s.selections(x)
    cmp = ref.compare_selections(got, o.selections(x), o.selections(x, "near"))
    print(case, json.dumps(cmp))
    # the densities (and so the density-well windows) are FP64 in both forms
    for k in ("dens_water", "dens_helix"):
        assert cmp[k]["cand"] == 0 and cmp[k]["got"] == cmp[k]["want"], (k, cmp[k])
    # distance predicates in FP32 flip only within 2e-6 of their threshold
    for k, v in cmp.items():
        if k != "xi_force":
            assert v["cand_far"] == 0, (k, v)
