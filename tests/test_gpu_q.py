"""Q order parameters on the GPU (awsem_q_create / awsem_q_value) against the
reference's compute qwolynes and compute qonuchic (compiled in the shim; the
golden values of tests/golden/q_*.npz) at the start and the end of the
20-step run, and on a replica inside a batch."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _case(name, tmp_path):
    import make_golden

    files = make_golden.write_q_case(name, str(tmp_path / name))
    g = np.load(os.path.join(GOLDEN, f"q_{name}.npz"))
    assert make_golden.dir_hash(files["workdir"]) == str(g["inputs_sha256"])
    x0 = np.load(os.path.join(GOLDEN, f"{name}.npz"))["x0"]
    return files, g, x0


@pytest.mark.parametrize("name", ["r1r69", "c0"])
def test_q_matches_reference(name, tmp_path, gpu_lib):
    from awsemmd_b200.engine import AwsemSystem

    files, g, x0 = _case(name, tmp_path)
    cwd = os.getcwd()
    os.chdir(files["workdir"])
    try:
        with AwsemSystem(files, precision="fp64") as s:
            qids = [s.q_create(str(w)) for w in g["words"]]
            for x, want in ((x0, g["q0"]), (g["xN"], g["qN"])):
                s.set_state(x, np.zeros_like(x))
                got = np.array([s.q_value(q) for q in qids])
                np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-14)
    finally:
        os.chdir(cwd)


def test_q_of_a_replica_in_a_batch(tmp_path, gpu_lib):
    """Two r1r69 replicas at the start and at the end of the run: each Q
    definition reads its own replica's positions."""
    from awsemmd_b200.engine import AwsemBatch

    f1, g1, x1 = _case("r1r69", tmp_path)
    with AwsemBatch([f1, f1], precision="mixed") as b:
        b.set_state(g1["xN"], np.zeros_like(x1), r=0)
        b.set_state(x1, np.zeros_like(x1), r=1)
        for k, w in enumerate(g1["words"]):
            words = " ".join(os.path.join(f1["workdir"], t) if t.endswith(".dat") else t for t in str(w).split())
            for rep, want in ((0, g1["qN"][k]), (1, g1["q0"][k])):
                q = b.q_create(words, rep=rep)
                assert abs(b.q_value(q) - want) <= 1e-12, (rep, str(w))


def test_q_errors(tmp_path, gpu_lib):
    from awsemmd_b200.engine import AwsemError, AwsemSystem

    files, g, x0 = _case("c0", tmp_path)
    wd = files["workdir"]
    with AwsemSystem(files, precision="fp64") as s:
        for words, msg in [("q alpha_carbons qwolynes x.dat 2", "Illegal compute qwolynes command"),
                           (f"q alpha_carbons qwolynes {wd}/missing.dat 2 0.15", "Native distance file can't be read"),
                           ("q alpha_carbons qonuchic ring 9.5 x.dat 1.2", "Wrong type for compute qonuchic"),
                           (f"q alpha_carbons qonuchic cutoff 9.5 {wd}/rnative.dat 1.2", "atom number mismatch")]:
            with pytest.raises(AwsemError, match=msg):
                s.q_create(words)
