"""awsem_fragmem_noalloc: the fragment-memory entry point that allocates nothing.

It exists for callers that cannot call cudaMalloc when forces are needed
(a host code owning all device memory through its own pool, a step being
recorded into a CUDA graph, an allocation-free real-time loop): they hand in
device buffers, and the force accumulator lives in a fixed __device__ array.
Checked through the C ABI against the existing entry point, awsem_compute,
on a handle whose only term is fragment memory, over two calls in a row.
Collected last so that a failing run stops after every other test ran.
"""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def fm_only_case(tmp_path, weights="uniform"):
    from awsemmd_b200 import synth

    s = synth.make_system([90], box=200.0, seed=515)
    files = synth.write_system(s, str(tmp_path / "fm_only"))
    # a coefficient file whose only term is fragment memory
    with open(os.path.join(files["workdir"], files["coeff"]), "w") as f:
        f.write("[Epsilon]\n1.0\n\n[Fragment_Memory]\n1.0\nfrags.mem\nuniform.gamma\n")
    if weights == "varied":
        # memory weights 0.5, 0.75, 1.0, ...: every record carries its own
        # coefficient (the per-record path of the kernel)
        path = os.path.join(files["workdir"], "frags.mem")
        lines = open(path).read().split("\n")
        k = lines.index("[Memories]") + 1
        for m in range(k, len(lines)):
            t = lines[m].split()
            if len(t) == 5:
                t[4] = repr(0.5 + 0.25 * ((m - k) % 4))
                lines[m] = " ".join(t)
        open(path, "w").write("\n".join(lines))
    return files


@pytest.mark.parametrize("weights", ["uniform", "varied"])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("mixed", 1e-12)])
def test_noalloc_matches_existing_entry_point(prec, tol, weights, tmp_path, gpu_lib):
    import torch

    from awsemmd_b200.engine import TERMS_FIX, AwsemSystem

    lib = gpu_lib
    lib.awsem_fragmem_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    files = fm_only_case(tmp_path, weights)
    with AwsemSystem(files, precision=prec) as s:
        x_ext, _ = s.get_state()
        nat = s.natoms
        # internal order: per residue CA, CB, O (the data file lists CA, O, CB)
        order = np.arange(nat).reshape(-1, 3)[:, [0, 2, 1]].reshape(-1)
        x_int = np.ascontiguousarray(x_ext[order])
        d_x = torch.tensor(x_int, dtype=torch.float64, device="cuda")
        d_f = torch.full((nat, 3), 7.0, dtype=torch.float64, device="cuda")  # stale contents must not leak
        d_e = torch.full((1,), 3.0, dtype=torch.float64, device="cuda")
        for call in range(2):
            f_ref, e_ref = s.compute(x_ext, terms=TERMS_FIX)
            rc = lib.awsem_fragmem_noalloc(s.h, d_x.data_ptr(), d_f.data_ptr(), d_e.data_ptr(), None)
            assert rc == 0, lib.awsem_last_error()
            torch.cuda.synchronize()
            f_new = np.empty_like(f_ref)
            f_new[order] = d_f.cpu().numpy()
            assert np.abs(f_new - f_ref).max() <= tol * np.abs(f_ref).max(), call
            assert abs(float(d_e.item()) - e_ref[12]) <= 1e-9 * abs(e_ref[12]), call
            assert abs(e_ref[12]) > 1.0


def test_noalloc_rejects_handles_beyond_its_scratch(tmp_path, gpu_lib):
    """8,500 residues (25,500 atoms) exceed the 24,576-atom scratch: a clear
    error before any device work (the tiny buffers are never touched)."""
    import torch

    from awsemmd_b200 import synth
    from awsemmd_b200.engine import AwsemBatch

    lib = gpu_lib
    lib.awsem_fragmem_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    ff = synth.forcefield_dir(str(tmp_path / "ff"))
    chains = [synth.chain_arrays(500, seed=900 + k, n_mem_per_window=1) for k in range(17)]
    with AwsemBatch.from_arrays(ff, chains, precision="mixed") as b:
        assert b.natoms == 25500
        tiny = torch.zeros(4, dtype=torch.float64, device="cuda")
        rc = lib.awsem_fragmem_noalloc(b.h, tiny.data_ptr(), tiny.data_ptr(), tiny.data_ptr(), None)
        assert rc == -1
        assert b"exceed" in lib.awsem_last_error()
