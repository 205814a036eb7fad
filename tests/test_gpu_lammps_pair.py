"""`pair_style vexcluded/gpu` (awsemmd_b200/lammps) dropped into a LAMMPS
host in place of the reference `pair_style vexcluded`: the same host
(read_data, the reference fix backbone, bonds, fix nve + langevin, Verlet
hook order; the shim-hosted reference build) runs either pair style through
the LAMMPS pair interface (settings, coeff, init_one mixing, compute), and
the pair energy, the forces and a 20-step trajectory agree.

Tolerances: FP64 form, pair energy 1e-9 relative and total forces 1e-9 of
the largest force (the same pairs and arithmetic as the reference);
trajectories 1e-6 A; mixed form, pair energy 1e-5 and forces 1e-4."""
import numpy as np
import pytest

from conftest import write_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec,etol,ftol", [("fp64", 1e-9, 1e-9), ("mixed", 1e-5, 1e-4)])
@pytest.mark.parametrize("name", ["c0", "sheet", "r1r69"])
def test_pair_vexcluded_gpu_replaces_the_reference_pair(name, prec, etol, ftol, tmp_path, gpu_lib, oracle_built):
    import ref

    assert ref.gpufix_available(), "oracle/_ref/libawsem_ref_gpufix.so is not built (make -C oracle gpufix)"
    files, g = write_case(name, tmp_path)
    cpu = ref.RefSystem(files)
    gpu = ref.RefSystem(files, gpu_pair=prec)
    f_cpu, f_gpu = cpu.compute(0), gpu.compute(0)
    e_cpu, e_gpu = cpu.energies(), gpu.energies()
    assert e_cpu[18] > 1.0
    assert abs(e_gpu[18] - e_cpu[18]) <= etol * abs(e_cpu[18]), (e_gpu[18], e_cpu[18])
    assert np.abs(f_gpu - f_cpu).max() <= ftol * np.abs(f_cpu).max()
    if prec == "fp64":
        t_cpu = cpu.run(20, seed=77)
        t_gpu = gpu.run(20, seed=77)
        np.testing.assert_allclose(t_gpu, t_cpu, rtol=1e-6, atol=1e-6)
        assert np.abs(gpu.get("x") - cpu.get("x")).max() < 1e-6


def test_pair_vexcluded_gpu_mixes_like_the_reference(tmp_path, gpu_lib, oracle_built):
    """Only the diagonal coefficients given: init_one mixes lambda and both
    cutoffs geometrically for the other type pairs, as the reference does."""
    import ref

    files, g = write_case("c0", tmp_path)
    files = dict(files, pair_coeffs="1 1 20.0 3.5 4.5;2 2 0.0 3.5 3.5;3 3 20.0 3.5 3.5;4 4 15.0 3.0 4.0;5 5 5.0 2.0 2.5")
    cpu = ref.RefSystem(files)
    gpu = ref.RefSystem(files, gpu_pair="fp64")
    f_cpu, f_gpu = cpu.compute(0), gpu.compute(0)
    e_cpu, e_gpu = cpu.energies(), gpu.energies()
    assert e_cpu[18] > 0.1
    assert abs(e_gpu[18] - e_cpu[18]) <= 1e-9 * abs(e_cpu[18])
    assert np.abs(f_gpu - f_cpu).max() <= 1e-9 * np.abs(f_cpu).max()
