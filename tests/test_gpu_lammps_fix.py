"""`fix backbone/gpu` (awsemmd_b200/lammps) dropped into a LAMMPS host in
place of the reference `fix backbone`: the same host (read_data, pair
vexcluded, bonds, fix nve + langevin, Verlet hook order; the shim-hosted
reference build) runs either fix through the LAMMPS fix hooks, and the
forces, the energy vector and a 20-step trajectory agree."""
import numpy as np
import pytest

from conftest import neigh_of, write_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["c0", "sheet", "r1r69"])
def test_fix_backbone_gpu_replaces_the_reference_fix(name, tmp_path, gpu_lib, oracle_built):
    import ref

    assert ref.gpufix_available(), "oracle/_ref/libawsem_ref_gpufix.so is not built (make -C oracle gpufix)"
    files, g = write_case(name, tmp_path)
    cpu = ref.RefSystem(files)
    gpu = ref.RefSystem(files, gpu_fix="fp64")
    f_cpu, f_gpu = cpu.compute(0), gpu.compute(0)
    e_cpu, e_gpu = cpu.energies(), gpu.energies()
    assert np.abs(f_gpu - f_cpu).max() <= 1e-5 * np.abs(f_cpu).max()
    for k in range(18):
        assert abs(e_gpu[k] - e_cpu[k]) <= 1e-6 * max(abs(e_cpu[k]), 1e-3), (k, e_gpu[k], e_cpu[k])
    t_cpu = cpu.run(20, seed=99)
    t_gpu = gpu.run(20, seed=99)
    np.testing.assert_allclose(t_gpu, t_cpu, rtol=1e-6, atol=1e-6)
    assert np.abs(gpu.get("x") - cpu.get("x")).max() < 1e-6


@pytest.mark.parametrize("name", ["r1r69go", "c0go", "c0x"])
def test_fix_backbone_gpu_follows_the_hosts_list_builds(name, tmp_path, gpu_lib, oracle_built):
    """[AMH-Go], the solvent barrier and Debye-Hueckel read LAMMPS's
    neighbour lists: the adapter tells the engine on which steps the host
    rebuilt them (neighbor->ago == 0), so with neighbor 0.6 / delay 3 /
    every 2 the run matches the reference fix's."""
    import ref

    assert ref.gpufix_available()
    files, g = write_case(name, tmp_path)
    skin, delay, every, check = neigh_of(g)
    kw = dict(skin=skin, every=every, delay=delay, check=check)
    cpu = ref.RefSystem(files, **kw)
    gpu = ref.RefSystem(files, gpu_fix="fp64", **kw)
    nsteps, dt, t0, t1, damp, seed = g["run"]
    run = dict(dt=dt, langevin=True, t_start=t0, t_stop=t1, damp=damp, seed=int(seed))
    t_cpu = cpu.run(int(nsteps), **run)
    t_gpu = gpu.run(int(nsteps), **run)
    assert gpu.nbuilds() == cpu.nbuilds() > 1
    np.testing.assert_allclose(t_gpu, t_cpu, rtol=1e-6, atol=1e-6)
    assert np.abs(gpu.get("x") - cpu.get("x")).max() < 1e-6
    np.testing.assert_allclose(t_cpu, g["thermo"], rtol=1e-9, atol=1e-9)

