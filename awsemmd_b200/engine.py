"""Python host API over the C ABI of libawsem_gpu.so (include/awsem_gpu.h).

Mirrors the reference plugin surface for one system:

* construction from a reference-style run directory (``fix backbone``
  coefficient file and tables, sequence, fragment memories, an
  ``atom_style awsemmd`` data file, ``pair_style vexcluded`` settings);
* ``compute`` -- the drop-in force call (FixBackbone::pre_force and
  PairExcludedVolume::compute: forces added into the caller's array, the
  18-term energy vector of the fix plus the pair, bond and kinetic terms);
* ``run`` -- device-resident MD (fix nve + fix langevin) with the step
  captured in CUDA graphs.

There is no CPU fallback: constructing a system without the CUDA library, or
without a GPU, raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libawsem_gpu.so")

FP64 = 0
MIXED = 1
TERMS_FIX, TERMS_PAIR, TERMS_BOND = 1, 2, 4
TERMS_ALL = 7
NKERNELS = 12  # AWSEM_NKERNELS: kernels of one MD step, in launch order

ENERGY_NAMES = ["total", "chain", "shake", "chi", "rama", "excluded", "dssp", "p_ap", "water", "burial",
                "helix", "amh_go", "frag_mem", "vec_fm", "contact_restraints", "membrane", "ssb", "dh",
                "vexcluded", "bond", "kinetic"]


class RunParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("langevin", C.c_int), ("t_start", C.c_double), ("t_stop", C.c_double),
                ("damp", C.c_double), ("seed", C.c_ulonglong), ("skin", C.c_double), ("neigh_every", C.c_int)]


class ReplicaDesc(C.Structure):
    _fields_ = [("n_res", C.c_int), ("n_chains", C.c_int), ("chain_len", C.c_void_p), ("seq", C.c_char_p),
                ("ssweight", C.c_void_p), ("x", C.c_void_p), ("v", C.c_void_p), ("n_mem", C.c_int),
                ("mem_pos", C.c_void_p), ("mem_len", C.c_void_p), ("mem_weight", C.c_void_p),
                ("mem_seq", C.c_char_p), ("mem_ca", C.c_void_p), ("mem_cb", C.c_void_p),
                ("seed", C.c_ulonglong)]


class AwsemError(RuntimeError):
    pass


def replica_desc(c: dict, seed: int = 0) -> ReplicaDesc:
    """awsem_replica_desc over the arrays of one chain dict (synth.chain_arrays
    layout); the arrays must stay alive while the descriptor is in use."""
    d = ReplicaDesc()
    d.n_res = int(c["n_res"])
    d.n_chains = len(c["chain_len"])
    d.chain_len = c["chain_len"].ctypes.data
    d.seq = c["seq"]
    d.ssweight = c["ssweight"].ctypes.data if c.get("ssweight") is not None else None
    d.x = c["x"].ctypes.data
    d.v = c["v"].ctypes.data if c.get("v") is not None else None
    d.n_mem = int(c["n_mem"])
    d.mem_pos = c["mem_pos"].ctypes.data
    d.mem_len = c["mem_len"].ctypes.data
    d.mem_weight = c["mem_weight"].ctypes.data
    d.mem_seq = c["mem_seq"]
    d.mem_ca = c["mem_ca"].ctypes.data
    d.mem_cb = c["mem_cb"].ctypes.data
    d.seed = int(seed)
    return d


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libawsem_gpu.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise AwsemError(f"CUDA library not built: {path} (run awsemmd_b200/build.py)")
    lib = C.CDLL(path)
    vp, cp, dp, ip = C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.c_int
    lib.awsem_last_error.restype = cp
    lib.awsem_version.restype = ip
    lib.awsem_create_from_files.argtypes = [cp, cp, cp, cp, cp, cp, ip, ip, C.POINTER(vp)]
    lib.awsem_destroy.argtypes = [vp]
    lib.awsem_destroy.restype = None
    lib.awsem_natoms.argtypes = [vp]
    lib.awsem_nres.argtypes = [vp]
    lib.awsem_step.argtypes = [vp]
    lib.awsem_step.restype = C.c_longlong
    lib.awsem_compute.argtypes = [vp, C.c_longlong, vp, vp, vp, ip]
    lib.awsem_set_state.argtypes = [vp, vp, vp]
    lib.awsem_get_state.argtypes = [vp, vp, vp]
    lib.awsem_run.argtypes = [vp, C.c_longlong, C.POINTER(RunParams), vp]
    lib.awsem_energies.argtypes = [vp, vp]
    lib.awsem_forces.argtypes = [vp, vp]
    lib.awsem_residue_arrays.argtypes = [vp, vp]
    lib.awsem_debug_selections.argtypes = [vp, C.c_longlong, vp, vp, C.c_longlong, C.POINTER(C.c_longlong)]
    lib.awsem_set_wait_limits.argtypes = [vp, C.c_longlong, C.c_longlong, ip]
    lib.awsem_neighbor_stats.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int)]
    lib.awsem_last_run_ms.argtypes = [vp]
    lib.awsem_last_run_ms.restype = C.c_double
    lib.awsem_kernel_name.argtypes = [ip]
    lib.awsem_kernel_name.restype = cp
    lib.awsem_profile_step.argtypes = [vp, ip, vp]
    lib.awsem_autotune.argtypes = [vp, ip, vp]
    lib.awsem_set_step_form.argtypes = [vp, ip, ip, ip]
    lib.awsem_get_step_form.argtypes = [vp, vp]
    lib.awsem_set_launch_shapes.argtypes = [vp, vp]
    lib.awsem_set_neighbor.argtypes = [vp, C.c_double, ip, ip, ip]
    lib.awsem_set_list_built.argtypes = [vp, ip]
    lib.awsem_q_create.argtypes = [vp, ip, cp, vp]
    lib.awsem_q_value.argtypes = [vp, ip, vp]
    lib.awsem_run_window.argtypes = [vp, C.c_longlong, C.POINTER(RunParams), C.c_longlong, C.c_longlong, ip, vp]
    lib.awsem_create_from_atoms.argtypes = [cp, cp, cp, ip, vp, vp, vp, vp, vp, vp, ip, vp, ip, vp, vp, vp, vp, cp, cp,
                                            ip, ip, C.POINTER(vp)]
    lib.awsem_model_info.argtypes = [vp, vp]
    lib.awsem_batch_create.argtypes = [ip, ip, C.POINTER(vp)]
    lib.awsem_batch_add_files.argtypes = [vp, cp, cp, cp, cp, cp, cp, C.c_ulonglong, C.POINTER(ip)]
    lib.awsem_batch_commit.argtypes = [vp]
    lib.awsem_nreplicas.argtypes = [vp]
    lib.awsem_replica_natoms.argtypes = [vp, ip]
    lib.awsem_replica_nres.argtypes = [vp, ip]
    lib.awsem_replica_set_state.argtypes = [vp, ip, vp, vp]
    lib.awsem_replica_get_state.argtypes = [vp, ip, vp, vp]
    lib.awsem_replica_energies.argtypes = [vp, ip, vp]
    lib.awsem_replica_forces.argtypes = [vp, ip, vp]
    lib.awsem_batch_set_forcefield.argtypes = [vp, cp, cp, cp, cp]
    lib.awsem_batch_add_replica.argtypes = [vp, C.POINTER(ReplicaDesc), C.POINTER(ip)]
    lib.awsem_batch_set_state.argtypes = [vp, vp, vp]
    lib.awsem_batch_get_state.argtypes = [vp, vp, vp]
    ll = C.c_longlong
    lib.awsem_server_create.argtypes = [cp, cp, cp, cp, ip, ip, ll, ip, ll, C.c_double, C.c_double, C.POINTER(vp)]
    lib.awsem_server_admit.argtypes = [vp, C.POINTER(ReplicaDesc), ll, C.c_double, C.c_double, C.POINTER(ip)]
    lib.awsem_server_prepare.argtypes = [vp, C.POINTER(ReplicaDesc), C.POINTER(vp)]
    lib.awsem_server_admit_prepared.argtypes = [vp, vp, ll, C.c_double, C.c_double, C.POINTER(ip)]
    lib.awsem_request_free.argtypes = [vp]
    lib.awsem_request_free.restype = None
    lib.awsem_server_advance.argtypes = [vp, ll]
    lib.awsem_server_progress.argtypes = [vp, ip, C.POINTER(ll), C.POINTER(ll)]
    lib.awsem_server_collect.argtypes = [vp, ip, vp, vp, vp]
    lib.awsem_server_usage.argtypes = [vp, vp]
    _lib = lib
    return lib


def _check(lib, rc: int, what: str):
    if rc != 0:
        raise AwsemError(f"{what} failed ({rc}): {lib.awsem_last_error().decode()}")


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class AwsemSystem:
    """One AWSEM system on one GPU (the `fix backbone` + `pair vexcluded` path)."""

    def __init__(self, files: dict, precision: str | int = "fp64", device: int = 0):
        lib = load_library()
        self.lib = lib
        prec = {"fp64": FP64, "mixed": MIXED}.get(precision, precision)
        h = C.c_void_p()
        rc = lib.awsem_create_from_files(files["workdir"].encode(), files["data"].encode(), files["coeff"].encode(),
                                         files["seq"].encode(), files["pair_style"].encode(),
                                         files.get("pair_coeffs", "").encode(), int(prec), int(device), C.byref(h))
        _check(lib, rc, "awsem_create_from_files")
        self.h = h
        self.natoms = lib.awsem_natoms(h)
        self.nres = lib.awsem_nres(h)
        self.precision = prec

    @classmethod
    def from_atoms(cls, workdir: str, coeff: str, seq: str, role, residue, molecule, atom_type, tag, mass_by_type,
                   x=None, bonds=None, pair_style: str = "2 3.5 3.5", pair_coeffs: str = "",
                   precision: str | int = "fp64", device: int = 0):
        """A system from per-atom arrays in the caller's order (awsem_create_from_atoms):
        role 0 CA, 1 CB / H-beta, 2 O; mass_by_type[t] for t = 1..ntypes (index 0 unused);
        bonds = (a, b, K, r0) with 0-based caller indices, or None."""
        self = cls.__new__(cls)
        lib = load_library()
        self.lib = lib
        prec = {"fp64": FP64, "mixed": MIXED}.get(precision, precision)
        ints = [np.ascontiguousarray(v, dtype=np.int32) for v in (role, residue, molecule, atom_type, tag)]
        n = len(ints[0])
        mass = np.ascontiguousarray(mass_by_type, dtype=np.float64)
        xa = None if x is None else np.ascontiguousarray(x, dtype=np.float64).reshape(n, 3)
        if bonds is not None and len(bonds[0]):
            ba, bb = (np.ascontiguousarray(v, dtype=np.int32) for v in bonds[:2])
            bk, br = (np.ascontiguousarray(v, dtype=np.float64) for v in bonds[2:])
            nb, bp = len(ba), [_ptr(ba), _ptr(bb), _ptr(bk), _ptr(br)]
        else:
            nb, bp = 0, [None] * 4
        h = C.c_void_p()
        rc = lib.awsem_create_from_atoms(workdir.encode(), coeff.encode(), seq.encode(), n, *[_ptr(v) for v in ints],
                                         _ptr(mass), len(mass) - 1, None if xa is None else _ptr(xa), nb, *bp,
                                         pair_style.encode(), pair_coeffs.encode(), int(prec), int(device), C.byref(h))
        _check(lib, rc, "awsem_create_from_atoms")
        self.h = h
        self.natoms = lib.awsem_natoms(h)
        self.nres = lib.awsem_nres(h)
        self.precision = prec
        return self

    def close(self):
        if getattr(self, "h", None):
            self.lib.awsem_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run_window(self, nsteps: int, window: tuple, cont: bool, dt=2.0, langevin=True, t_start=300.0,
                   t_stop=300.0, damp=500.0, seed=1, skin=2.0, neigh_every=0, thermo=False):
        """nsteps of the run window (begin, end) (awsem_run_window); cont continues the previous call."""
        rp = RunParams(dt, int(langevin), t_start, t_stop, damp, seed, skin, neigh_every)
        nrep = getattr(self, "nreplicas", 1)
        rows = np.zeros((nrep, nsteps + (0 if cont else 1), 4)) if thermo else None
        _check(self.lib, self.lib.awsem_run_window(self.h, nsteps, C.byref(rp), int(window[0]), int(window[1]),
                                                   int(bool(cont)), None if rows is None else _ptr(rows)),
               "awsem_run_window")
        return rows if rows is None or nrep > 1 else rows[0]

    @property
    def step(self) -> int:
        return int(self.lib.awsem_step(self.h))

    def compute(self, x: np.ndarray, step: int = 0, terms: int = TERMS_ALL, f: np.ndarray | None = None):
        """Forces at x added into f (zeros when not given) and the energy vector."""
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(self.natoms, 3)
        if f is None:
            f = np.zeros((self.natoms, 3))
        e = np.zeros(21)
        _check(self.lib, self.lib.awsem_compute(self.h, step, _ptr(x), _ptr(f), _ptr(e), terms), "awsem_compute")
        return f, e

    def set_state(self, x: np.ndarray | None = None, v: np.ndarray | None = None):
        xa = None if x is None else np.ascontiguousarray(x, dtype=np.float64).reshape(self.natoms, 3)
        va = None if v is None else np.ascontiguousarray(v, dtype=np.float64).reshape(self.natoms, 3)
        _check(self.lib, self.lib.awsem_set_state(self.h, None if xa is None else _ptr(xa),
                                                  None if va is None else _ptr(va)), "awsem_set_state")

    def get_state(self):
        x = np.zeros((self.natoms, 3))
        v = np.zeros((self.natoms, 3))
        _check(self.lib, self.lib.awsem_get_state(self.h, _ptr(x), _ptr(v)), "awsem_get_state")
        return x, v

    def run(self, nsteps: int, dt=2.0, langevin=True, t_start=300.0, t_stop=300.0, damp=500.0, seed=1,
            skin=2.0, neigh_every=0, thermo=False):
        rp = RunParams(dt, int(langevin), t_start, t_stop, damp, seed, skin, neigh_every)
        rows = np.zeros((nsteps + 1, 4)) if thermo else None
        _check(self.lib, self.lib.awsem_run(self.h, nsteps, C.byref(rp), None if rows is None else _ptr(rows)),
               "awsem_run")
        return rows

    def energies(self) -> np.ndarray:
        e = np.zeros(21)
        _check(self.lib, self.lib.awsem_energies(self.h, _ptr(e)), "awsem_energies")
        return e

    def forces(self) -> np.ndarray:
        f = np.zeros((self.natoms, 3))
        _check(self.lib, self.lib.awsem_forces(self.h, _ptr(f)), "awsem_forces")
        return f

    def residue_arrays(self) -> np.ndarray:
        out = np.zeros((self.nres, 8))
        _check(self.lib, self.lib.awsem_residue_arrays(self.h, _ptr(out)), "awsem_residue_arrays")
        return out

    def selections(self, x: np.ndarray, step: int = 0) -> np.ndarray:
        """Sorted AWSEM_SEL_* selection keys of one evaluation at x
        (awsem_debug_selections; kind << 56 | aux << 44 | i << 22 | j)"""
        x = np.ascontiguousarray(x, dtype=np.float64)
        cap = 96 * self.nres + 4096
        while True:
            keys = np.zeros(cap, dtype=np.uint64)
            got = C.c_longlong()
            rc = self.lib.awsem_debug_selections(self.h, step, _ptr(x), _ptr(keys), cap, C.byref(got))
            if rc == 0:
                return np.sort(keys[:got.value])
            if got.value <= cap:
                _check(self.lib, rc, "awsem_debug_selections")
            cap = got.value + 1024

    def neighbor_stats(self) -> dict:
        nb, mc, ov = C.c_int(), C.c_int(), C.c_int()
        rad = C.c_double()
        _check(self.lib, self.lib.awsem_neighbor_stats(self.h, C.byref(nb), C.byref(rad), C.byref(mc), C.byref(ov)),
               "awsem_neighbor_stats")
        return {"builds": nb.value, "radius": rad.value, "max_count": mc.value, "overflow": ov.value}

    # ------------------------------------------------------------------
    # measurement helpers
    def last_run_ms(self) -> float:
        return float(self.lib.awsem_last_run_ms(self.h))

    def profile_step(self, reps: int = 20) -> dict:
        ms = np.zeros(NKERNELS)
        _check(self.lib, self.lib.awsem_profile_step(self.h, reps, _ptr(ms)), "awsem_profile_step")
        return {self.lib.awsem_kernel_name(k).decode(): float(ms[k]) for k in range(NKERNELS)}

    def autotune(self, reps: int = 5) -> dict:
        """Pick the fastest launch shapes and step form on this system (awsem_autotune)."""
        got = np.zeros(4, dtype=np.int32)
        _check(self.lib, self.lib.awsem_autotune(self.h, int(reps), _ptr(got)), "awsem_autotune")
        return {"fragmem_separations_per_warp": int(got[0]), "pair_pass_blocks": int(got[1]),
                "hbond_blocks": int(got[2]), "fragmem_blocks": int(got[3]), **self.step_form()}

    SHAPE_KEYS = ("fragmem_separations_per_warp", "pair_pass_blocks", "hbond_blocks", "fragmem_blocks")

    def set_launch_shapes(self, shapes) -> None:
        """Apply launch shapes (a dict as `autotune` returns, or four ints in its order)."""
        v = [shapes[k] for k in self.SHAPE_KEYS] if isinstance(shapes, dict) else list(shapes)
        arr = np.array(v, dtype=np.int32)
        _check(self.lib, self.lib.awsem_set_launch_shapes(self.h, _ptr(arr)), "awsem_set_launch_shapes")

    def set_neighbor(self, skin: float = 0.0, delay: int = 0, every: int = 1, check: bool = True) -> None:
        """LAMMPS `neighbor` skin (> 0 sets it) and neigh_modify delay/every/check
        of the neighbour list [AMH-Go] reads (awsem_set_neighbor); LAMMPS's
        defaults until called."""
        chk = int(check) if not isinstance(check, bool) else int(check is True)
        _check(self.lib, self.lib.awsem_set_neighbor(self.h, float(skin), int(delay), int(every), chk),
               "awsem_set_neighbor")

    def q_create(self, words: str, rep: int = 0) -> int:
        """A Q order parameter (awsem_q_create): `words` as after LAMMPS's
        `compute` (ID group qwolynes ... / qonuchic ...)."""
        qid = C.c_int()
        _check(self.lib, self.lib.awsem_q_create(self.h, int(rep), words.encode(), C.byref(qid)), "awsem_q_create")
        return qid.value

    def q_value(self, qid: int) -> float:
        """The Q order parameter on the replica's current positions (awsem_q_value)."""
        v = C.c_double()
        _check(self.lib, self.lib.awsem_q_value(self.h, int(qid), C.byref(v)), "awsem_q_value")
        return v.value

    def set_wait_limits(self, fm_cycles: int = 0, barrier_cycles: int = 0, hold: int = 0) -> None:
        """Limits of the bounded device waits in SM clock cycles (0: the
        defaults); hold (tests) makes waits run out: bit 0 the fragment-memory
        copy waits, bit 1 the grid barriers (awsem_set_wait_limits)"""
        _check(self.lib, self.lib.awsem_set_wait_limits(self.h, int(fm_cycles), int(barrier_cycles), int(hold)),
               "awsem_set_wait_limits")

    def set_step_form(self, form: str, blocks: int = 0, stream_warps: int = 2) -> None:
        """'kernels': each MD step a graph of per-pass kernels; 'persistent':
        one cooperative launch per step (awsem_set_step_form)."""
        f = {"kernels": 0, "persistent": 1}[form]
        _check(self.lib, self.lib.awsem_set_step_form(self.h, f, int(blocks), int(stream_warps)),
               "awsem_set_step_form")

    def step_form(self) -> dict:
        got = np.zeros(3, dtype=np.int32)
        _check(self.lib, self.lib.awsem_get_step_form(self.h, _ptr(got)), "awsem_get_step_form")
        return {"step_form": "persistent" if got[0] else "kernels", "persistent_blocks": int(got[1]),
                "stream_warps": int(got[2])}

    def model_info(self) -> np.ndarray:
        info = np.zeros(8, dtype=np.int64)
        _check(self.lib, self.lib.awsem_model_info(self.h, _ptr(info)), "awsem_model_info")
        return info


class AwsemBatch(AwsemSystem):
    """Independent replicas advanced together by one launch sequence."""

    def __init__(self, replicas: list, precision: str | int = "mixed", device: int = 0, seeds=None):
        lib = load_library()
        self.lib = lib
        prec = {"fp64": FP64, "mixed": MIXED}.get(precision, precision)
        h = C.c_void_p()
        _check(lib, lib.awsem_batch_create(int(prec), int(device), C.byref(h)), "awsem_batch_create")
        self.h = h
        try:
            for k, files in enumerate(replicas):
                seed = 0 if seeds is None else int(seeds[k])
                rid = C.c_int()
                _check(lib, lib.awsem_batch_add_files(h, files["workdir"].encode(), files["data"].encode(),
                                                      files["coeff"].encode(), files["seq"].encode(),
                                                      files["pair_style"].encode(),
                                                      files.get("pair_coeffs", "").encode(), seed, C.byref(rid)),
                       "awsem_batch_add_files")
            _check(lib, lib.awsem_batch_commit(h), "awsem_batch_commit")
        except Exception:
            self.close()
            raise
        self.natoms = lib.awsem_natoms(h)
        self.nres = lib.awsem_nres(h)
        self.nreplicas = lib.awsem_nreplicas(h)
        self.precision = prec

    @classmethod
    def from_arrays(cls, forcefield: dict, chains, precision: str | int = "mixed", device: int = 0, seeds=None):
        """Replicas described by arrays (see synth.chain_arrays) sharing the
        force field of a run directory (synth.forcefield_dir)."""
        self = cls.__new__(cls)
        lib = load_library()
        self.lib = lib
        prec = {"fp64": FP64, "mixed": MIXED}.get(precision, precision)
        h = C.c_void_p()
        _check(lib, lib.awsem_batch_create(int(prec), int(device), C.byref(h)), "awsem_batch_create")
        self.h = h
        try:
            _check(lib, lib.awsem_batch_set_forcefield(h, forcefield["workdir"].encode(),
                                                       forcefield["coeff"].encode(),
                                                       forcefield["pair_style"].encode(),
                                                       forcefield.get("pair_coeffs", "").encode()),
                   "awsem_batch_set_forcefield")
            for k, c in enumerate(chains):
                d = replica_desc(c, 0 if seeds is None else int(seeds[k]))
                rid = C.c_int()
                _check(lib, lib.awsem_batch_add_replica(h, C.byref(d), C.byref(rid)), "awsem_batch_add_replica")
            _check(lib, lib.awsem_batch_commit(h), "awsem_batch_commit")
        except Exception:
            self.close()
            raise
        self.natoms = lib.awsem_natoms(h)
        self.nres = lib.awsem_nres(h)
        self.nreplicas = lib.awsem_nreplicas(h)
        self.precision = prec
        return self

    def replica_natoms(self, r: int) -> int:
        return int(self.lib.awsem_replica_natoms(self.h, r))

    def get_state(self, r: int = 0):
        n = self.replica_natoms(r)
        x, v = np.zeros((n, 3)), np.zeros((n, 3))
        _check(self.lib, self.lib.awsem_replica_get_state(self.h, r, _ptr(x), _ptr(v)), "awsem_replica_get_state")
        return x, v

    def set_state(self, x=None, v=None, r: int = 0):
        n = self.replica_natoms(r)
        xa = None if x is None else np.ascontiguousarray(x, dtype=np.float64).reshape(n, 3)
        va = None if v is None else np.ascontiguousarray(v, dtype=np.float64).reshape(n, 3)
        _check(self.lib, self.lib.awsem_replica_set_state(self.h, r, None if xa is None else _ptr(xa),
                                                          None if va is None else _ptr(va)),
               "awsem_replica_set_state")

    def energies(self, r: int = 0) -> np.ndarray:
        e = np.zeros(21)
        _check(self.lib, self.lib.awsem_replica_energies(self.h, r, _ptr(e)), "awsem_replica_energies")
        return e

    def set_state_all(self, x=None, v=None):
        """Every replica at once: [natoms][3] arrays, replicas concatenated in
        order, each in its caller atom order (awsem_batch_set_state)."""
        xa = None if x is None else np.ascontiguousarray(x, dtype=np.float64).reshape(self.natoms, 3)
        va = None if v is None else np.ascontiguousarray(v, dtype=np.float64).reshape(self.natoms, 3)
        _check(self.lib, self.lib.awsem_batch_set_state(self.h, None if xa is None else _ptr(xa),
                                                        None if va is None else _ptr(va)), "awsem_batch_set_state")

    def get_state_all(self, x: np.ndarray | None = None, v: np.ndarray | None = None):
        """Every replica at once into x, v (allocated when not given)."""
        x = np.zeros((self.natoms, 3)) if x is None else x
        v = np.zeros((self.natoms, 3)) if v is None else v
        assert x.flags.c_contiguous and v.flags.c_contiguous and x.dtype == np.float64 and v.dtype == np.float64
        _check(self.lib, self.lib.awsem_batch_get_state(self.h, _ptr(x), _ptr(v)), "awsem_batch_get_state")
        return x, v

    def forces(self, r: int = 0) -> np.ndarray:
        f = np.zeros((self.replica_natoms(r), 3))
        _check(self.lib, self.lib.awsem_replica_forces(self.h, r, _ptr(f)), "awsem_replica_forces")
        return f

    def run(self, nsteps: int, dt=2.0, langevin=True, t_start=300.0, t_stop=300.0, damp=500.0, seed=1,
            skin=2.0, neigh_every=0, thermo=False):
        rp = RunParams(dt, int(langevin), t_start, t_stop, damp, seed, skin, neigh_every)
        rows = np.zeros((self.nreplicas, nsteps + 1, 4)) if thermo else None
        _check(self.lib, self.lib.awsem_run(self.h, nsteps, C.byref(rp), None if rows is None else _ptr(rows)),
               "awsem_run")
        return rows


EBUSY = -6


class PreparedRequest:
    """A request prepared on the host for one serving handle (awsem_request)."""

    def __init__(self, lib, h, n_res: int):
        self.lib, self.h, self.n_res = lib, h, n_res

    def free(self):
        if getattr(self, "h", None):
            self.lib.awsem_request_free(self.h)
            self.h = None

    def __del__(self):
        self.free()


class AwsemServer:
    """Continuous batching of MD requests on one GPU (awsem_server_* C ABI).

    All device memory is allocated at creation from the three capacities;
    `admit` places a request or returns None when it does not fit now,
    `advance` runs every admitted request, `collect` returns a finished
    request's final state and energies and frees its room."""

    def __init__(self, forcefield: dict, max_residues: int, max_requests: int, max_memory_records: int,
                 precision: str | int = "mixed", device: int = 0, dt: float = 2.0, damp: float = 500.0):
        lib = load_library()
        self.lib = lib
        prec = {"fp64": FP64, "mixed": MIXED}.get(precision, precision)
        h = C.c_void_p()
        _check(lib, lib.awsem_server_create(forcefield["workdir"].encode(), forcefield["coeff"].encode(),
                                            forcefield["pair_style"].encode(),
                                            forcefield.get("pair_coeffs", "").encode(), int(prec), int(device),
                                            int(max_residues), int(max_requests), int(max_memory_records),
                                            float(dt), float(damp), C.byref(h)), "awsem_server_create")
        self.h = h
        self.precision = prec
        self.natoms = {}

    def close(self):
        if getattr(self, "h", None):
            self.lib.awsem_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def prepare(self, chain: dict, seed: int = 1) -> "PreparedRequest":
        """Host-side preparation of a request (awsem_server_prepare): safe to
        call from another thread while `advance` runs."""
        d = replica_desc(chain, seed)
        out = C.c_void_p()
        _check(self.lib, self.lib.awsem_server_prepare(self.h, C.byref(d), C.byref(out)), "awsem_server_prepare")
        return PreparedRequest(self.lib, out, int(chain["n_res"]))

    def admit(self, chain, nsteps: int, t_start: float = 300.0, t_stop: float = 300.0, seed: int = 1):
        """Place a request (chain arrays, or a PreparedRequest whose seed was
        given to `prepare`); None when it does not fit now."""
        slot = C.c_int()
        if isinstance(chain, PreparedRequest):
            rc = self.lib.awsem_server_admit_prepared(self.h, chain.h, int(nsteps), float(t_start), float(t_stop),
                                                      C.byref(slot))
            what, n_res = "awsem_server_admit_prepared", chain.n_res
        else:
            d = replica_desc(chain, seed)
            rc = self.lib.awsem_server_admit(self.h, C.byref(d), int(nsteps), float(t_start), float(t_stop),
                                             C.byref(slot))
            what, n_res = "awsem_server_admit", int(chain["n_res"])
        if rc == EBUSY:
            return None
        _check(self.lib, rc, what)
        self.natoms[slot.value] = 3 * n_res
        return slot.value

    def advance(self, nsteps: int):
        _check(self.lib, self.lib.awsem_server_advance(self.h, int(nsteps)), "awsem_server_advance")

    def progress(self, slot: int):
        done, total = C.c_longlong(), C.c_longlong()
        _check(self.lib, self.lib.awsem_server_progress(self.h, slot, C.byref(done), C.byref(total)),
               "awsem_server_progress")
        return done.value, total.value

    def collect(self, slot: int):
        n = self.natoms.pop(slot)
        x, v, e = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(21)
        _check(self.lib, self.lib.awsem_server_collect(self.h, slot, _ptr(x), _ptr(v), _ptr(e)),
               "awsem_server_collect")
        return x, v, e

    # step form of `advance` (awsem_set_step_form), as on the batch handles
    set_step_form = AwsemSystem.set_step_form
    step_form = AwsemSystem.step_form

    def usage(self) -> dict:
        info = np.zeros(8, dtype=np.int64)
        _check(self.lib, self.lib.awsem_server_usage(self.h, _ptr(info)), "awsem_server_usage")
        keys = ["requests", "residues", "residue_capacity", "records", "record_capacity", "device_bytes", "step",
                "request_capacity"]
        return {k: int(v) for k, v in zip(keys, info)}

    def last_run_ms(self) -> float:
        return float(self.lib.awsem_last_run_ms(self.h))
