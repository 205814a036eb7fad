"""ctypes bindings for the oracle libraries (test infrastructure only).

* ``RefSystem``: the reference FixBackbone + PairExcludedVolume, compiled
  unmodified from the reference sources against the LAMMPS-API shim
  (``oracle/_ref/libawsem_ref.so``, built by ``make -C oracle ref``).
  ``RefSystem(files, gpu_fix="fp64" | "mixed")`` runs the same host with the
  GPU adapter ``fix backbone/gpu`` in place of the reference fix, and
  ``RefSystem(files, gpu_pair=...)`` with ``pair_style vexcluded/gpu`` in place
  of the reference pair style (``oracle/_ref/libawsem_ref_gpufix.so``,
  ``make -C oracle gpufix``).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference source tree the oracle recipe compiles (oracle/Makefile's REF);
# AWSEM_REFERENCE_DIR overrides it
REFERENCE_DIR = os.environ.get("AWSEM_REFERENCE_DIR", "/root/reference")
REF_LIB = os.path.join(HERE, "_ref", "libawsem_ref.so")
GPUFIX_LIB = os.path.join(HERE, "_ref", "libawsem_ref_gpufix.so")

_libs = {}


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def gpufix_available() -> bool:
    return os.path.exists(GPUFIX_LIB)


def _load_ref(path=REF_LIB):
    if path not in _libs:
        lib = C.CDLL(path)
        lib.ref_create.restype = C.c_void_p
        lib.ref_create.argtypes = [C.c_char_p] * 6 + [C.c_double, C.c_int, C.c_int, C.c_int]
        lib.ref_destroy.argtypes = [C.c_void_p]
        lib.ref_natoms.argtypes = [C.c_void_p]
        lib.ref_fix_cutoff.argtypes = [C.c_void_p]
        lib.ref_fix_cutoff.restype = C.c_double
        lib.ref_get.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        lib.ref_set.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        lib.ref_energies.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_compute.argtypes = [C.c_void_p, C.c_longlong, C.c_void_p]
        lib.ref_residue_arrays.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_run.argtypes = [C.c_void_p, C.c_longlong, C.c_double, C.c_int, C.c_double, C.c_double,
                                C.c_double, C.c_ulonglong, C.c_void_p]
        lib.ref_compute_q.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        lib.ref_touches.restype = C.c_longlong
        lib.ref_touches.argtypes = [C.c_void_p, C.c_void_p, C.c_longlong]
        lib.ref_nbuilds.argtypes = [C.c_void_p]
        lib.ref_nbuilds.restype = C.c_long
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_uniform.restype = C.c_double
        lib.ref_uniform.argtypes = [C.c_ulonglong, C.c_longlong, C.c_longlong, C.c_int]
        if path == GPUFIX_LIB:
            for fn in (lib.ref_create_gpufix, lib.ref_create_gpupair):
                fn.restype = C.c_void_p
                fn.argtypes = [C.c_char_p] * 6 + [C.c_double, C.c_int, C.c_int, C.c_int, C.c_int]
        _libs[path] = lib
    return _libs[path]


class RefSystem:
    """One reference FixBackbone system hosted by the shim MD loop."""

    def __init__(self, files: dict, skin=2.0, every=1, delay=0, check=1, gpu_fix: str | None = None,
                 gpu_pair: str | None = None):
        assert not (gpu_fix and gpu_pair)
        lib = _load_ref(GPUFIX_LIB if gpu_fix or gpu_pair else REF_LIB)
        self.lib = lib
        args = (files["workdir"].encode(), files["data"].encode(), files["coeff"].encode(), files["seq"].encode(),
                files["pair_style"].encode(), files["pair_coeffs"].encode(), skin, every, delay, check)
        if gpu_fix:
            self.h = lib.ref_create_gpufix(*args, {"fp64": 0, "mixed": 1}[gpu_fix])
        elif gpu_pair:
            self.h = lib.ref_create_gpupair(*args, {"fp64": 0, "mixed": 1}[gpu_pair])
        else:
            self.h = lib.ref_create(*args)
        if not self.h:
            raise RuntimeError(lib.ref_last_error().decode())
        self.natoms = lib.ref_natoms(self.h)

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def get(self, what: str) -> np.ndarray:
        out = np.zeros((self.natoms, 3))
        self.lib.ref_get(self.h, what.encode(), out.ctypes.data)
        return out

    def set(self, what: str, arr: np.ndarray):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        self.lib.ref_set(self.h, what.encode(), a.ctypes.data)

    def energies(self) -> np.ndarray:
        out = np.zeros(21)
        self.lib.ref_energies(self.h, out.ctypes.data)
        return out

    def compute(self, step=0) -> np.ndarray:
        f = np.zeros((self.natoms, 3))
        if self.lib.ref_compute(self.h, step, f.ctypes.data) != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return f

    def compute_q(self, words: str) -> float:
        """the reference's `compute <words>` (qwolynes / qonuchic) at the current positions"""
        out = C.c_double()
        if self.lib.ref_compute_q(self.h, words.encode(), C.byref(out)) != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return out.value

    def nbuilds(self) -> int:
        """neighbour-list builds so far (run setups included)"""
        return int(self.lib.ref_nbuilds(self.h))

    def residue_arrays(self, n_res: int) -> np.ndarray:
        out = np.zeros((n_res, 6))
        self.lib.ref_residue_arrays(self.h, out.ctypes.data)
        return out

    def touches(self) -> np.ndarray:
        """sorted keys of the reference's n x n cache entries that the last
        evaluation read or filled (kinds 32-36, oracle/ref_host.cpp)"""
        n = self.lib.ref_touches(self.h, None, 0)
        if n < 0:
            raise RuntimeError("no reference fix hosted")
        out = np.zeros(max(n, 1), dtype=np.uint64)
        self.lib.ref_touches(self.h, out.ctypes.data, n)
        return out[:n]

    def run(self, nsteps, dt=2.0, langevin=True, t_start=300.0, t_stop=300.0, damp=500.0, seed=1):
        thermo = np.zeros((nsteps + 1, 4))
        if self.lib.ref_run(self.h, nsteps, dt, int(langevin), t_start, t_stop, damp, seed, thermo.ctypes.data) != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return thermo


# --------------------------------------------------------------------------
# FP64 restatement (oracle/_build/liboracle.so, built by ``make -C oracle``)

ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
_orc = None


def oracle_available() -> bool:
    return os.path.exists(ORACLE_LIB)


def _load_oracle():
    global _orc
    if _orc is None:
        lib = C.CDLL(ORACLE_LIB)
        lib.oracle_create.restype = C.c_void_p
        lib.oracle_create.argtypes = [C.c_char_p] * 6
        lib.oracle_destroy.argtypes = [C.c_void_p]
        lib.oracle_last_error.restype = C.c_char_p
        lib.oracle_natoms.argtypes = [C.c_void_p]
        lib.oracle_nres.argtypes = [C.c_void_p]
        lib.oracle_compute.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.oracle_residue_arrays.argtypes = [C.c_void_p, C.c_void_p]
        lib.oracle_selections.restype = C.c_longlong
        lib.oracle_selections.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_longlong]
        lib.oracle_run.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong, C.c_longlong, C.c_double,
                                   C.c_int, C.c_double, C.c_double, C.c_double, C.c_ulonglong, C.c_void_p]
        lib.oracle_set_neighbor.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int]
        lib.oracle_q.argtypes = [C.c_void_p, C.c_void_p, C.c_char_p, C.c_void_p]
        lib.oracle_uniform.restype = C.c_double
        lib.oracle_uniform.argtypes = [C.c_ulonglong, C.c_longlong, C.c_longlong, C.c_int]
        _orc = lib
    return _orc


class OracleSystem:
    """FP64 restatement of the AWSEM force field (the oracle proper)."""

    def __init__(self, files: dict):
        lib = _load_oracle()
        self.lib = lib
        self.h = lib.oracle_create(files["workdir"].encode(), files["data"].encode(), files["coeff"].encode(),
                                   files["seq"].encode(), files["pair_style"].encode(), files["pair_coeffs"].encode())
        if not self.h:
            raise RuntimeError(lib.oracle_last_error().decode())
        self.natoms = lib.oracle_natoms(self.h)
        self.nres = lib.oracle_nres(self.h)

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def compute(self, x: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float64)
        f = np.zeros((self.natoms, 3))
        e = np.zeros(21)
        if self.lib.oracle_compute(self.h, x.ctypes.data, f.ctypes.data, e.ctypes.data) != 0:
            raise RuntimeError(self.lib.oracle_last_error().decode())
        return f, e

    def q(self, x: np.ndarray, words: str) -> float:
        """compute qwolynes / qonuchic (`words` after `compute`) at positions x"""
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = C.c_double()
        if self.lib.oracle_q(self.h, x.ctypes.data, words.encode(), C.byref(out)) != 0:
            raise RuntimeError(self.lib.oracle_last_error().decode())
        return out.value

    def set_neighbor(self, skin=2.0, delay=0, every=1, check=True):
        """neighbor skin and neigh_modify delay/every/check of the list [AMH-Go] reads"""
        if self.lib.oracle_set_neighbor(self.h, float(skin), int(delay), int(every), 1 if check else 0) != 0:
            raise RuntimeError(self.lib.oracle_last_error().decode())

    def residue_arrays(self) -> np.ndarray:
        out = np.zeros((self.nres, 8))
        self.lib.oracle_residue_arrays(self.h, out.ctypes.data)
        return out

    def selections(self, x: np.ndarray, which: str = "sel") -> np.ndarray:
        """Sorted keys of one evaluation at x: "sel" the AWSEM_SEL_* selection
        records (include/awsem_gpu.h), "near" the distance predicates decided
        within 2e-6 of their threshold, "touch" the reference cache entries the
        evaluation reads or fills (kinds 32-36, as RefSystem.touches)"""
        w = {"sel": 0, "near": 1, "touch": 2}[which]
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = self.lib.oracle_selections(self.h, x.ctypes.data, w, None, 0)
        if n < 0:
            raise RuntimeError(self.lib.oracle_last_error().decode())
        out = np.zeros(max(n, 1), dtype=np.uint64)
        self.lib.oracle_selections(self.h, x.ctypes.data, w, out.ctypes.data, n)
        return out[:n]

    def run(self, x, v, nsteps, step0=0, dt=2.0, langevin=True, t_start=300.0, t_stop=300.0, damp=500.0, seed=1):
        x = np.ascontiguousarray(x, dtype=np.float64).copy()
        v = np.ascontiguousarray(v, dtype=np.float64).copy()
        thermo = np.zeros((nsteps + 1, 4))
        if self.lib.oracle_run(self.h, x.ctypes.data, v.ctypes.data, step0, nsteps, dt, int(langevin), t_start,
                               t_stop, damp, seed, thermo.ctypes.data) != 0:
            raise RuntimeError(self.lib.oracle_last_error().decode())
        return x, v, thermo


# --------------------------------------------------------------------------
# selection records (AWSEM_SEL_* keys, include/awsem_gpu.h)

SEL_KINDS = {1: "dens_water", 2: "dens_helix", 3: "xi_water", 4: "water", 5: "xi_force", 6: "helix_force",
             7: "helix_pair", 8: "dssp", 9: "pap", 10: "ev"}
# kinds whose aux carries gates on transcendental outputs (not the identity of the predicate)
_GATED = (5, 7, 8, 9)
_AUX = np.uint64(0xFFF << 44)


def _kind(keys):
    return (np.asarray(keys, dtype=np.uint64) >> np.uint64(56)).astype(np.int64)


def compare_selections(got, want, near=None) -> dict:
    """Compare two sets of selection keys kind by kind.

    ``cand`` counts items selected by one side only (for the gated kinds
    XI_FORCE, HELIX_PAIR, DSSP, PAP compared without their gate bits);
    ``cand_far`` those of them that are not in ``near`` (distance predicates
    decided within 2e-6 of their threshold by the oracle); ``gate`` counts
    items both select whose gate bits differ."""
    got = np.unique(np.asarray(got, dtype=np.uint64))
    want = np.unique(np.asarray(want, dtype=np.uint64))
    near = np.unique(np.asarray(near if near is not None else [], dtype=np.uint64))
    out = {}
    for k, name in SEL_KINDS.items():
        g, w = got[_kind(got) == k], want[_kind(want) == k]
        gated = k in _GATED
        gb, wb = (g & ~_AUX, w & ~_AUX) if gated else (g, w)
        nb = near[_kind(near) == k]
        if gated:
            nb = nb & ~_AUX
        diff = np.setxor1d(gb, wb)
        far = np.setdiff1d(diff, nb)
        common = np.intersect1d(gb, wb)
        gate = 0
        if gated and len(common):
            gmap = dict(zip((gb).tolist(), g.tolist()))
            wmap = dict(zip((wb).tolist(), w.tolist()))
            gate = sum(1 for c in common.tolist() if gmap[c] != wmap[c])
        out[name] = {"got": int(len(g)), "want": int(len(w)), "cand": int(len(diff)), "cand_far": int(len(far)),
                     "gate": int(gate)}
    return out
