"""ctypes interface to the oracle (test infrastructure only).

The oracle is a CPU restatement of Hybrid IBIsCO's per-step path
(`ibisco_oracle.cpp`).  Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline legs of ``bench.py`` use this module; the product never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libibisco_oracle.so")
_lib = None

INFO_INT = ["NATOMS", "NVIRTA", "NITEMS", "NTYPE", "NUMATOMS", "NUMBEADS", "NCOARSE", "ENSEMBLE",
            "NSTEP", "NUPDATE", "HALT_DRIFT", "NTRJ", "NMTS", "IBRDESCR", "NONBEXC_ATOM", "NONBEXC_BEAD",
            "NBTYPE", "NATYPE", "NTTYPE", "NNBTYPE", "NOTYPE", "WB", "WA", "WT", "WNB", "WO",
            "VIRT_MAXATOMS", "RESTART", "NMOL"]
INFO_FLOAT = ["DT", "FAC", "PFAC", "TEMP_IN", "PRESSURE", "MKTEMP", "MKTEMP_ATOM", "MKTEMP_BEAD",
              "RCUT_ATOM", "RCUTSQ_ATOM", "RLIST_ATOM", "RCUT_BEAD", "RCUTSQ_BEAD", "RLIST_BEAD",
              "BOX1", "BOX2", "BOX3", "R2D", "D2R", "TIMESCALE", "VSCALE", "CONV", "PSCALE",
              "TEMPSCALE", "ESCALE", "NA", "MASSSCALE"]
OBS = (["EK1", "EK2", "TEMP", "TEMP_ATOM", "TEMP_BEAD"]
       + [f"V_NB{i}" for i in (1, 2, 3)] + [f"V_BOND{i}" for i in (1, 2, 3)]
       + [f"V_ANGLE{i}" for i in (1, 2, 3)] + [f"V_TORSION{i}" for i in (1, 2, 3)]
       + [f"V_OOP{i}" for i in (1, 2, 3)]
       + ["PT11", "PT22", "PT33", "PT12", "PT13", "PT23", "BOX1", "BOX2", "BOX3",
          "BOND_OVEREXT", "CELL_CLAMPS"])


def build() -> str:
    """Compile the oracle library with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, ip, fp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)
        L.orc_open.restype = vp
        L.orc_open.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        L.orc_close.argtypes = [vp]
        L.orc_set_threads.argtypes = [vp, ctypes.c_int]
        L.orc_set_com_fix.argtypes = [vp, ctypes.c_int]
        L.orc_info_int.argtypes = [vp, ip, ctypes.c_int]
        L.orc_info_float.argtypes = [vp, fp, ctypes.c_int]
        L.orc_array_size.restype = ctypes.c_long
        L.orc_array_size.argtypes = [vp, ctypes.c_char_p]
        L.orc_get_int_array.argtypes = [vp, ctypes.c_char_p, ip, ctypes.c_long]
        L.orc_get_float_array.argtypes = [vp, ctypes.c_char_p, fp, ctypes.c_long]
        L.orc_set_state.argtypes = [vp, ctypes.c_int, fp, fp, fp]
        L.orc_init.argtypes = [vp, ctypes.c_int]
        L.orc_step.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.orc_run.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_forces.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.orc_error.restype = ctypes.c_char_p
        L.orc_error.argtypes = [vp, ctypes.c_int]
        L.orc_get_state.argtypes = [vp, ctypes.c_int, dp, dp, dp, dp]
        L.orc_get_obs.argtypes = [vp, ctypes.c_int, dp]
        L.orc_nonbonded_list.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, dp]
        L.orc_get_list.argtypes = [vp, ctypes.c_int, ctypes.c_int, ip, ctypes.c_int, ip]
        _lib = L
    return _lib


def _ptr(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


class OracleError(RuntimeError):
    pass


class Oracle:
    """One system read from a directory of reference-format input files.

    ``prec`` selects the engine: 0 = REAL*4 restatement, 1 = same algorithm in
    double precision.
    """

    def __init__(self, directory: str, threads: int = 1, com_fix: bool = True):
        L = lib()
        err = ctypes.create_string_buffer(512)
        h = L.orc_open(directory.encode(), int(threads), err, 512)
        if not h:
            raise OracleError(err.value.decode())
        self._h = h
        L.orc_set_com_fix(h, 1 if com_fix else 0)
        iv = np.zeros(64, np.int32)
        n = L.orc_info_int(h, _ptr(iv, ctypes.c_int), 64)
        self.info = {k: int(v) for k, v in zip(INFO_INT, iv[:n])}
        fv = np.zeros(64, np.float32)
        n = L.orc_info_float(h, _ptr(fv, ctypes.c_float), 64)
        self.finfo = {k: np.float32(v) for k, v in zip(INFO_FLOAT, fv[:n])}

    def close(self):
        if getattr(self, "_h", None):
            lib().orc_close(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def set_threads(self, n: int):
        lib().orc_set_threads(self._h, int(n))

    def array(self, name: str) -> np.ndarray:
        L = lib()
        n = L.orc_array_size(self._h, name.encode())
        if n < 0:
            raise KeyError(name)
        a = np.zeros(max(n, 1), np.int32)
        if L.orc_get_int_array(self._h, name.encode(), _ptr(a, ctypes.c_int), n) == 0:
            return a[:n]
        a = np.zeros(max(n, 1), np.float32)
        if L.orc_get_float_array(self._h, name.encode(), _ptr(a, ctypes.c_float), n) == 0:
            return a[:n]
        raise KeyError(name)

    def _check(self, rc: int, prec: int):
        if rc != 0:
            raise OracleError(f"oracle error {rc}: {lib().orc_error(self._h, prec).decode()}")

    def init(self, prec: int = 0):
        self._check(lib().orc_init(self._h, prec), prec)

    def set_state(self, sxyz, vxyz, box, prec: int = 0):
        s = np.ascontiguousarray(sxyz, np.float32).ravel()
        v = np.ascontiguousarray(vxyz, np.float32).ravel()
        b = np.ascontiguousarray(box, np.float32).ravel()
        self._check(lib().orc_set_state(self._h, prec, _ptr(s, ctypes.c_float), _ptr(v, ctypes.c_float),
                                        _ptr(b, ctypes.c_float)), prec)

    def step(self, step: int, prec: int = 0):
        self._check(lib().orc_step(self._h, prec, int(step)), prec)

    def run(self, first: int, nsteps: int, prec: int = 0):
        self._check(lib().orc_run(self._h, prec, int(first), int(nsteps)), prec)

    def forces(self, step: int, prec: int = 0):
        self._check(lib().orc_forces(self._h, prec, int(step)), prec)

    def nonbonded_list(self, which: int, prec: int = 0):
        """NONBONDED_FORCE.F90 on list `which` alone: forces (NITEMS,3) and
        V_NB(1..3), PT11, PT22, PT33, PT12, PT13, PT23 (not divided by the
        volume).  The engine's force arrays are replaced."""
        ni = self.info["NITEMS"]
        f = np.zeros(3 * ni)
        sums = np.zeros(9)
        dp = ctypes.c_double
        self._check(lib().orc_nonbonded_list(self._h, prec, int(which), _ptr(f, dp), _ptr(sums, dp)), prec)
        return f.reshape(ni, 3), sums

    def state(self, prec: int = 0):
        ni, na = self.info["NITEMS"], self.info["NATOMS"]
        s = np.zeros(3 * ni); r = np.zeros(3 * ni); f = np.zeros(3 * ni); v = np.zeros(3 * na)
        dp = ctypes.c_double
        lib().orc_get_state(self._h, prec, _ptr(s, dp), _ptr(r, dp), _ptr(v, dp), _ptr(f, dp))
        return {"sxyz": s.reshape(ni, 3), "rxyz": r.reshape(ni, 3), "vxyz": v.reshape(na, 3),
                "fxyz": f.reshape(ni, 3)}

    def obs(self, prec: int = 0) -> dict:
        o = np.zeros(64)
        n = lib().orc_get_obs(self._h, prec, _ptr(o, ctypes.c_double))
        return {k: float(v) for k, v in zip(OBS, o[:n])}

    def neighbour_list(self, which: int, prec: int = 0, maxnab: int = 1000):
        n = self.info["NUMATOMS"] if which == 0 else self.info["NCOARSE"]
        lst = np.zeros((max(n, 1), maxnab), np.int32)
        nn = np.zeros(max(n, 1), np.int32)
        r = lib().orc_get_list(self._h, prec, which, _ptr(lst, ctypes.c_int), maxnab, _ptr(nn, ctypes.c_int))
        if r < 0:
            raise OracleError("maxnab too small")
        return lst[:n], nn[:n]
