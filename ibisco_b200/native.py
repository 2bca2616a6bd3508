"""ctypes bindings of ``include/ibisco_gpu.h`` and a small host-side driver.

The driver mirrors the reference's program flow: the setup phase of
``main.F90:107-237`` (``ibg_setup_read`` + ``ibg_create`` + ``ibg_set_state``)
followed by the loop body of ``NEW_LOOP.F90`` / ``MTS_LOOP.f90`` (``ibg_step``
or the graph-replayed ``ibg_run``).  Status codes are those of the header; a
non-zero status raises :class:`IbiscoError`, the analogue of the reference's
``ISTOP``/``STOP`` paths.
"""
from __future__ import annotations

import ctypes
import os
import time

import numpy as np

from . import build as _build

IBG_PREC_FP32_FIXED = 0
IBG_PREC_FP64_PLAIN = 1

STATUS = {
    0: "IBG_OK", -1: "IBG_E_INVALID", -2: "IBG_E_LIST_OVERFLOW", -3: "IBG_E_TORSION_TABLE",
    -4: "IBG_E_OOP_RANGE", -5: "IBG_E_FIXED_OVERFLOW", -6: "IBG_E_CELL_GRID", -7: "IBG_E_CUDA",
    -8: "IBG_E_TIMEOUT", -9: "IBG_E_TABLE_RANGE", -10: "IBG_E_MISSING_TABLE", -11: "IBG_E_CAPACITY",
    -12: "IBG_E_IO", -13: "IBG_E_MEMORY",
}

STATUS_CODE = {v: k for k, v in STATUS.items()}

# Every entry point the header declares (checked by the CPU tests).
EXPORTS = [
    "ibg_setup_read", "ibg_setup_desc", "ibg_setup_initial_state", "ibg_setup_control",
    "ibg_setup_array_i", "ibg_setup_array_f", "ibg_setup_free",
    "ibg_create", "ibg_set_state", "ibg_step", "ibg_forces", "ibg_run", "ibg_get_state",
    "ibg_get_state_f64", "ibg_get_neighbour_list", "ibg_get_exclusions", "ibg_set_timing",
    "ibg_get_timing", "ibg_last_error", "ibg_destroy", "ibg_version", "ibg_set_l2_flush", "ibg_set_device",
    "ibg_set_list_rows", "ibg_set_list_form", "ibg_get_list_form", "ibg_nonbonded_static",
    "ibg_batch_create", "ibg_batch_run", "ibg_batch_size", "ibg_batch_get_timing", "ibg_batch_last_error",
    "ibg_batch_destroy", "ibg_device_bytes", "ibg_estimate_bytes",
    "ibg_server_create", "ibg_server_submit", "ibg_server_wait", "ibg_server_drain", "ibg_server_result",
    "ibg_server_job_error", "ibg_server_get_stats", "ibg_server_destroy",
    "ibg_get_tuning", "ibg_set_tuning", "ibg_autotune", "ibg_set_vsite_com",
    "ibg_setup_read_mem", "ibg_setup_set_nb_table",
    "ibg_trz_open", "ibg_trz_write", "ibg_trz_close", "ibg_write_restart",
]

IBG_JOB_QUEUED, IBG_JOB_RUNNING, IBG_JOB_DONE, IBG_JOB_FAILED = 0, 1, 2, 3
IBG_VS_COM_FIXED, IBG_VS_COM_REFERENCE = 0, 1
LIST_AUTO, LIST_PER_PARTICLE, LIST_PER_SLICE = -1, 0, 1  # ibg_set_list_form


_I, _F, _PI, _PF = ctypes.c_int, ctypes.c_float, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)


class IbgDesc(ctypes.Structure):
    """Mirror of ``ibg_desc`` (field order of include/ibisco_gpu.h)."""
    _fields_ = (
        [(n, _I) for n in ("natoms", "nvirta", "nitems", "ntype", "numatoms", "numbeads", "ncoarse", "ensemble",
                           "nupdate", "halt_drift", "nmts", "ibrdescr", "maxnab")]
        + [(n, _F) for n in ("dt", "fac", "pfac", "temp_in", "pressure", "mktemp", "mktemp_atom", "mktemp_bead",
                             "rcut_atom", "rcutsq_atom", "rlist_atom", "rcut_bead", "rcutsq_bead", "rlist_bead")]
        + [("mass", _PF), ("invmass", _PF), ("itype", _PI), ("type_label", _PI), ("atom", _PI), ("bead", _PI),
           ("nbonds", _PI), ("jbond", _PI), ("ld_bond", _I),
           ("nijk", _PI), ("jangleijk", _PI), ("kangleijk", _PI), ("ld_angle", _I),
           ("nijkl", _PI), ("jtorijkl", _PI), ("ktorijkl", _PI), ("ltorijkl", _PI), ("ld_torsion", _I),
           ("noopijkl", _PI), ("joopijkl", _PI), ("koopijkl", _PI), ("loopijkl", _PI), ("ld_oop", _I),
           ("connections", _PI), ("connected_to", _PI), ("ld_conn", _I),
           ("ibondt", _PI), ("inbondt", _PI), ("iangt", _PI), ("itort", _PI), ("ioopt", _PI),
           ("bond_type_label", _PI), ("angle_type_label", _PI), ("torsion_type_label", _PI),
           ("oop_type_label", _PI),
           ("nbtype", _I), ("natype", _I), ("nttype", _I), ("nnbtype", _I), ("notype", _I),
           ("ld_b", _I), ("ld_a", _I), ("ld_t", _I), ("ld_nb", _I), ("ld_o", _I)]
        + [(f"{p}{q}", t) for p in ("b", "a", "t", "nb", "o")
           for q, t in (("_ndat", _PI), ("_bin", _PF), ("_x", _PF), ("_pot", _PF), ("_force", _PF))]
        + [("ld_vs", _I), ("vs_maxatoms", _I), ("vitype", _PI), ("virt_center", _PI), ("virt_numatoms", _PI),
           ("virt_atm_ind", _PI), ("virt_invmass", _PF), ("virt_masscoeff", _PF)]
    )


class Tuning(ctypes.Structure):
    _fields_ = [("nb_tables_smem", ctypes.c_int), ("nb_blocks_per_sm", ctypes.c_int), ("nb_chunk", ctypes.c_int),
                ("nb_rows", ctypes.c_int), ("nb_window", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_longlong) for k in ("submitted", "done", "failed", "running", "queued")] + \
               [(k, ctypes.c_double) for k in ("p50_s", "p99_s", "mean_s", "span_s", "jobs_per_s")] + \
               [("atom_steps", ctypes.c_longlong), ("atom_steps_per_s", ctypes.c_double), ("gpu_s", ctypes.c_double)] + \
               [(k, ctypes.c_longlong) for k in ("ticks", "batch_builds", "peak_jobs", "peak_bytes", "budget_bytes")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class IbgObs(ctypes.Structure):
    _fields_ = [
        ("ek", ctypes.c_double * 2), ("temp", ctypes.c_double), ("temp_atom", ctypes.c_double),
        ("temp_bead", ctypes.c_double), ("v_nb", ctypes.c_double * 3), ("v_bond", ctypes.c_double * 3),
        ("v_angle", ctypes.c_double * 3), ("v_torsion", ctypes.c_double * 3), ("v_oop", ctypes.c_double * 3),
        ("pt", ctypes.c_double * 6), ("box", ctypes.c_double * 3), ("bond_overext", ctypes.c_longlong),
        ("cell_clamps", ctypes.c_longlong), ("step", ctypes.c_int), ("status", ctypes.c_int),
    ]

    def as_dict(self) -> dict:
        d = {"EK1": self.ek[0], "EK2": self.ek[1], "TEMP": self.temp, "TEMP_ATOM": self.temp_atom,
             "TEMP_BEAD": self.temp_bead}
        for name in ("v_nb", "v_bond", "v_angle", "v_torsion", "v_oop"):
            for k in range(3):
                d[f"{name.upper()}{k + 1}"] = getattr(self, name)[k]
        for k, n in enumerate(("PT11", "PT22", "PT33", "PT12", "PT13", "PT23")):
            d[n] = self.pt[k]
        for k in range(3):
            d[f"BOX{k + 1}"] = self.box[k]
        d["BOND_OVEREXT"] = self.bond_overext
        d["CELL_CLAMPS"] = self.cell_clamps
        d["STEP"] = self.step
        return d


_lib = None


def library_path() -> str:
    return _build.LIB


def lib(build_if_missing: bool = True):
    """Load ``libibisco_b200.so`` (building it in-tree when it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path):
        if not build_if_missing:
            raise OSError(f"{path} is not built")
        _build.build()
    L = ctypes.CDLL(path)
    vp, cp, ip, fp, dp = (ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int),
                          ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double))
    pvp = ctypes.POINTER(ctypes.c_void_p)
    sig = {
        "ibg_setup_read": (ctypes.c_int, [cp, pvp, cp, ctypes.c_int]),
        "ibg_setup_desc": (vp, [vp]),
        "ibg_setup_read_mem": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                              ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_long), pvp,
                                              cp, ctypes.c_int]),
        "ibg_setup_set_nb_table": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, fp, fp]),
        "ibg_trz_open": (ctypes.c_int, [vp, cp, pvp]),
        "ibg_trz_write": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(IbgObs), fp, fp]),
        "ibg_trz_close": (None, [vp]),
        "ibg_write_restart": (ctypes.c_int, [vp, cp, ctypes.c_int, fp, fp, fp]),
        "ibg_setup_initial_state": (ctypes.c_int, [vp, fp, fp, fp]),
        "ibg_setup_control": (ctypes.c_int, [vp, ip, ctypes.c_int]),
        "ibg_setup_array_i": (ctypes.c_long, [vp, cp, ip, ctypes.c_long]),
        "ibg_setup_array_f": (ctypes.c_long, [vp, cp, fp, ctypes.c_long]),
        "ibg_setup_free": (None, [vp]),
        "ibg_create": (ctypes.c_int, [vp, ctypes.c_int, pvp]),
        "ibg_set_state": (ctypes.c_int, [vp, fp, fp, fp]),
        "ibg_step": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(IbgObs)]),
        "ibg_forces": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(IbgObs)]),
        "ibg_run": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(IbgObs)]),
        "ibg_get_state": (ctypes.c_int, [vp, fp, fp, fp, fp]),
        "ibg_get_state_f64": (ctypes.c_int, [vp, dp, dp, dp]),
        "ibg_get_neighbour_list": (ctypes.c_int, [vp, ctypes.c_int, ip, ctypes.c_int, ip]),
        "ibg_get_exclusions": (ctypes.c_int, [vp, ip, ip]),
        "ibg_set_timing": (ctypes.c_int, [vp, ctypes.c_int]),
        "ibg_get_timing": (ctypes.c_int, [vp, dp, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]),
        "ibg_last_error": (cp, [vp]),
        "ibg_destroy": (None, [vp]),
        "ibg_version": (cp, []),
        "ibg_set_l2_flush": (ctypes.c_int, [vp, ctypes.c_longlong]),
        "ibg_set_device": (ctypes.c_int, [ctypes.c_int]),
        "ibg_set_list_rows": (ctypes.c_int, [vp, ctypes.c_int]),
        "ibg_set_list_form": (ctypes.c_int, [vp, ctypes.c_int]),
        "ibg_get_list_form": (ctypes.c_int, [vp]),
        "ibg_set_vsite_com": (ctypes.c_int, [vp, ctypes.c_int]),
        "ibg_nonbonded_static": (ctypes.c_int, [ctypes.c_int, ctypes.c_int] + [vp] * 5 + [ctypes.c_int, vp, ctypes.c_int, vp,
                                                ctypes.c_int, ctypes.c_int] + [vp] * 5 + [vp, ctypes.c_float, vp, vp, vp,
                                                                                        cp, ctypes.c_int]),
        "ibg_batch_create": (ctypes.c_int, [pvp, ctypes.c_int, pvp]),
        "ibg_batch_run": (ctypes.c_int, [vp, ctypes.c_int, ip, ctypes.POINTER(IbgObs)]),
        "ibg_batch_size": (ctypes.c_int, [vp]),
        "ibg_batch_get_timing": (ctypes.c_int, [vp, dp, ctypes.POINTER(ctypes.c_longlong)]),
        "ibg_batch_last_error": (cp, [vp]),
        "ibg_batch_destroy": (None, [vp]),
        "ibg_get_tuning": (ctypes.c_int, [vp, ctypes.POINTER(Tuning)]),
        "ibg_set_tuning": (ctypes.c_int, [vp, ctypes.POINTER(Tuning)]),
        "ibg_autotune": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(Tuning), ctypes.POINTER(Tuning), dp,
                                         ctypes.c_int]),
        "ibg_device_bytes": (ctypes.c_longlong, [vp]),
        "ibg_estimate_bytes": (ctypes.c_longlong, [vp, ctypes.c_int, fp]),
        "ibg_server_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                             pvp]),
        "ibg_server_submit": (ctypes.c_int, [vp, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]),
        "ibg_server_wait": (ctypes.c_int, [vp, ctypes.c_longlong, ctypes.c_double]),
        "ibg_server_drain": (ctypes.c_int, [vp, ctypes.c_double]),
        "ibg_server_result": (ctypes.c_int, [vp, ctypes.c_longlong, fp, fp, ctypes.POINTER(IbgObs), dp]),
        "ibg_server_job_error": (cp, [vp, ctypes.c_longlong]),
        "ibg_server_get_stats": (ctypes.c_int, [vp, ctypes.POINTER(ServerStats)]),
        "ibg_server_destroy": (None, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return _lib


class IbiscoError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Setup:
    """The reference's setup phase run on the host from an input directory,
    or (files=) from the input files held in memory, {name: bytes or str}."""

    def __init__(self, directory: str = None, files: dict = None):
        L = lib()
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        if files is not None:
            items = [(k.encode(), v.encode() if isinstance(v, str) else bytes(v)) for k, v in files.items()]
            n = len(items)
            names = (ctypes.c_char_p * n)(*[k for k, _ in items])
            data = (ctypes.c_char_p * n)(*[v for _, v in items])
            sizes = (ctypes.c_long * n)(*[len(v) for _, v in items])
            rc = L.ibg_setup_read_mem(n, names, data, sizes, ctypes.byref(h), err, 512)
        else:
            rc = L.ibg_setup_read(directory.encode(), ctypes.byref(h), err, 512)
        if rc != 0:
            raise IbiscoError(rc, err.value.decode())
        self._h = h
        iv = np.zeros(8, np.int32)
        L.ibg_setup_control(h, _ip(iv), 8)
        self.nstep, self.ntrj, self.restart = int(iv[0]), int(iv[1]), int(iv[2])

    @property
    def handle(self):
        return self._h

    def desc(self):
        return lib().ibg_setup_desc(self._h)

    def array(self, name: str) -> np.ndarray:
        L = lib()
        n = L.ibg_setup_array_i(self._h, name.encode(), None, 0)
        if n >= 0:
            a = np.zeros(max(n, 1), np.int32)
            L.ibg_setup_array_i(self._h, name.encode(), _ip(a), n)
            return a[:n]
        n = L.ibg_setup_array_f(self._h, name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        a = np.zeros(max(n, 1), np.float32)
        L.ibg_setup_array_f(self._h, name.encode(), _fp(a), n)
        return a[:n]

    def set_nb_table(self, table: int, r, v):
        """Replace nonbonded table `table` (1-based) by rows r (nm), V (kJ/mol)."""
        r = np.ascontiguousarray(r, np.float32)
        v = np.ascontiguousarray(v, np.float32)
        rc = lib().ibg_setup_set_nb_table(self._h, int(table), len(r), _fp(r), _fp(v))
        if rc != 0:
            raise IbiscoError(rc, "ibg_setup_set_nb_table failed")

    def release(self):
        """Hand the setup over (to ibg_server_submit, which frees it)."""
        h, self._h = self._h, None
        return h

    def initial_state(self):
        itype = self.array("ITYPE")
        n = len(self.array("SXYZ")) // 3
        s = np.zeros((n, 3), np.float32)
        v = np.zeros((n, 3), np.float32)
        b = np.zeros(3, np.float32)
        lib().ibg_setup_initial_state(self._h, _fp(s), _fp(v), _fp(b))
        del itype
        return s, v, b

    def close(self):
        if getattr(self, "_h", None):
            if _lib is not None:  # None while the interpreter shuts down
                _lib.ibg_setup_free(self._h)
            self._h = None

    def __del__(self):
        self.close()


class System:
    """One system on the current CUDA device (``ibg_ctx``)."""

    def __init__(self, setup: Setup, precision: int = IBG_PREC_FP32_FIXED, **desc_overrides):
        L = lib()
        h = ctypes.c_void_p()
        desc = setup.desc()
        if desc_overrides:  # e.g. maxnab=...: a modified copy of the descriptor
            copy = IbgDesc.from_address(desc)
            copy = IbgDesc.from_buffer_copy(copy)
            for k, v in desc_overrides.items():
                setattr(copy, k, v)
            self._desc_copy = copy
            desc = ctypes.addressof(copy)
        rc = L.ibg_create(desc, int(precision), ctypes.byref(h))
        if rc != 0:
            raise IbiscoError(rc, "ibg_create failed")
        self._h = h
        self.setup = setup
        self.precision = precision
        s, _, _ = setup.initial_state()
        self.natoms = s.shape[0]
        self.nitems = len(setup.array("ITYPE"))

    def _check(self, rc: int):
        if rc != 0:
            raise IbiscoError(rc, lib().ibg_last_error(self._h).decode())

    def set_state(self, sxyz=None, vxyz=None, box=None):
        if sxyz is None or vxyz is None or box is None:
            s0, v0, b0 = self.setup.initial_state()
        s = np.ascontiguousarray(s0 if sxyz is None else sxyz, np.float32)
        v = np.ascontiguousarray(v0 if vxyz is None else vxyz, np.float32)
        b = np.ascontiguousarray(b0 if box is None else box, np.float32)
        self._check(lib().ibg_set_state(self._h, _fp(s), _fp(v), _fp(b)))

    def step(self, step: int) -> dict:
        o = IbgObs()
        self._check(lib().ibg_step(self._h, int(step), ctypes.byref(o)))
        return o.as_dict()

    def forces(self, step: int) -> dict:
        o = IbgObs()
        self._check(lib().ibg_forces(self._h, int(step), ctypes.byref(o)))
        return o.as_dict()

    def run(self, first: int, nsteps: int, observe: bool = False):
        if observe:
            arr = (IbgObs * max(nsteps, 1))()
            self._check(lib().ibg_run(self._h, int(first), int(nsteps), arr))
            return [arr[k].as_dict() for k in range(nsteps)]
        self._check(lib().ibg_run(self._h, int(first), int(nsteps), None))
        return None

    def state(self) -> dict:
        n, na = self.nitems, self.natoms
        s = np.zeros((n, 3), np.float32); r = np.zeros((n, 3), np.float32)
        f = np.zeros((n, 3), np.float32); v = np.zeros((na, 3), np.float32)
        self._check(lib().ibg_get_state(self._h, _fp(s), _fp(r), _fp(v), _fp(f)))
        return {"sxyz": s, "rxyz": r, "vxyz": v, "fxyz": f}

    def state64(self) -> dict:
        n, na = self.nitems, self.natoms
        s = np.zeros((n, 3)); f = np.zeros((n, 3)); v = np.zeros((na, 3))
        self._check(lib().ibg_get_state_f64(self._h, _dp(s), _dp(v), _dp(f)))
        return {"sxyz": s, "vxyz": v, "fxyz": f}

    def neighbour_list(self, which: int, maxnab: int = 1000):
        n = len(self.setup.array("ATOM")) if which == 0 else len(self.setup.array("BEAD"))
        lst = np.zeros((max(n, 1), maxnab), np.int32)
        nn = np.zeros(max(n, 1), np.int32)
        rc = lib().ibg_get_neighbour_list(self._h, which, _ip(lst), maxnab, _ip(nn))
        if rc < 0:
            self._check(rc)
        return lst[:n], nn[:n]

    def neighbour_counts(self, which: int) -> np.ndarray:
        """NNEBS of list `which` (0 atoms, 1 beads) alone."""
        n = len(self.setup.array("ATOM")) if which == 0 else len(self.setup.array("BEAD"))
        nn = np.zeros(max(n, 1), np.int32)
        rc = lib().ibg_get_neighbour_list(self._h, which, None, 0, _ip(nn))
        if rc < 0:
            self._check(rc)
        return nn[:n]

    def exclusions(self):
        n = self.nitems
        c = np.zeros(n, np.int32)
        t = np.zeros(n * 20, np.int32)
        self._check(lib().ibg_get_exclusions(self._h, _ip(c), _ip(t)))
        return c, t

    def timing(self) -> dict:
        ms = (ctypes.c_double * 9)()
        n = ctypes.c_longlong()
        lib().ibg_get_timing(self._h, ms, 9, ctypes.byref(n))
        return {"list_ms": ms[0], "nonbonded_ms": ms[1], "bonded_ms": ms[2], "integrate_ms": ms[3],
                "other_ms": ms[4], "run_ms": ms[5], "nonbonded_launches": int(ms[6]), "list_growths": int(ms[7]),
                "nonbonded_bead_launches": int(ms[8]), "launches": n.value}

    def tuning(self) -> dict:
        t = Tuning()
        self._check(lib().ibg_get_tuning(self._h, ctypes.byref(t)))
        return t.as_dict()

    def set_vsite_com(self, form: int):
        """Centre-of-mass virtual sites: IBG_VS_COM_FIXED (each site its centre
        of mass) or IBG_VS_COM_REFERENCE (VIRTUAL_DEF.f90:31 resets only the x
        sum).  Call before set_state."""
        self._check(lib().ibg_set_vsite_com(self._h, int(form)))

    def set_tuning(self, nb_tables_smem: int = 0, nb_blocks_per_sm: int = 0, nb_chunk: int = 0, nb_rows: int = 0,
                   nb_window: int = 0):
        t = Tuning(nb_tables_smem, nb_blocks_per_sm, nb_chunk, nb_rows, nb_window)
        self._check(lib().ibg_set_tuning(self._h, ctypes.byref(t)))

    def autotune(self, reps: int = 20):
        """Time the candidate tunings of the nonbonded kernel and keep the
        fastest; returns (best, [(candidate, us per launch)])."""
        best = Tuning()
        cap = 64
        cand = (Tuning * cap)()
        us = (ctypes.c_double * cap)()
        n = lib().ibg_autotune(self._h, int(reps), ctypes.byref(best), cand, us, cap)
        if n < 0:
            self._check(n)
        return best.as_dict(), [((c.nb_tables_smem, c.nb_blocks_per_sm, c.nb_chunk, c.nb_rows, c.nb_window), us[k])
                                for k, c in enumerate(cand[:min(n, cap)])]

    def set_timing(self, on: bool):
        self._check(lib().ibg_set_timing(self._h, 1 if on else 0))

    def set_list_form(self, form: int):
        """Verlet-list form of the FP32 path: LIST_AUTO (-1, the default:
        slice lists for lists of at least 2*64*32 particles per SM),
        LIST_PER_PARTICLE (0) or LIST_PER_SLICE (1).  The lists are rebuilt by
        the next set_state, which must follow."""
        self._check(lib().ibg_set_list_form(self._h, int(form)))

    def list_form(self) -> int:
        return int(lib().ibg_get_list_form(self._h))

    def set_l2_flush(self, nbytes: int):
        self._check(lib().ibg_set_l2_flush(self._h, int(nbytes)))

    def close(self):
        if getattr(self, "_h", None):
            if _lib is not None:  # None while the interpreter shuts down
                _lib.ibg_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class Batch:
    """Systems stepped together, one launch per stage (``ibg_batch``).

    Holds references to its ``System`` objects so that they outlive it."""

    def __init__(self, systems):
        self.systems = list(systems)
        arr = (ctypes.c_void_p * len(self.systems))(*[x._h.value for x in self.systems])
        h = ctypes.c_void_p()
        rc = lib().ibg_batch_create(arr, len(self.systems), ctypes.byref(h))
        if rc != 0:
            raise IbiscoError(rc, "ibg_batch_create failed")
        self._h = h

    def run(self, nsteps: int, last_step=None, observe: bool = False):
        n = len(self.systems)
        last = None
        if last_step is not None:
            last = np.ascontiguousarray(last_step, np.int32)
        obs = (IbgObs * n)() if observe else None
        rc = lib().ibg_batch_run(self._h, int(nsteps), _ip(last) if last is not None else None, obs)
        if rc != 0:
            raise IbiscoError(rc, lib().ibg_batch_last_error(self._h).decode())
        return [obs[k].as_dict() for k in range(n)] if observe else None

    def timing(self) -> dict:
        ms = ctypes.c_double()
        n = ctypes.c_longlong()
        lib().ibg_batch_get_timing(self._h, ctypes.byref(ms), ctypes.byref(n))
        return {"run_ms": ms.value, "launches": n.value}

    def close(self):
        if getattr(self, "_h", None):
            if _lib is not None:  # None while the interpreter shuts down
                _lib.ibg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class Server:
    """Continuous-batching service of simulation jobs on one GPU (``ibg_server``)."""

    def __init__(self, device: int = 0, precision: int = IBG_PREC_FP32_FIXED, hbm_budget: int = 0,
                 max_jobs: int = 64, tick_steps: int = 100):
        h = ctypes.c_void_p()
        rc = lib().ibg_server_create(int(device), int(precision), int(hbm_budget), int(max_jobs), int(tick_steps),
                                     ctypes.byref(h))
        if rc != 0:
            raise IbiscoError(rc, "ibg_server_create failed")
        self._h = h
        self._shapes = {}
        self._submitted = {}  # job -> time.perf_counter() at ibg_server_submit

    def submit(self, system, nsteps: int) -> int:
        """Queue a job: a system directory (the reference's input files, read
        here) or a Setup (made from files in memory, say), which the server
        takes over."""
        if isinstance(system, Setup):
            h = system.release()
        else:
            h = ctypes.c_void_p()
            err = ctypes.create_string_buffer(512)
            rc = lib().ibg_setup_read(system.encode(), ctypes.byref(h), err, 512)
            if rc != 0:
                raise IbiscoError(rc, err.value.decode())
        d = IbgDesc.from_address(lib().ibg_setup_desc(h))
        shape = (d.nitems, d.natoms)
        job = ctypes.c_longlong()
        t = time.perf_counter()
        rc = lib().ibg_server_submit(self._h, h, int(nsteps), ctypes.byref(job))
        if rc != 0:
            lib().ibg_setup_free(h)
            raise IbiscoError(rc, "ibg_server_submit failed")
        self._shapes[job.value] = shape
        self._submitted[job.value] = t
        return job.value

    def wait(self, job: int, timeout_s: float = -1.0) -> int:
        return lib().ibg_server_wait(self._h, int(job), float(timeout_s))

    def drain(self, timeout_s: float = -1.0) -> bool:
        return lib().ibg_server_drain(self._h, float(timeout_s)) == 0

    def result(self, job: int) -> dict:
        nitems, natoms = self._shapes[job]
        s = np.zeros((nitems, 3), np.float32)
        v = np.zeros((natoms, 3), np.float32)
        o = IbgObs()
        t = (ctypes.c_double * 3)()
        rc = lib().ibg_server_result(self._h, int(job), _fp(s), _fp(v), ctypes.byref(o), t)
        if rc != 0:
            raise IbiscoError(rc, lib().ibg_server_job_error(self._h, int(job)).decode())
        return {"sxyz": s, "vxyz": v, "obs": o.as_dict(), "queued_s": t[0], "run_s": t[1], "latency_s": t[2],
                "submitted_at": self._submitted[job]}

    def stats(self) -> dict:
        st = ServerStats()
        lib().ibg_server_get_stats(self._h, ctypes.byref(st))
        return st.as_dict()

    def close(self):
        if getattr(self, "_h", None):
            if _lib is not None:  # None while the interpreter shuts down
                _lib.ibg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class Trajectory:
    """A TRZ trajectory file written as WRITETRJ.F90 writes it (ibg_trz_*)."""

    def __init__(self, setup: Setup, path: str):
        h = ctypes.c_void_p()
        rc = lib().ibg_trz_open(setup.handle, path.encode(), ctypes.byref(h))
        if rc != 0:
            raise IbiscoError(rc, f"cannot open {path}")
        self._h = h
        self.setup = setup

    def write(self, step: int, obs: "IbgObs", sxyz, vxyz):
        s = np.ascontiguousarray(sxyz, np.float32)
        v = np.ascontiguousarray(vxyz, np.float32)
        rc = lib().ibg_trz_write(self._h, int(step), ctypes.byref(obs), _fp(s), _fp(v))
        if rc != 0:
            raise IbiscoError(rc, "ibg_trz_write failed")

    def close(self):
        if getattr(self, "_h", None):
            if _lib is not None:  # None while the interpreter shuts down
                _lib.ibg_trz_close(self._h)
            self._h = None

    def __del__(self):
        self.close()


def write_restart(setup: Setup, path: str, step: int, box, sxyz, vxyz):
    """The restart file of WRITE_RESTART (coordinate format) for this state."""
    b = np.ascontiguousarray(box, np.float32)
    s = np.ascontiguousarray(sxyz, np.float32)
    v = np.ascontiguousarray(vxyz, np.float32)
    rc = lib().ibg_write_restart(setup.handle, path.encode(), int(step), _fp(b), _fp(s), _fp(v))
    if rc != 0:
        raise IbiscoError(rc, f"cannot write {path}")


def run_with_output(g: "System", first: int, nsteps: int, trz_path: str, restart_path: str = None,
                    ntrj: int = None):
    """Steps first..first+nsteps-1 in runs of NTRJ steps (the control file's
    trajectory interval unless given); after each run a TRZ frame of its last
    step and, when restart_path is given, the restart file, as NEW_LOOP.F90
    calls WRITETRJ every NTRJ steps.  Each run's observables come from the
    device's per-step ring (ibg_run) and its state from ibg_get_state.
    Returns the observables of every step."""
    ntrj = ntrj or g.setup.ntrj
    trz = Trajectory(g.setup, trz_path)
    out = []
    st = first
    last = first + nsteps - 1
    while st <= last:
        end = min(last, -(-st // ntrj) * ntrj)  # the next step that writes output
        arr = (IbgObs * (end - st + 1))()
        g._check(lib().ibg_run(g._h, int(st), int(end - st + 1), arr))
        out += [arr[k].as_dict() for k in range(end - st + 1)]
        if end % ntrj == 0:
            x = g.state()
            trz.write(end, arr[end - st], x["sxyz"][: g.natoms], x["vxyz"])
            if restart_path:
                write_restart(g.setup, restart_path, end, [arr[end - st].box[k] for k in range(3)],
                              x["sxyz"][: g.natoms], x["vxyz"])
        st = end + 1
    trz.close()
    return out


def tune_steps(make_system, candidates, steps: int = 100, l2_flush: int = 0):
    """Pick one system's launch tuning by whole steps: for each candidate
    tuning (a dict for System.set_tuning), make the system (make_system()
    returns a fresh System after set_state), apply it, run 10 + `steps` steps
    (with the L2 flushed before each, if l2_flush > 0) and keep the fastest.
    The list build, positions and bonded kernels of a step leave the L2 in the
    state the nonbonded kernel meets, which timing its launches alone does not
    reproduce.  Returns (best tuning, [(tuning, us per step)])."""
    times = []
    for tun in candidates:
        g = make_system()
        g.set_tuning(**tun)
        if l2_flush:
            g.set_l2_flush(l2_flush)
        g.run(1, 10)
        g.run(11, steps)
        times.append((tun, 1000.0 * g.timing()["run_ms"] / steps))
        g.close()
    return min(times, key=lambda t: t[1])[0], times


def tune_batch(make_systems, candidates, steps: int = 100):
    """Pick the launch tuning of a batch by timing: for each candidate tuning
    (a dict for System.set_tuning), make the systems (make_systems() returns
    fresh Systems after set_state), apply it, run `steps` batch steps and keep
    the fastest.  Returns (best tuning, [(tuning, us per batch step)])."""
    times = []
    for tun in candidates:
        systems = make_systems()
        for x in systems:
            x.set_tuning(**tun)
        b = Batch(systems)
        b.run(10)
        b.run(steps)
        times.append((tun, 1000.0 * b.timing()["run_ms"] / steps))
        b.close()
        for x in systems:
            x.close()
    return min(times, key=lambda t: t[1])[0], times
