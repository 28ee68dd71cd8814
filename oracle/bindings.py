"""ctypes bindings for the two CPU oracles (TEST INFRASTRUCTURE).

* ``COracle``   - oracle/build/liboracle.so, the plain-C restatement (hpc_oracle.c).
* ``RefOracle`` - oracle/_ref/libhpcref.so, the reference HPCrack sources compiled
                  as they are (plus a single-rank MPI stand-in), driven through
                  oracle/ref_harness.cpp.

Both expose the same methods over the same field ids, so a test scenario can be
run on either.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg use this module; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libhpcref.so")

# field ids shared by hpc_oracle.h and ref_harness.cpp
BULK, G, GC, D, H, FD, KE, GE, R, DOLD, DOLDF = 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10
U, FU, RU, UOLD = 16, 17, 18, 19
VECTOR_FIELDS = (U, FU, RU, UOLD)

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build(quiet: bool = True, ref: str | None = None) -> None:
    """Compile the oracles (make -C oracle).  `ref` is the reference source tree; the reference part
    is skipped when it is not given or its sources are absent, keeping any prebuilt
    oracle/_ref/libhpcref.so."""
    cmd = ["make", "-C", HERE, "all"] + ([f"REF={ref}"] if ref else [])
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _ptr(a: np.ndarray, ctype=C.c_double):
    return a.ctypes.data_as(C.POINTER(ctype))


def _i3(v):
    return (C.c_int * 3)(*[int(x) for x in v])


def _d3(v):
    return (C.c_double * 3)(*[float(x) for x in v])


class _Base:
    prefix = ""
    so_path = ""
    _lib_cache: dict = {}

    def __init__(self, maxlevel, enb, x0=(0.0, 0.0, 0.0), roi=(0, 0, 0)):
        self.lib = self._load()
        self.maxlevel = int(maxlevel)
        self.enb = tuple(int(e) for e in enb)
        self.h = self._create(self.maxlevel, _i3(enb), _d3(x0), _i3(roi))
        if not self.h:
            raise RuntimeError("oracle context creation failed")
        self.dims = []
        for l in range(self.maxlevel + 1):
            self.dims.append(tuple(e * (1 << l) + 1 for e in self.enb))

    # --- library plumbing ---
    @classmethod
    def _load(cls):
        if cls.so_path not in cls._lib_cache:
            if not os.path.exists(cls.so_path):
                raise FileNotFoundError(cls.so_path + " missing: run make -C oracle")
            lib = C.CDLL(cls.so_path)
            cls._declare(lib)
            cls._lib_cache[cls.so_path] = lib
        return cls._lib_cache[cls.so_path]

    @classmethod
    def _declare(cls, lib):
        p = cls.prefix
        vp = C.c_void_p
        sig = {
            "set": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, _dp]),
            "get": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, _dp]),
            "set_choice": (C.c_int, [vp, C.c_int, C.POINTER(C.c_short)]),
            "get_choice": (C.c_int, [vp, C.c_int, C.POINTER(C.c_short)]),
            "initial_residual_u": (C.c_double, [vp, C.c_int, C.c_double]),
            "pcg_u": (C.c_int, [vp, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, _dp]),
            "initial_residual_d": (C.c_double, [vp, C.c_int, C.c_double]),
            "pcg_d": (C.c_int, [vp, C.c_int, C.c_double, C.c_int, C.c_int, _dp]),
            "cycle_u": (C.c_int, [vp, C.c_int, _ip, C.c_double, C.c_double, C.c_int, _dp]),
            "cycle_d": (C.c_int, [vp, C.c_int, _ip, C.c_double, C.c_int, _dp]),
            "mp_choice": (None, [vp]),
            "mp_all_element": (None, [vp, C.c_double]),
            "vr_all_level": (C.c_int, [vp, C.c_int]),
            "voigt_all_level": (C.c_int, [vp, C.c_int]),
            "coarse_vr": (C.c_int, [vp, C.c_int]),
            "strain_history": (None, [vp, C.c_double, C.c_double]),
            "fd_h": (None, [vp, C.c_int]),
            "delta_d_max": (C.c_double, [vp]),
            "d_max": (C.c_double, [vp]),
            "U_e": (C.c_double, [vp, C.c_double]),
            "externe_force_nodal": (None, [vp, C.c_double, C.c_double]),
            "externe_force_sum": (C.c_double, [vp]),
            "initial_crack": (None, [vp, C.c_double, C.c_int]),
            "dirichlet_bd": (C.c_int, [vp, C.c_int, C.c_int, C.c_double]),
            "dirichlet_force": (C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
            "dirichlet_residual": (C.c_int, [vp, C.c_int, C.c_int]),
            "solution_injection": (C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
            "coarsen_f_standard": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "refine_standard": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
        }
        sig.update(cls._extra_sigs())
        for name, (res, args) in sig.items():
            fn = getattr(lib, cls._cname(name))
            fn.restype = res
            fn.argtypes = args

    @classmethod
    def _cname(cls, name):
        return cls.prefix + name

    @classmethod
    def _extra_sigs(cls):
        return {}

    def _f(self, name):
        return getattr(self.lib, self._cname(name))

    # --- fields ---
    def n(self, level):
        d = self.dims[level]
        return d[0] * d[1] * d[2]

    def set(self, field, level, arr):
        """Upload a field.  Vector fields take an array of shape (3, n) or (3*n,)."""
        nn = self.n(level)
        if field in VECTOR_FIELDS:
            a = np.ascontiguousarray(arr, dtype=np.float64).reshape(3, nn)
            for c in range(3):
                row = np.ascontiguousarray(a[c])
                assert self._f("set")(self.h, field, level, c, _ptr(row)) == 0
        else:
            a = np.ascontiguousarray(arr, dtype=np.float64).reshape(nn)
            assert self._f("set")(self.h, field, level, 0, _ptr(a)) == 0

    def get(self, field, level):
        nn = self.n(level)
        if field in VECTOR_FIELDS:
            out = np.empty((3, nn))
            for c in range(3):
                row = np.empty(nn)
                assert self._f("get")(self.h, field, level, c, _ptr(row)) == 0
                out[c] = row
            return out
        out = np.empty(nn)
        assert self._f("get")(self.h, field, level, 0, _ptr(out)) == 0
        return out

    def set_choice(self, level, arr):
        a = np.ascontiguousarray(arr, dtype=np.int16).reshape(self.n(level))
        self._f("set_choice")(self.h, level, _ptr(a, C.c_short))

    def get_choice(self, level):
        a = np.empty(self.n(level), dtype=np.int16)
        self._f("get_choice")(self.h, level, _ptr(a, C.c_short))
        return a

    # --- operators ---
    def internal_force(self, level, src, dst, small_k):
        assert self._f(self._op("internal_force"))(self.h, level, src, dst, C.c_double(small_k)) == 0

    def prem_u(self, level, dst, small_k):
        assert self._f(self._op("prem_u"))(self.h, level, dst, C.c_double(small_k)) == 0

    def fld(self, level, src, dst, lc):
        assert self._f(self._op("fld"))(self.h, level, src, dst, C.c_double(lc)) == 0

    def precondition_m(self, level, dst, lc):
        assert self._f(self._op("precondition_m"))(self.h, level, dst, C.c_double(lc)) == 0

    def _op(self, name):
        return name

    def initial_residual_u(self, level, small_k):
        return self._f("initial_residual_u")(self.h, level, small_k)

    def pcg_u(self, level, small_k, Ut, nb_relax, t, f_norm):
        fn = C.c_double(f_norm)
        it = self._f("pcg_u")(self.h, level, small_k, Ut, nb_relax, t, C.byref(fn))
        return it, fn.value

    def initial_residual_d(self, level, lc):
        return self._f("initial_residual_d")(self.h, level, lc)

    def pcg_d(self, level, lc, nb_relax, t, fd_norm):
        fn = C.c_double(fd_norm)
        it = self._f("pcg_d")(self.h, level, lc, nb_relax, t, C.byref(fn))
        return it, fn.value

    def cycle_u(self, level, mg5, small_k, Ut, t, f_norm):
        fn = C.c_double(f_norm)
        it = self._f("cycle_u")(self.h, level, (C.c_int * 5)(*mg5), small_k, Ut, t, C.byref(fn))
        return it, fn.value

    def cycle_d(self, level, mg5, lc, t, fd_norm):
        fn = C.c_double(fd_norm)
        it = self._f("cycle_d")(self.h, level, (C.c_int * 5)(*mg5), lc, t, C.byref(fn))
        return it, fn.value

    def mp_choice(self):
        self._f("mp_choice")(self.h)

    def mp_all_element(self, small_k):
        self._f("mp_all_element")(self.h, small_k)

    def vr_all_level(self, field):
        assert self._f("vr_all_level")(self.h, field) == 0

    def voigt_all_level(self, field):
        assert self._f("voigt_all_level")(self.h, field) == 0

    def coarse_vr(self, field):
        assert self._f("coarse_vr")(self.h, field) == 0

    def strain_history(self, lc, u_proportion):
        self._f("strain_history")(self.h, lc, u_proportion)

    def fd_h(self, level):
        self._f("fd_h")(self.h, level)

    def delta_d_max(self):
        return self._f("delta_d_max")(self.h)

    def d_max(self):
        return self._f("d_max")(self.h)

    def U_e(self, lc):
        return self._f("U_e")(self.h, lc)

    def externe_force_nodal(self, Ut, small_k):
        self._f("externe_force_nodal")(self.h, Ut, small_k)

    def externe_force_sum(self):
        return self._f("externe_force_sum")(self.h)

    def initial_crack(self, H_crack, level):
        self._f("initial_crack")(self.h, H_crack, level)

    def dirichlet_bd(self, level, field, Ut):
        assert self._f("dirichlet_bd")(self.h, level, field, Ut) == 0

    def dirichlet_force(self, level, f_field, fi_field):
        assert self._f("dirichlet_force")(self.h, level, f_field, fi_field) == 0

    def dirichlet_residual(self, level, field):
        assert self._f("dirichlet_residual")(self.h, level, field) == 0

    def solution_injection(self, field, comp, lf):
        assert self._f("solution_injection")(self.h, field, comp, lf) == 0

    def coarsen_f_standard(self, fc_field, rf_field, fic_field, comp, lf):
        assert self._f("coarsen_f_standard")(self.h, fc_field, rf_field, fic_field, comp, lf) == 0

    def refine_standard(self, uf_field, uc_field, ucold_field, comp, lf):
        assert self._f("refine_standard")(self.h, uf_field, uc_field, ucold_field, comp, lf) == 0

    def state(self):
        s = (C.c_double * 6)()
        self._f("state" if self.prefix == "ref_" else "state_scalars")(self.h, s)
        return list(s)

    def set_state(self, s6):
        self._f("set_state" if self.prefix == "ref_" else "set_state_scalars")(self.h, (C.c_double * 6)(*s6))


class COracle(_Base):
    """The plain-C restatement (hpc_oracle.c)."""

    prefix = "orc_"
    so_path = ORACLE_SO

    @classmethod
    def _extra_sigs(cls):
        vp = C.c_void_p
        return {
            "state_create": (vp, [C.c_int, _ip, _dp, _ip]),
            "state_destroy": (None, [vp]),
            "st_internal_force": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_double]),
            "st_prem_u": (C.c_int, [vp, C.c_int, C.c_int, C.c_double]),
            "st_fld": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_double]),
            "st_precondition_m": (C.c_int, [vp, C.c_int, C.c_int, C.c_double]),
            "u_entire": (C.c_int, [vp, _ip, C.c_double, C.c_double, C.c_int, _dp, _ip, C.c_double]),
            "phase_field": (C.c_int, [vp, _ip, C.c_double, C.c_int, _dp, _ip, C.c_double]),
            "state_scalars": (None, [vp, _dp]),
            "set_state_scalars": (None, [vp, _dp]),
            "set_choice_quirk": (None, [vp, C.c_int]),
            "image_material": (C.c_int, [vp, C.POINTER(C.c_ubyte), _ip, C.c_int, _ip, _dp, _dp, _dp,
                                         C.c_double]),
            "step": (C.c_int, [vp, C.c_int, _ip, _ip, C.c_double, C.c_double, C.c_double, C.c_double,
                               C.c_double, C.c_double, C.c_double, C.c_double, _dp]),
        }

    def _create(self, maxlevel, enb, x0, roi):
        return self.lib.orc_state_create(maxlevel, enb, x0, roi)

    def _op(self, name):
        return "st_" + name

    def close(self):
        if getattr(self, "h", None):
            self.lib.orc_state_destroy(self.h)
            self.h = None

    __del__ = close

    def set_choice_quirk(self, reproduce: bool):
        self.lib.orc_set_choice_quirk(self.h, int(bool(reproduce)))

    def u_entire(self, mg5, small_k, Ut, t, f_norm, mech_tol=1e-6):
        fn = C.c_double(f_norm)
        it = C.c_int(0)
        cy = self.lib.orc_u_entire(self.h, (C.c_int * 5)(*mg5), small_k, Ut, t, C.byref(fn), C.byref(it),
                                   mech_tol)
        return cy, it.value, fn.value

    def phase_field(self, mg5, lc, t, fd_norm, pf_tol=1e-12):
        fn = C.c_double(fd_norm)
        it = C.c_int(0)
        cy = self.lib.orc_phase_field(self.h, (C.c_int * 5)(*mg5), lc, t, C.byref(fn), C.byref(it), pf_tol)
        return cy, it.value, fn.value

    def image_material(self, image, voxel_n, table, voxel_size):
        gray, E, nu, gcv = table
        img = np.ascontiguousarray(image, dtype=np.uint8).ravel()
        g = np.ascontiguousarray(gray, dtype=np.int32)
        E = np.ascontiguousarray(E, dtype=np.float64)
        nu = np.ascontiguousarray(nu, dtype=np.float64)
        gcv = np.ascontiguousarray(gcv, dtype=np.float64)
        rc = self.lib.orc_image_material(self.h, _ptr(img, C.c_ubyte), _i3(voxel_n), len(g), _ptr(g, C.c_int),
                                         _ptr(E), _ptr(nu), _ptr(gcv), voxel_size)
        if rc != 0:
            raise ValueError("gray level outside the material table")

    def step(self, t, mg_u, mg_d, small_k, lc, voxel_size, ut0=0.0, dU=0.0, dU_factor=1.5e-3,
             mech_tol=1e-6, pf_tol=1e-12):
        out = (C.c_double * 8)()
        rc = self.lib.orc_step(self.h, t, (C.c_int * 5)(*mg_u), (C.c_int * 5)(*mg_d), small_k, lc,
                               voxel_size, ut0, dU, dU_factor, mech_tol, pf_tol, out)
        if rc != 0:
            raise RuntimeError("oracle step failed (zero diagonal)")
        return list(out)


class RefOracle(_Base):
    """The reference HPCrack sources compiled as they are (oracle/_ref)."""

    prefix = "ref_"
    so_path = REF_SO

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.so_path)

    @classmethod
    def _extra_sigs(cls):
        vp = C.c_void_p
        return {
            "ctx_create": (vp, [C.c_int, _ip, _dp, _ip]),
            "ctx_destroy": (None, [vp]),
            "set_quiet": (None, [C.c_int]),
            "set_threads": (None, [C.c_int]),
            "get_threads": (C.c_int, []),
            "level_info": (None, [vp, C.c_int, _ip, _dp, C.POINTER(C.c_long)]),
            "domain": (None, [vp, _dp]),
            "internal_force": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_double]),
            "prem_u": (C.c_int, [vp, C.c_int, C.c_int, C.c_double]),
            "fld": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_double]),
            "precondition_m": (C.c_int, [vp, C.c_int, C.c_int, C.c_double]),
            "u_entire": (C.c_int, [vp, _ip, C.c_double, C.c_double, C.c_int, _dp, _ip]),
            "phase_field": (C.c_int, [vp, _ip, C.c_double, C.c_int, _dp, _ip]),
            "state": (None, [vp, _dp]),
            "set_state": (None, [vp, _dp]),
            "input_total": (C.c_int, [vp, C.c_char_p, C.c_char_p, _ip, C.c_double]),
            "step": (C.c_int, [vp, C.c_int, _ip, _ip, C.c_double, C.c_double, C.c_double, C.c_double,
                               C.c_double, C.c_double, C.c_double, C.c_double, _dp]),
            "u_entire_tol": (C.c_int, [vp, _ip, C.c_double, C.c_double, C.c_int, _dp, _ip, C.c_double]),
            "phase_field_tol": (C.c_int, [vp, _ip, C.c_double, C.c_int, _dp, _ip, C.c_double]),
            "last_output": (C.c_char_p, []),
            "write_vector_3d": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_int]),
            "read_vector_3d": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_int]),
            "write_vtk": (C.c_int, [vp, C.c_char_p, C.c_int, C.c_int, C.c_char_p, C.c_char_p, C.c_int,
                                    C.c_double, C.c_char_p]),
        }

    def _create(self, maxlevel, enb, x0, roi):
        return self.lib.ref_ctx_create(maxlevel, enb, x0, roi)

    def close(self):
        if getattr(self, "h", None):
            self.lib.ref_ctx_destroy(self.h)
            self.h = None

    __del__ = close

    def set_threads(self, n):
        self.lib.ref_set_threads(int(n))

    def level_info(self, level):
        n3 = (C.c_int * 3)()
        h3 = (C.c_double * 3)()
        e3 = (C.c_long * 3)()
        self.lib.ref_level_info(self.h, level, n3, h3, e3)
        return tuple(n3), tuple(h3), tuple(e3)

    def domain(self):
        b = (C.c_double * 6)()
        self.lib.ref_domain(self.h, b)
        return tuple(b)

    def u_entire(self, mg5, small_k, Ut, t, f_norm, mech_tol=1e-6):
        """The reference's u_entire at its own threshold (1e-6); any other threshold goes through
        the harness driver that makes u_entire's calls with the threshold as a parameter."""
        fn = C.c_double(f_norm)
        it = C.c_int(0)
        if mech_tol == 1e-6:
            cy = self.lib.ref_u_entire(self.h, (C.c_int * 5)(*mg5), small_k, Ut, t, C.byref(fn), C.byref(it))
        else:
            cy = self.lib.ref_u_entire_tol(self.h, (C.c_int * 5)(*mg5), small_k, Ut, t, C.byref(fn), C.byref(it),
                                           mech_tol)
        return cy, it.value, fn.value

    def phase_field(self, mg5, lc, t, fd_norm, pf_tol=1e-12):
        fn = C.c_double(fd_norm)
        it = C.c_int(0)
        if pf_tol == 1e-12:
            cy = self.lib.ref_phase_field(self.h, (C.c_int * 5)(*mg5), lc, t, C.byref(fn), C.byref(it))
        else:
            cy = self.lib.ref_phase_field_tol(self.h, (C.c_int * 5)(*mg5), lc, t, C.byref(fn), C.byref(it), pf_tol)
        return cy, it.value, fn.value

    def input_total(self, workdir, raw_path, voxel_n, voxel_size):
        rc = self.lib.ref_input_total(self.h, workdir.encode(), raw_path.encode(), _i3(voxel_n), voxel_size)
        if rc != 0:
            raise RuntimeError(f"ref_input_total failed ({rc})")

    def step(self, t, mg_u, mg_d, small_k, lc, voxel_size, ut0=0.0, dU=0.0, dU_factor=1.5e-3,
             mech_tol=1e-6, pf_tol=1e-12):
        out = (C.c_double * 8)()
        self.lib.ref_step(self.h, t, (C.c_int * 5)(*mg_u), (C.c_int * 5)(*mg_d), small_k, lc, voxel_size,
                          ut0, dU, dU_factor, mech_tol, pf_tol, out)
        return list(out)

    def last_output(self) -> str:
        return self.lib.ref_last_output().decode(errors="replace")

    def write_vector_3d(self, field, level, comp, path, t=0):
        """The reference's write_vector_3D (write_read_history.cpp:18-53) of one grid to `path`."""
        if self.lib.ref_write_vector_3d(self.h, field, level, comp, path.encode(), t) != 0:
            raise ValueError("bad field")

    def read_vector_3d(self, field, level, comp, path, t=0):
        """The reference's read_vector_3D (write_read_history.cpp:55-86) of `path` into one grid."""
        if self.lib.ref_read_vector_3d(self.h, field, level, comp, path.encode(), t) != 0:
            raise ValueError("bad field")

    def write_vtk(self, option, field, level, filename, field_name, t, workdir, u_proportion=1.0):
        """The reference's write_total_de ("S"), write_total_u ("V") or write_total_H ("C")
        (vtk_output.cpp:420-469), one rank, writing below `workdir`/Output."""
        if self.lib.ref_write_vtk(self.h, option.encode(), field, level, filename.encode(), field_name.encode(),
                                  t, u_proportion, workdir.encode()) != 0:
            raise ValueError("bad option, field or workdir")
