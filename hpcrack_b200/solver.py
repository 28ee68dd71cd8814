"""Host-side mirror of HPCrack's solver interface over the B200 library.

:class:`Hierarchy` owns one device context (the mg / mgvec containers of the
reference: crack_propagation.cpp:40-45) and exposes the reference's operations
under their own names - ``internal_force`` (Internal_Force), ``pcg_u``,
``cycle_u``, ``u_entire``, ``fld``, ``pcg_d``, ``cycle_d``, ``phase_field``,
``strain_history``, ``fd_h``, ``delta_d_max``, ... - with the same argument
meaning.  Arrays cross the boundary in the reference's layout: x-fastest
nx*ny*nz doubles per level, vector fields as (3, n).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib as _L

# field ids (include/hpcrack.h enum hpc_field)
BULK, G, GC, D, H, FD, KE, GE, R, DOLD, DOLDF = 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10
U, FU, RU, UOLD = 16, 17, 18, 19
VECTOR_FIELDS = (U, FU, RU, UOLD)
KC_MECH_PCG_FINEST, KC_PF_PCG_FINEST, KC_MECH_UPDATE_FINEST, KC_MECH32_PCG_FINEST = 0, 1, 2, 3
MECH_FAS, MECH_FCG, MECH_MIXED = 0, 1, 2  # hpc_step_params.mech_solver
# V-cycle (nu0, nu1, nu2, gamma) of the flexible forms' preconditioner: more post-smoothing than the
# reference's V(4, 2) pays off once the cycle is a preconditioner (257^3 specimen, precision form:
# V(4,2) 1.15 solves/s, V(4,4) 1.31)
PRECISION_MG = (50, 4, 4, 1)
# Coarsest iterations when the coarsest level is too large for the one-block solver: there each
# iteration costs three launches, and a 20-iteration coarse solve is the better preconditioner per
# unit time (64-specimen mix: 50 iterations 4.2-4.8 solves/s, 20 iterations 5.9; 10 iterations 2.3).
# With a one-block coarsest solve (e.g. 9^3 under a 257^3 specimen) 50 stays best (1.35 vs 0.84).
PRECISION_NU0_LARGE_COARSEST = 20


def coarsest_in_one_block(maxlevel: int, element_nb) -> bool:
    """Whether the library solves the coarsest level in one thread block (the rule of
    coarse_pcg_fits in coarse_kernels.cu: 15 N + 26 E + 33 doubles of shared memory, at most 220 KiB,
    and a coarsest level below the finest)."""
    e = [int(v) for v in element_nb]
    n_nodes = (e[0] + 1) * (e[1] + 1) * (e[2] + 1)
    n_elem = e[0] * e[1] * e[2]
    return maxlevel >= 1 and 8 * (15 * n_nodes + 26 * n_elem + 33) <= 220 * 1024


def precision_mg(maxlevel: int, element_nb, ncy: int) -> tuple:
    """The flexible forms' preconditioner cycle for a hierarchy (PRECISION_MG, with fewer coarsest
    iterations when the coarsest level does not fit one thread block)."""
    nu0 = PRECISION_MG[0] if coarsest_in_one_block(maxlevel, element_nb) else PRECISION_NU0_LARGE_COARSEST
    return (nu0,) + tuple(PRECISION_MG[1:]) + (int(ncy),)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def mg_params(mg5) -> _L.hpc_mg:
    """(nu0, nu1, nu2, gamma, ncy) -> hpc_mg (the reference's MG struct, mg.h:18-25)."""
    return _L.hpc_mg(*[int(v) for v in mg5])


def step_params(t, mg_u, mg_d, small_k, lc, voxel_size, ut0=0.0, dU=0.0, dU_factor=1.5e-3, mech_tol=1e-6,
                pf_tol=1e-12, mech_solver=MECH_FAS) -> _L.hpc_step_params:
    """hpc_step_params of one staggered increment (the arguments of Hierarchy.step)."""
    return _L.hpc_step_params(int(t), mg_params(mg_u), mg_params(mg_d), small_k, lc, voxel_size, ut0, dU, dU_factor,
                              mech_tol, pf_tol, int(mech_solver))


class Batch:
    """hpc_batch: one staggered increment of many specimens per call (hpc_batch_step).

    Every specimen's mechanical and phase-field solve runs as a device-driven loop inside one CUDA graph
    per batch (one launch per solve phase for all specimens, each converging at its own pace); the
    results are the same bits as Hierarchy.step on each specimen alone."""

    def __init__(self):
        self.lib = _L.load()
        h = C.c_void_p()
        _L.check("hpc_batch_create", self.lib.hpc_batch_create(C.byref(h)))
        self.h = h

    def step(self, hiers, params):
        """Advances hiers[i] by the increment params[i] (step_params); returns one 8-value output per
        specimen, as Hierarchy.step returns."""
        n = len(hiers)
        ctxs = (C.c_void_p * n)(*[hh.h.value for hh in hiers])
        ps = (_L.hpc_step_params * n)(*params)
        out = (C.c_double * (8 * n))()
        _L.check("hpc_batch_step", self.lib.hpc_batch_step(self.h, ctxs, n, ps, out))
        return [list(out[8 * i:8 * i + 8]) for i in range(n)]

    def timing(self, on=None) -> dict:
        """hpc_batch_timing: cumulative host seconds (enqueue/read, graph builds, graph waits when
        on) and counts of graph builds and launches; on=True/False switches the per-launch wait."""
        out = (C.c_double * 5)()
        _L.check("hpc_batch_timing", self.lib.hpc_batch_timing(self.h, -1 if on is None else int(bool(on)), out))
        return {"host_s": out[0], "build_s": out[1], "wait_s": out[2], "builds": int(out[3]), "launches": int(out[4])}

    def close(self):
        if getattr(self, "h", None):
            self.lib.hpc_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def slab_level(maxlevel, enb, nranks, rank, level):
    """(local nz, global z of local plane 0, first owned plane, one past the last) of a z-slab rank on
    `level` (hpc_slab_level; host only)."""
    lib = _L.load()
    geo = _L.hpc_geometry(int(maxlevel), (C.c_int * 3)(*map(int, enb)), (C.c_double * 3)(0.0, 0.0, 0.0),
                          (C.c_int * 3)(0, 0, 0))
    out = (C.c_int * 4)()
    _L.check("hpc_slab_level", lib.hpc_slab_level(C.byref(geo), int(nranks), int(rank), int(level), out))
    return tuple(out)


class Hierarchy:
    """Device-resident multigrid hierarchy of one specimen."""

    def __init__(self, maxlevel, enb, x0=(0.0, 0.0, 0.0), roi=(0, 0, 0), device: int = 0, slab=None):
        """slab = (nranks, rank): this context holds rank `rank`'s z planes of a specimen split over
        `nranks` ranks (hpc_create_slab); its arrays (dims, set, get) are the local ones, ghost planes
        included, and it joins a transport (hpcrack_b200.slab) before it solves."""
        self.lib = _L.load()
        self.maxlevel = int(maxlevel)
        self.enb = tuple(int(e) for e in enb)
        self.geo = _L.hpc_geometry(self.maxlevel, (C.c_int * 3)(*self.enb), (C.c_double * 3)(*map(float, x0)),
                                   (C.c_int * 3)(*map(int, roi)))
        h = C.c_void_p()
        self.dims = [tuple(e * (1 << l) + 1 for e in self.enb) for l in range(self.maxlevel + 1)]
        self.slab = None
        if slab is None:
            _L.check("hpc_create", self.lib.hpc_create(C.byref(h), C.byref(self.geo), int(device)))
        else:
            nranks, rank = int(slab[0]), int(slab[1])
            _L.check("hpc_create_slab", self.lib.hpc_create_slab(C.byref(h), C.byref(self.geo), int(device), nranks,
                                                                 rank))
            self.slab = (nranks, rank)
            self.plans = [slab_level(self.maxlevel, self.enb, nranks, rank, l) for l in range(self.maxlevel + 1)]
            self.dims = [(d[0], d[1], p[0]) for d, p in zip(self.dims, self.plans)]
        self.h = h

    # ------------------------------------------------------------ lifetime
    def close(self):
        if getattr(self, "h", None):
            self.lib.hpc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def footprint(maxlevel, enb, x0=(0.0, 0.0, 0.0), roi=(0, 0, 0), slab=None) -> int:
        """Device bytes of a context (hpc_footprint), or of one rank's slab: slab = (nranks, rank)."""
        lib = _L.load()
        geo = _L.hpc_geometry(int(maxlevel), (C.c_int * 3)(*map(int, enb)), (C.c_double * 3)(*map(float, x0)),
                              (C.c_int * 3)(*map(int, roi)))
        out = C.c_size_t(0)
        if slab is None:
            _L.check("hpc_footprint", lib.hpc_footprint(C.byref(geo), C.byref(out)))
        else:
            _L.check("hpc_footprint_slab", lib.hpc_footprint_slab(C.byref(geo), int(slab[0]), int(slab[1]),
                                                                  C.byref(out)))
        return out.value

    def _c(self, name, *args):
        _L.check(name, getattr(self.lib, name)(self.h, *args))

    # ------------------------------------------------------------ fields
    def n(self, level):
        d = self.dims[level]
        return d[0] * d[1] * d[2]

    def level_dims(self, level):
        n3 = (C.c_int * 3)()
        h3 = (C.c_double * 3)()
        self._c("hpc_level_dims", level, n3, h3)
        return tuple(n3), tuple(h3)

    def set(self, field, level, arr):
        nn = self.n(level)
        if field in VECTOR_FIELDS:
            a = np.ascontiguousarray(arr, dtype=np.float64).reshape(3, nn)
            for c in range(3):
                row = np.ascontiguousarray(a[c])
                self._c("hpc_upload", field, level, c, _dptr(row))
        else:
            a = np.ascontiguousarray(arr, dtype=np.float64).reshape(nn)
            self._c("hpc_upload", field, level, 0, _dptr(a))

    def get(self, field, level):
        nn = self.n(level)
        if field in VECTOR_FIELDS:
            out = np.empty((3, nn))
            for c in range(3):
                row = np.empty(nn)
                self._c("hpc_download", field, level, c, _dptr(row))
                out[c] = row
            return out
        out = np.empty(nn)
        self._c("hpc_download", field, level, 0, _dptr(out))
        return out

    def set_choice(self, level, arr):
        a = np.ascontiguousarray(arr, dtype=np.int16).reshape(self.n(level))
        self._c("hpc_upload_choice", level, a.ctypes.data_as(C.POINTER(C.c_int16)))

    def get_choice(self, level):
        a = np.empty(self.n(level), dtype=np.int16)
        self._c("hpc_download_choice", level, a.ctypes.data_as(C.POINTER(C.c_int16)))
        return a

    def set_tensor_apply(self, on: bool = True):
        """Precision form: the FP32 V-cycle's element operator on the tensor cores (TF32 GEMMs)."""
        self._c("hpc_set_tensor_apply", int(bool(on)))

    def set_fused_coarsest(self, on: bool):
        """Coarsest-level pcg_u in one thread block (default) or as per-iteration kernels."""
        self._c("hpc_set_fused_coarsest", int(bool(on)))

    def set_tma_staging(self, on: bool = True):
        """hpc_set_tma_staging: finest-level applies stage node rows with tensor copies (default) or
        per-lane cp.async (False); the same bits either way."""
        self._c("hpc_set_tma_staging", int(bool(on)))

    def set_autotune(self, on: bool):
        """Measure strip shapes on first use of each kernel and level size (see hpc_set_autotune)."""
        self._c("hpc_set_autotune", int(bool(on)))

    @staticmethod
    def tuned_shapes():
        """[(nx, ny, nz, element rows, planes)] measured so far in this process."""
        lib = _L.load()
        buf = (C.c_int * (5 * 512))()
        n = C.c_int(0)
        _L.check("hpc_tuned_shapes", lib.hpc_tuned_shapes(buf, 512, C.byref(n)))
        return [tuple(buf[5 * i:5 * i + 5]) for i in range(n.value)]

    def set_choice_quirk(self, reproduce: bool):
        self._c("hpc_set_choice_quirk", int(bool(reproduce)))

    def state(self):
        s = (C.c_double * 6)()
        self._c("hpc_get_state", s)
        return list(s)

    def set_state(self, s6):
        self._c("hpc_set_state", (C.c_double * 6)(*s6))

    # ------------------------------------------------------------ checkpoint / restart
    CHECKPOINT_FIELDS = ("u", "v", "w", "H", "d", "d_old")

    def vtk_write(self, option: str, field: int, level: int, filename: str, field_name: str, t: int,
                  scale: float = 1.0):
        """The reference's write_total_de ("S"), write_total_u ("V", values times `scale`) or
        write_total_H ("C") of one field of one level: Output/<filename>_l_<level>_t_<t>_Proc_0.vti
        and the .pvti index, relative to the working directory.  Asynchronous: vtk_wait() (or the
        next vtk_write) waits for the files."""
        self._c("hpc_vtk_write", option.encode(), int(field), int(level), float(scale), filename.encode(),
                field_name.encode(), int(t))

    def vtk_wait(self):
        self._c("hpc_vtk_wait")

    def checkpoint_begin(self, t: int):
        """Snapshot the loop state on the device and start its copy to host memory (asynchronous)."""
        self._c("hpc_checkpoint_begin", int(t))

    def checkpoint_wait(self):
        """-> (t, {name: dense finest array}, state6) of the last checkpoint_begin (copies made)."""
        t = C.c_int(0)
        p = C.POINTER(C.c_double)()
        s = (C.c_double * 6)()
        self._c("hpc_checkpoint_wait", C.byref(t), C.byref(p), s)
        nn = self.n(self.maxlevel)
        flat = np.ctypeslib.as_array(p, shape=(6 * nn,)).copy()
        return t.value, {k: flat[i * nn:(i + 1) * nn] for i, k in enumerate(self.CHECKPOINT_FIELDS)}, list(s)

    def checkpoint_restore(self, fields: dict, state6):
        arrs = [np.ascontiguousarray(fields[k], dtype=np.float64).reshape(self.n(self.maxlevel))
                for k in self.CHECKPOINT_FIELDS]
        self._c("hpc_checkpoint_restore", *[_dptr(a) for a in arrs], (C.c_double * 6)(*state6))

    def launch_count(self, reset=False) -> int:
        v = C.c_longlong(0)
        self._c("hpc_launch_count", C.byref(v), int(reset))
        return v.value

    def sync(self):
        self._c("hpc_sync")

    def stream(self) -> int:
        return self.lib.hpc_stream(self.h) or 0

    def kernel_timing(self, kernel_class: int):
        """Start recording CUDA-event durations of every launch of `kernel_class` (-1 stops)."""
        self._c("hpc_kernel_timing", int(kernel_class))

    def kernel_time(self):
        """(launches, total device ms) recorded since kernel_timing()."""
        n = C.c_longlong(0)
        ms = C.c_double(0)
        self._c("hpc_kernel_time", C.byref(n), C.byref(ms))
        return n.value, ms.value

    # ------------------------------------------------------------ operators
    def internal_force(self, level, src, dst, small_k):
        self._c("hpc_internal_force", level, src, dst, small_k)

    def prem_u(self, level, dst, small_k):
        self._c("hpc_prem_u", level, dst, small_k)

    def fld(self, level, src, dst, lc):
        self._c("hpc_fld", level, src, dst, lc)

    def precondition_m(self, level, dst, lc):
        self._c("hpc_precondition_m", level, dst, lc)

    # ------------------------------------------------------------ smoothers / solves
    def initial_residual_u(self, level, small_k):
        r = C.c_double(0)
        self._c("hpc_initial_residual_u", level, small_k, C.byref(r))
        return r.value

    def pcg_u(self, level, small_k, Ut, nb_relax, t, f_norm):
        fn = C.c_double(f_norm)
        self._c("hpc_pcg_u", level, small_k, Ut, nb_relax, t, C.byref(fn))
        return nb_relax, fn.value

    def initial_residual_d(self, level, lc):
        r = C.c_double(0)
        self._c("hpc_initial_residual_d", level, lc, C.byref(r))
        return r.value

    def pcg_d(self, level, lc, nb_relax, t, fd_norm):
        fn = C.c_double(fd_norm)
        self._c("hpc_pcg_d", level, lc, nb_relax, t, C.byref(fn))
        return nb_relax, fn.value

    def cycle_u(self, level, mg5, small_k, Ut, t, f_norm):
        fn = C.c_double(f_norm)
        mg = mg_params(mg5)
        self._c("hpc_cycle_u", level, C.byref(mg), small_k, Ut, t, C.byref(fn))
        return None, fn.value

    def cycle_d(self, level, mg5, lc, t, fd_norm):
        fn = C.c_double(fd_norm)
        mg = mg_params(mg5)
        self._c("hpc_cycle_d", level, C.byref(mg), lc, t, C.byref(fn))
        return None, fn.value

    def u_entire(self, mg5, small_k, Ut, t, f_norm, mech_tol=1e-6):
        fn = C.c_double(f_norm)
        cy, it = C.c_int(0), C.c_int(0)
        mg = mg_params(mg5)
        self._c("hpc_u_entire", C.byref(mg), small_k, Ut, t, C.byref(fn), mech_tol, C.byref(cy), C.byref(it))
        return cy.value, it.value, fn.value

    def u_entire_fcg(self, mg5, small_k, Ut, t, f_norm, mech_tol=1e-6, mixed=False):
        """Flexible PCG with one V-cycle per iteration as the preconditioner (FP32 cycle if mixed)."""
        mg = mg_params(mg5)
        fn = C.c_double(f_norm)
        cy = C.c_int(0)
        it = C.c_int(0)
        self._c("hpc_u_entire_fcg", C.byref(mg), small_k, Ut, t, C.byref(fn), mech_tol, int(bool(mixed)),
                C.byref(cy), C.byref(it))
        return cy.value, it.value, fn.value

    def phase_field(self, mg5, lc, t, fd_norm, pf_tol=1e-12):
        fn = C.c_double(fd_norm)
        cy, it = C.c_int(0), C.c_int(0)
        mg = mg_params(mg5)
        self._c("hpc_phase_field", C.byref(mg), lc, t, C.byref(fn), pf_tol, C.byref(cy), C.byref(it))
        return cy.value, it.value, fn.value

    def step(self, t, mg_u, mg_d, small_k, lc, voxel_size, ut0=0.0, dU=0.0, dU_factor=1.5e-3, mech_tol=1e-6,
             pf_tol=1e-12, mech_solver=MECH_FAS):
        """One staggered increment; mech_solver MECH_FAS (the reference's V-cycles), MECH_FCG (flexible
        PCG preconditioned by one V-cycle per iteration) or MECH_MIXED (the same with the V-cycle in FP32)."""
        p = step_params(t, mg_u, mg_d, small_k, lc, voxel_size, ut0, dU, dU_factor, mech_tol, pf_tol, mech_solver)
        out = (C.c_double * 8)()
        self._c("hpc_step", C.byref(p), out)
        return list(out)

    # ------------------------------------------------------------ material / history
    def mp_choice(self):
        self._c("hpc_mp_choice")

    def mp_all_element(self, small_k):
        self._c("hpc_mp_all_element", small_k)

    def vr_all_level(self, field):
        self._c("hpc_vr_all_level", field)

    def voigt_all_level(self, field):
        self._c("hpc_voigt_all_level", field)

    def coarse_vr(self, field):
        self._c("hpc_coarse_vr", field)

    def strain_history(self, lc, u_proportion):
        self._c("hpc_strain_history", lc, u_proportion)

    def fd_h(self, level):
        self._c("hpc_fd_h", level)

    def _scalar(self, name, *args):
        v = C.c_double(0)
        self._c(name, *args, C.byref(v))
        return v.value

    def delta_d_max(self):
        return self._scalar("hpc_delta_d_max")

    def d_max(self):
        return self._scalar("hpc_d_max")

    def U_e(self, lc):
        return self._scalar("hpc_U_e", lc)

    def externe_force_nodal(self, Ut, small_k):
        self._c("hpc_externe_force_nodal", Ut, small_k)

    def externe_force_sum(self):
        return self._scalar("hpc_externe_force_sum")

    def initial_crack(self, H_crack, level):
        self._c("hpc_initial_crack", H_crack, level)

    # ------------------------------------------------------------ boundary conditions / transfers
    def dirichlet_bd(self, level, field, Ut):
        self._c("hpc_dirichlet_bd", level, field, Ut)

    def dirichlet_force(self, level, f_field, fi_field):
        self._c("hpc_dirichlet_force", level, f_field, fi_field)

    def dirichlet_residual(self, level, field):
        self._c("hpc_dirichlet_residual", level, field)

    def solution_injection(self, field, comp, lf):
        self._c("hpc_solution_injection", field, comp, lf)

    def coarsen_f_standard(self, fc_field, rf_field, fic_field, comp, lf):
        self._c("hpc_coarsen_f_standard", fc_field, rf_field, fic_field, comp, lf)

    def refine_standard(self, uf_field, uc_field, ucold_field, comp, lf):
        self._c("hpc_refine_standard", uf_field, uc_field, ucold_field, comp, lf)

    # ------------------------------------------------------------ input path
    def image_material(self, image, voxel_n, table, voxel_size):
        gray, E, nu, gcv = table
        img = np.ascontiguousarray(image, dtype=np.uint8).ravel()
        g = np.ascontiguousarray(gray, dtype=np.int32)
        E = np.ascontiguousarray(E, dtype=np.float64)
        nu = np.ascontiguousarray(nu, dtype=np.float64)
        gcv = np.ascontiguousarray(gcv, dtype=np.float64)
        self._c("hpc_image_material", img.ctypes.data_as(C.POINTER(C.c_uint8)), (C.c_int * 3)(*map(int, voxel_n)),
                len(g), g.ctypes.data_as(C.POINTER(C.c_int)), _dptr(E), _dptr(nu), _dptr(gcv), voxel_size)
