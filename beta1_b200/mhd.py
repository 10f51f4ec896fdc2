"""ctypes binding of the C ABI in include/beta1_mhd.h, plus a small solver
facade that sets a case up the way the reference's LunarSolver constructor
does (geometry, boundary tables, constants, restart state) and then steps it
on the GPU.

The compiled library is required: importing works without a GPU, but every
call that touches the device fails with an error naming the cause; there is
no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Iterable, List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbeta1_mhd.so")

MHD_OK = 0
ERRORS = {1: "EINVAL", 2: "ECUDA", 3: "ENOMEM", 4: "EDT", 5: "ESTATE", 6: "EKRYLOV"}

NOALLOC_MAX_DOUBLES = 1 << 21

PREC_FP64 = 0
PREC_MIXED = 1

# the default variant of each tunable kernel, in the values mhd_autotune
# reports (minimum CTAs per SM of its launch bounds, 0: none; 12: the
# face-tiled k_fluid_mixed, 16: the same with staged face states; 14:
# k_pv_uplus_dt with J_cell in its own pass;
# k_gmres_resist: the CTAs of the persistent grid, 0: two per SM)
DEFAULT_TUNE = {"k_pv_uplus_dt": 4, "k_fluid_ucontra": 0, "k_bcell_jedge": 0, "k_eface": 0, "k_curl_e2f": 0,
                "k_eedge": 0, "k_fluid_mixed": 3, "k_gmres_resist": 0, "k_hall_edge": 0}

STAGE_TIMESTEP, STAGE_FLUID_RHS, STAGE_INDUCTION, STAGE_UPDATE, STAGE_DIVB, STAGE_HALL_EMF = 1, 2, 3, 4, 5, 6
STAGE_HALL_SOLVE = 7

INTEGRATOR_EULER, INTEGRATOR_SSPRK2 = 0, 1


class BlockDesc(C.Structure):
    _fields_ = [("ni", C.c_int32), ("nj", C.c_int32), ("nk", C.c_int32)]


class Params(C.Structure):
    _fields_ = [("gamma", C.c_double), ("cfl", C.c_double), ("inver_MA2", C.c_double),
                ("momentum_hall_coeff", C.c_double), ("state_coeff", C.c_double), ("M_H", C.c_double),
                ("M_ref", C.c_double), ("ne_hall_floor", C.c_double), ("dt_abort", C.c_double),
                ("ngg", C.c_int32), ("precision", C.c_int32)]


# every symbol the header declares, with its signature
_SIGS = {
    "mhd_ctx_create": (C.c_int, [C.POINTER(BlockDesc), C.c_int32, C.POINTER(Params), C.POINTER(C.c_void_p)]),
    "mhd_batch_create": (C.c_int, [C.POINTER(BlockDesc), C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.POINTER(Params),
                                   C.POINTER(C.c_void_p)]),
    "mhd_run_time": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                               C.POINTER(C.c_int64)]),
    "mhd_batch_step": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int32]),
    "mhd_set_flux_reference_run": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "mhd_autotune": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.c_int32]),
    "mhd_tune_name": (C.c_char_p, [C.c_int32]),
    "mhd_set_tune": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.c_int32]),
    "mhd_ctx_destroy": (C.c_int, [C.c_void_p]),
    "mhd_last_error": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32]),
    "mhd_field_info": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                 C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "mhd_upload_field": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32, C.c_void_p, C.c_int64]),
    "mhd_download_field": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32, C.c_void_p, C.c_int64]),
    "mhd_download_field_noalloc": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32, C.c_void_p, C.c_int64]),
    "mhd_point_id": (C.c_int64, [C.c_void_p, C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "mhd_set_sync_map": (C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_int64]),
    "mhd_sync": (C.c_int, [C.c_void_p, C.c_char_p]),
    "mhd_test_stall_barrier": (C.c_int, [C.c_void_p, C.c_uint32]),
    "mhd_set_integrator": (C.c_int, [C.c_void_p, C.c_int32]),
    "mhd_set_sync_consts": (C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_int64]),
    "mhd_set_sync_wall": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32, C.c_int32]),
    "mhd_set_sync_map_post": (C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_int64]),
    "mhd_set_pole": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "mhd_build_geometry": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p]),
    "mhd_diagnostics": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "mhd_set_resistive": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_int32, C.c_int32]),
    "mhd_set_hall_implicit": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_double, C.c_double, C.c_int32, C.c_double, C.c_int32]),
    "mhd_hall_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                 C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "mhd_set_hall": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_int32]),
    "mhd_set_resistive_explicit": (C.c_int, [C.c_void_p, C.c_double, C.c_int32]),
    "mhd_set_flux_reference": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "mhd_resistive_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "mhd_update_derived": (C.c_int, [C.c_void_p]),
    "mhd_step": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "mhd_step_host": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_double)]),
    "mhd_state_count": (C.c_int64, [C.c_void_p]),
    "mhd_step_host_inner": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64,
                                      C.POINTER(C.c_double)]),
    "mhd_state_count_inner": (C.c_int64, [C.c_void_p]),
    "mhd_host_alloc": (C.c_int, [C.c_int64, C.POINTER(C.c_void_p)]),
    "mhd_host_free": (C.c_int, [C.c_void_p]),
    "mhd_stage": (C.c_int, [C.c_void_p, C.c_int32]),
    "mhd_get_time": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    "mhd_set_time": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_int64]),
    "mhd_kernel_launches": (C.c_int64, [C.c_void_p]),
    "mhd_profile_step": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_float),
                                   C.POINTER(C.c_int32)]),
    "mhd_kernel_name": (C.c_char_p, [C.c_int32]),
    "mhd_stream": (C.c_void_p, [C.c_void_p]),
    "mhd_field_spec": (C.c_int, [C.c_int32, C.POINTER(C.c_char_p), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                 C.POINTER(C.c_int32)]),
}

_lib: Optional[C.CDLL] = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Loads the CUDA library (built by beta1_b200.build); raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with beta1_b200.build.build_library()")
    lib = C.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols() -> List[str]:
    return list(_SIGS)


class MHDError(RuntimeError):
    pass


def field_table():
    """[(name, loc, ncomp, nghost)] in the library's field-index order."""
    lib = load()
    out = []
    i = 0
    while True:
        nm, loc, nc, ng = C.c_char_p(), C.c_int32(), C.c_int32(), C.c_int32()
        if lib.mhd_field_spec(i, C.byref(nm), C.byref(loc), C.byref(nc), C.byref(ng)) != MHD_OK:
            break
        out.append((nm.value.decode(), loc.value, nc.value, ng.value))
        i += 1
    return out


class HostLayout:
    """Host-side twin of a context's field addressing (field boxes and point
    ids), usable without a GPU to compile sync tables."""

    PLUS = {0: (0, 0, 0), 1: (1, 0, 0), 2: (0, 1, 0), 3: (0, 0, 1), 4: (0, 1, 1), 5: (1, 0, 1), 6: (1, 1, 0)}

    def __init__(self, ncells):
        self.ncells = [tuple(map(int, n)) for n in ncells]
        self.table = field_table()
        self.index = {t[0]: i for i, t in enumerate(self.table)}

    def field_info(self, name, block=0):
        _, loc, nc, ng = self.table[self.index[name]]
        n = self.ncells[block]
        p = self.PLUS[loc]
        return dict(loc=loc, ncomp=nc, nghost=ng, lo=(-ng, -ng, -ng),
                    hi=(n[0] + p[0] + ng, n[1] + p[1] + ng, n[2] + p[2] + ng))

    def point_base(self, name, block):
        return (self.index[name] << 56) | (int(block) << 40)



def _same_size(*named):
    """the arrays a call passes with one count hold that many values each"""
    n = named[0][1].size
    for name, a in named:
        if a.size != n:
            raise ValueError(f"{name} holds {a.size} values, {named[0][0]} {n}")


def check_state_buffers(state_in: np.ndarray, state_out: np.ndarray, count: int) -> None:
    """The host buffers of a host-buffer step: C-contiguous float64 arrays of
    exactly `count` values each, the output writable (the library reads
    `count` values from one and writes as many to the other; the input is
    read in full before the output is written, so both may be one array)."""
    for name, a in (("state_in", state_in), ("state_out", state_out)):
        if not isinstance(a, np.ndarray) or a.dtype != np.float64 or not a.flags.c_contiguous:
            raise TypeError(f"{name} must be a C-contiguous float64 numpy array")
        if a.size != count:
            raise ValueError(f"{name} holds {a.size} values, the state {count}")
    if not state_out.flags.writeable:
        raise ValueError("state_out is read-only")

class Context:
    """One device context (all blocks of one grid on the current GPU)."""

    def __init__(self, ncells: Sequence[Sequence[int]], params: Params, runs: Optional[Sequence[int]] = None):
        """runs: the run of every block for a batch of independent runs
        (mhd_batch_create); None for one run."""
        self.lib = load()
        arr = (BlockDesc * len(ncells))(*[BlockDesc(*map(int, n)) for n in ncells])
        h = C.c_void_p()
        if runs is None:
            self.nruns = 1
            rc = self.lib.mhd_ctx_create(arr, len(ncells), C.byref(params), C.byref(h))
        else:
            self.nruns = int(max(runs)) + 1
            ra = (C.c_int32 * len(runs))(*[int(r) for r in runs])
            rc = self.lib.mhd_batch_create(arr, len(ncells), ra, self.nruns, C.byref(params), C.byref(h))
        if rc != MHD_OK:
            raise MHDError(f"mhd_ctx_create failed: {ERRORS.get(rc, rc)}")
        self.h = h
        self.ncells = [tuple(map(int, n)) for n in ncells]
        self.params = params

    def close(self):
        if getattr(self, "h", None):
            self.lib.mhd_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != MHD_OK:
            buf = C.create_string_buffer(512)
            self.lib.mhd_last_error(self.h, buf, 512)
            raise MHDError(f"{what}: {ERRORS.get(rc, rc)}: {buf.value.decode(errors='replace')}")

    def field_info(self, name: str, block: int = 0):
        loc, nc, ng = C.c_int32(), C.c_int32(), C.c_int32()
        lo, hi = (C.c_int32 * 3)(), (C.c_int32 * 3)()
        self._check(self.lib.mhd_field_info(self.h, name.encode(), block, C.byref(loc), C.byref(nc), C.byref(ng),
                                            lo, hi), f"field_info {name}")
        return dict(loc=loc.value, ncomp=nc.value, nghost=ng.value, lo=tuple(lo), hi=tuple(hi))

    def upload(self, name: str, block: int, data: np.ndarray):
        a = np.ascontiguousarray(data, dtype=np.float64)
        self._check(self.lib.mhd_upload_field(self.h, name.encode(), block, a.ctypes.data, a.size), f"upload {name}")

    def download(self, name: str, block: int = 0) -> np.ndarray:
        inf = self.field_info(name, block)
        shape = tuple(h - l for l, h in zip(inf["lo"], inf["hi"])) + (inf["ncomp"],)
        out = np.empty(shape, dtype=np.float64)
        self._check(self.lib.mhd_download_field(self.h, name.encode(), block, out.ctypes.data, out.size),
                    f"download {name}")
        return out

    def download_noalloc(self, name: str, block: int = 0) -> np.ndarray:
        """As download(), through the library's fixed staging array: no device
        memory is allocated (fields up to NOALLOC_MAX_DOUBLES values)."""
        inf = self.field_info(name, block)
        shape = tuple(h - l for l, h in zip(inf["lo"], inf["hi"])) + (inf["ncomp"],)
        out = np.empty(shape, dtype=np.float64)
        self._check(self.lib.mhd_download_field_noalloc(self.h, name.encode(), block, out.ctypes.data, out.size),
                    f"download_noalloc {name}")
        return out

    def point_base(self, name: str, block: int) -> int:
        inf = self.field_info(name, block)
        pid = self.lib.mhd_point_id(self.h, name.encode(), block, *inf["lo"], 0)
        if pid < 0:
            raise MHDError(f"point id of {name}")
        return int(pid)

    def set_sync_map(self, group: str, dst: np.ndarray, src: np.ndarray):
        d = np.ascontiguousarray(dst, dtype=np.int64)
        s = np.ascontiguousarray(src, dtype=np.int64)
        _same_size(("dst", d), ("src", s))
        self._check(self.lib.mhd_set_sync_map(self.h, group.encode(), d.ctypes.data, s.ctypes.data, d.size),
                    f"set_sync_map {group}")

    def set_sync_consts(self, group: str, dst: np.ndarray, val: np.ndarray):
        d = np.ascontiguousarray(dst, dtype=np.int64)
        v = np.ascontiguousarray(val, dtype=np.float64)
        _same_size(("dst", d), ("val", v))
        self._check(self.lib.mhd_set_sync_consts(self.h, group.encode(), d.ctypes.data, v.ctypes.data, d.size),
                    f"set_sync_consts {group}")

    def set_sync_wall(self, group: str, block: int, direction: int):
        self._check(self.lib.mhd_set_sync_wall(self.h, group.encode(), block, direction), f"set_sync_wall {group}")

    def set_sync_map_post(self, group: str, dst: np.ndarray, src: np.ndarray):
        """copies run after the group's wall handlers (contexts with Poles)"""
        d = np.ascontiguousarray(dst, dtype=np.int64)
        s = np.ascontiguousarray(src, dtype=np.int64)
        _same_size(("dst", d), ("src", s))
        self._check(self.lib.mhd_set_sync_map_post(self.h, group.encode(), d.ctypes.data, s.ctypes.data, d.size),
                    f"set_sync_map_post {group}")

    def build_geometry(self, block: int, nodes: np.ndarray, B_imf=None):
        """every geometry field of a block from its ghost node mesh, on the
        device (nodes: the Padded array of geometry.block_ghost_mesh)"""
        a = np.ascontiguousarray(nodes, dtype=np.float64)
        bp = None
        if B_imf is not None:
            bv = np.ascontiguousarray(B_imf, dtype=np.float64)
            if bv.size != 3:
                raise ValueError("B_imf holds three values")
            bp = bv.ctypes.data
        self._check(self.lib.mhd_build_geometry(self.h, block, a.ctypes.data, a.size, bp), "build_geometry")

    def diagnostics(self, run: int = -1):
        """PrintMinMaxDiagnostics_ values: (mins of rho, p, Bx, By, Bz, |B|^2/2;
        their maxima and max |divB|) over a run's inner cells (-1: all)"""
        mins = (C.c_double * 6)()
        maxs = (C.c_double * 7)()
        self._check(self.lib.mhd_diagnostics(self.h, run, mins, maxs), "diagnostics")
        return list(mins), list(maxs)

    def set_pole(self, block: int, direction: int):
        """an eta Pole (direction -2: j = 0, +2: j = n_j) of a block"""
        self._check(self.lib.mhd_set_pole(self.h, block, direction), "set_pole")

    def set_resistive(self, unknowns, eta, alias, owner, sign, rtol, atol, maxit, restart=30):
        u = np.ascontiguousarray(unknowns, dtype=np.int64)
        e = np.ascontiguousarray(eta, dtype=np.float64)
        a = np.ascontiguousarray(alias, dtype=np.int64)
        o = np.ascontiguousarray(owner, dtype=np.int64)
        sg = np.ascontiguousarray(sign, dtype=np.float64)
        _same_size(("unknowns", u), ("eta", e))
        _same_size(("alias", a), ("owner", o), ("sign", sg))
        self._check(self.lib.mhd_set_resistive(self.h, u.size, u.ctypes.data, e.ctypes.data, a.size, a.ctypes.data,
                                               o.ctypes.data, sg.ctypes.data, rtol, atol, maxit, restart),
                    "set_resistive")

    def set_hall(self, hall_coef: float, zero_boxes):
        z = np.ascontiguousarray(np.asarray(zero_boxes, dtype=np.int32).reshape(-1, 8))
        self._check(self.lib.mhd_set_hall(self.h, float(hall_coef), z.ctypes.data, len(z)), "set_hall")

    def set_hall_implicit(self, unknowns, alias, owner, sign, rtol=1e-8, atol=1e-50, maxit=50, ksp_rtol=1e-5,
                          ksp_maxit=10000):
        u = np.ascontiguousarray(unknowns, dtype=np.int64)
        a = np.ascontiguousarray(alias, dtype=np.int64)
        o = np.ascontiguousarray(owner, dtype=np.int64)
        sg = np.ascontiguousarray(sign, dtype=np.float64)
        _same_size(("alias", a), ("owner", o), ("sign", sg))
        self._check(self.lib.mhd_set_hall_implicit(self.h, u.size, u.ctypes.data, a.size, a.ctypes.data,
                                                   o.ctypes.data, sg.ctypes.data, float(rtol), float(atol), int(maxit),
                                                   float(ksp_rtol), int(ksp_maxit)), "set_hall_implicit")

    def hall_stats(self):
        its, lin, fn, f0, rs = C.c_int32(), C.c_int32(), C.c_double(), C.c_double(), C.c_int32()
        self._check(self.lib.mhd_hall_stats(self.h, C.byref(its), C.byref(lin), C.byref(fn), C.byref(f0),
                                            C.byref(rs)), "hall_stats")
        return dict(its=its.value, linear_its=lin.value, fnorm=fn.value, fnorm0=f0.value, reason=rs.value)

    def set_resistive_explicit(self, inver_Rem: float, nsub: int):
        self._check(self.lib.mhd_set_resistive_explicit(self.h, float(inver_Rem), int(nsub)), "set_resistive_explicit")

    def set_flux_reference(self, prim, run: int = -1):
        """reference state (rho, u, v, w, p) of the mixed-precision deviation
        flux, of one run of a batch or (run -1) of every run"""
        a = (C.c_double * 5)(*[float(x) for x in prim])
        if run < 0:
            self._check(self.lib.mhd_set_flux_reference(self.h, a), "set_flux_reference")
        else:
            self._check(self.lib.mhd_set_flux_reference_run(self.h, int(run), a), "set_flux_reference_run")

    def autotune(self, reps: int = 10) -> Dict[str, int]:
        """times the register / occupancy variants of the hot kernels on the
        current state and keeps the fastest; returns kernel -> chosen minimum
        CTAs per SM"""
        n = len(DEFAULT_TUNE)
        out = (C.c_int32 * n)()
        self._check(self.lib.mhd_autotune(self.h, int(reps), out, n), "autotune")
        return {self.lib.mhd_tune_name(i).decode(): int(out[i]) for i in range(n)}

    def set_tune(self, chosen: Dict[str, int]):
        """applies a variant choice in autotune()'s values (kernel -> value);
        kernels not named get their default variant (DEFAULT_TUNE)"""
        n = len(DEFAULT_TUNE)
        names = [self.lib.mhd_tune_name(i).decode() for i in range(n)]
        vals = (C.c_int32 * n)(*[int(chosen.get(nm, DEFAULT_TUNE[nm])) for nm in names])
        self._check(self.lib.mhd_set_tune(self.h, vals, n), "set_tune")

    def batch_step(self, nsteps: int):
        """nsteps steps of every run; returns (dt of every run, time of every run)"""
        dt = (C.c_double * self.nruns)()
        t = (C.c_double * self.nruns)()
        self._check(self.lib.mhd_batch_step(self.h, int(nsteps), dt, t, self.nruns), "batch_step")
        return list(dt), list(t)

    def run_time(self, run: int):
        """(dt of the last step, time, step count) of one run"""
        dt, t, n = C.c_double(), C.c_double(), C.c_int64()
        self._check(self.lib.mhd_run_time(self.h, int(run), C.byref(dt), C.byref(t), C.byref(n)), "run_time")
        return dt.value, t.value, n.value

    def resistive_stats(self):
        its, rn, bn, rs = C.c_int32(), C.c_double(), C.c_double(), C.c_int32()
        self._check(self.lib.mhd_resistive_stats(self.h, C.byref(its), C.byref(rn), C.byref(bn), C.byref(rs)),
                    "resistive_stats")
        return dict(its=its.value, rnorm=rn.value, bnorm=bn.value, reason=rs.value)

    def set_integrator(self, integrator: int):
        """INTEGRATOR_EULER (the reference's StepOnce) or INTEGRATOR_SSPRK2
        (two Euler stages at one dt and their convex average)"""
        self._check(self.lib.mhd_set_integrator(self.h, int(integrator)), "set_integrator")

    def test_stall_barrier(self, spin_limit: int):
        """failure-detection hook: the next persistent resistive solve waits
        for a barrier arrival that never comes, each wait bounded at
        spin_limit polls, and the step reports EKRYLOV"""
        self._check(self.lib.mhd_test_stall_barrier(self.h, int(spin_limit)), "test_stall_barrier")

    def sync(self, group: str):
        self._check(self.lib.mhd_sync(self.h, group.encode()), f"sync {group}")

    def update_derived(self):
        self._check(self.lib.mhd_update_derived(self.h), "update_derived")

    def step(self, n: int = 1):
        dt, t = C.c_double(), C.c_double()
        self._check(self.lib.mhd_step(self.h, n, C.byref(dt), C.byref(t)), "step")
        return dt.value, t.value

    def stage(self, sid: int):
        self._check(self.lib.mhd_stage(self.h, sid), f"stage {sid}")

    def get_time(self):
        dt, t, s = C.c_double(), C.c_double(), C.c_int64()
        self._check(self.lib.mhd_get_time(self.h, C.byref(dt), C.byref(t), C.byref(s)), "get_time")
        return dt.value, t.value, s.value

    def set_time(self, dt: float, time: float, step: int):
        """dt, time and step count of every run"""
        self._check(self.lib.mhd_set_time(self.h, float(dt), float(time), int(step)), "set_time")

    def state_count(self) -> int:
        return int(self.lib.mhd_state_count(self.h))

    def step_host(self, nsteps: int, state_in: np.ndarray, state_out: np.ndarray) -> float:
        """mhd_step_host: the whole state arrays (ghost layers included)"""
        check_state_buffers(state_in, state_out, self.state_count())
        dt = C.c_double()
        self._check(self.lib.mhd_step_host(self.h, nsteps, state_in.ctypes.data, state_out.ctypes.data,
                                           state_in.size, C.byref(dt)), "step_host")
        return dt.value

    def state_count_inner(self) -> int:
        return int(self.lib.mhd_state_count_inner(self.h))

    def step_host_inner(self, nsteps: int, state_in: np.ndarray, state_out: np.ndarray) -> float:
        """mhd_step_host with the state's inner points only"""
        check_state_buffers(state_in, state_out, self.state_count_inner())
        dt = C.c_double()
        self._check(self.lib.mhd_step_host_inner(self.h, nsteps, state_in.ctypes.data, state_out.ctypes.data,
                                                 state_in.size, C.byref(dt)), "step_host_inner")
        return dt.value

    def launches(self) -> int:
        return int(self.lib.mhd_kernel_launches(self.h))

    def profile_step(self):
        """One eager StepOnce with per-launch CUDA events: list of (kernel, ms)."""
        cap = 4096
        ids = (C.c_int32 * cap)()
        ms = (C.c_float * cap)()
        n = C.c_int32()
        self._check(self.lib.mhd_profile_step(self.h, cap, ids, ms, C.byref(n)), "profile_step")
        return [(self.lib.mhd_kernel_name(ids[q]).decode(), float(ms[q])) for q in range(min(n.value, cap))]

    def stream(self) -> int:
        return int(self.lib.mhd_stream(self.h) or 0)


class PinnedArray:
    """Page-locked float64 host buffer from mhd_host_alloc, viewed as numpy."""

    def __init__(self, n: int):
        self.lib = load()
        p = C.c_void_p()
        rc = self.lib.mhd_host_alloc(int(n) * 8, C.byref(p))
        if rc != MHD_OK:
            raise MHDError("mhd_host_alloc failed")
        self.p = p
        self.a = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_double)), shape=(int(n),))

    def free(self):
        if self.p:
            self.lib.mhd_host_free(self.p)
            self.p = None
