"""ctypes binding of libatus_gpu.so (include/atus_gpu.h).

``Solver`` is the Python face of one GPU context.  Its methods carry the names
and argument meaning of the reference's solver classes, so a program written
against ``CRT_Base`` / ``CRT_Base_IF`` / ``CSOB_Base`` maps onto it call by
call:

    ft_step(half)          Do_FT_Step_half / Do_FT_Step_full (include/CRT_Base.h:336-392)
    nl_step()              CRT_Base::Do_NL_Step             (include/CRT_Base.h:396-441)
    nl_if_step(laser)      CRT_Base_IF::Do_NL_Step          (include/CRT_Base_IF.h:380-419)
    bragg_ad(laser, F)     Bragg_single::Do_Bragg_ad        (source/interferometry/src/bragg.cpp:185-304)
    block(nk, kind, ...)   one outer iteration of run_sequence (include/CRT_Base.h:776-786)
    particle_number(c)     Get_Particle_Number              (include/CRT_Base.h:586-599)
    expval_position/momentum, setup_momentum, rabi_integrals, sob_*  (see atus_gpu.h)

Errors from the library raise ``AtusError`` with the context's message.  There
is no CPU fallback: without the built library or without a CUDA device the
constructor raises.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libatus_gpu.so")

ATUS_OK = 0
PREC_FP64 = 0
PREC_MIXED = 1
STEP_NL, STEP_NL_IF, STEP_BRAGG_AD, STEP_DOUBLE_BRAGG_AD, STEP_NL_IF_2, STEP_BRAGG_DS_AD = 0, 1, 2, 3, 4, 5
STEP_NUMERICAL_BRAGG, STEP_NUMERICAL_RAMAN = 6, 7
MAX_COMP = 4

_ERRORS = {-1: "invalid argument", -2: "unsupported", -3: "CUDA error", -4: "bad state", -5: "out of device memory"}


class AtusError(RuntimeError):
    pass


class Grid(C.Structure):
    _fields_ = [("dim", C.c_int), ("n", C.c_int64 * 3), ("d", C.c_double * 3), ("dk", C.c_double * 3),
                ("t", C.c_double)]


class Laser(C.Structure):
    """atus_laser: the CRT_Base_IF laser members (include/CRT_Base_IF.h:65-77)."""

    _fields_ = [
        ("beta", C.c_double * 3),
        ("DeltaL", C.c_double * MAX_COMP),
        ("Amp", C.c_double * 2),
        ("laser_k", C.c_double * 2),
        ("laser_dk", C.c_double * 2),
        ("laser_domh", C.c_double * 2),
        ("phase", C.c_double * 2),
        ("chirp_rate", C.c_double * 2),
        ("chirp", C.c_double),
    ]

    @classmethod
    def make(cls, **kw):
        L = cls()
        for k, v in kw.items():
            f = getattr(L, k)
            if k == "chirp":
                setattr(L, k, float(v))
            elif isinstance(v, (int, float)):
                f[0] = float(v)
            else:
                for i, x in enumerate(v):
                    f[i] = float(x)
        return L


class BatchInstance(C.Structure):
    """atus_batch_instance: one bragg_ad run of a batched sweep."""

    _fields_ = [("grid", Grid), ("alpha", C.c_double), ("gs", C.c_double * 4), ("laser", Laser),
                ("pulse_tc", C.c_double), ("pulse_sigma", C.c_double), ("bragg_stable", C.c_int)]


# Every entry point of include/atus_gpu.h with its ctypes signature.
_vp, _dp, _i, _d = C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_double
SIGNATURES = {
    "atus_create": (_i, [C.POINTER(Grid), _i, _i, C.POINTER(C.c_void_p)]),
    "atus_clone": (_i, [_vp, C.POINTER(C.c_void_p)]),
    "atus_destroy": (None, [_vp]),
    "atus_last_error": (C.c_char_p, [_vp]),
    "atus_set_stream": (_i, [_vp, _vp]),
    "atus_synchronize": (_i, [_vp]),
    "atus_launch_count": (_i, [_vp, C.POINTER(C.c_int64)]),
    "atus_set_alpha": (_i, [_vp, _i, _dp]),
    "atus_set_dt": (_i, [_vp, _d]),
    "atus_get_dt": (_i, [_vp, _dp]),
    "atus_set_time": (_i, [_vp, _d]),
    "atus_get_time": (_i, [_vp, _dp]),
    "atus_set_gs": (_i, [_vp, _dp]),
    "atus_set_potential": (_i, [_vp, _i, _dp]),
    "atus_set_laser": (_i, [_vp, C.POINTER(Laser)]),
    "atus_set_laser2": (_i, [_vp, C.POINTER(Laser)]),
    "atus_set_pulse_windows": (_i, [_vp, _d, _dp]),
    "atus_upload_psi": (_i, [_vp, _i, _dp]),
    "atus_download_psi": (_i, [_vp, _i, _dp]),
    "atus_device_psi": (_i, [_vp, _i, C.POINTER(C.c_void_p)]),
    "atus_embed": (_i, [_vp, _i, _vp, _i]),
    "atus_ft": (_i, [_vp, _i, _i]),
    "atus_ft_step": (_i, [_vp, _i]),
    "atus_nl_step": (_i, [_vp, _i, _d]),
    "atus_strang_block": (_i, [_vp, _i, _i, _dp]),
    "atus_strang_block_rabi": (_i, [_vp, _i, _i, _dp, _i, C.POINTER(C.c_int), _dp, _i, C.c_double, _dp]),
    "atus_snapshot": (_i, [_vp]),
    "atus_snapshot_read": (_i, [_vp, _i, _dp]),
    "atus_profile_passes": (_i, [_vp, _i, _i, _dp, _dp, _dp, C.POINTER(C.c_int)]),
    "atus_particle_number": (_i, [_vp, _i, _dp]),
    "atus_set_bragg_stable": (_i, [_vp, _i]),
    "atus_set_wait_limits": (_i, [_vp, C.c_int64, _i]),
    "atus_particle_number_noalloc": (_i, [_vp, C.c_int64, _i, C.c_double, _vp, _vp]),
    "atus_guess_init": (_i, [C.c_uint64, _dp]),
    "atus_guess_grad": (_i, [_dp, _dp, _dp, _i, _dp, _dp]),
    "atus_guess_train": (_i, [_dp, _dp, _dp, _i, _i, _d, _dp]),
    "atus_guess_predict": (_i, [_dp, _dp, _i, _dp]),
    "atus_guess_decode": (_i, [_vp, _i, _dp, _dp]),
    "atus_batch_create": (_i, [C.POINTER(BatchInstance), _i, _i, _d, C.POINTER(C.c_void_p)]),
    "atus_batch_destroy": (None, [_vp]),
    "atus_batch_last_error": (C.c_char_p, [_vp]),
    "atus_batch_upload_psi": (_i, [_vp, _i, _i, _dp]),
    "atus_batch_download_psi": (_i, [_vp, _i, _i, _dp]),
    "atus_batch_get_time": (_i, [_vp, _i, _dp]),
    "atus_batch_tune": (_i, [_vp, _i]),
    "atus_batch_run": (_i, [_vp, _i, _dp]),
    "atus_batch_schedule": (_i, [_vp, C.c_char_p, _i]),
    "atus_expval_position": (_i, [_vp, _i, _dp]),
    "atus_expval_momentum": (_i, [_vp, _i, _dp]),
    "atus_setup_momentum": (_i, [_vp, _i, _dp]),
    "atus_rabi_integrals": (_i, [_vp, _dp, _i, _d, _dp]),
    "atus_rabi_integrals_comp": (_i, [_vp, _i, _dp, _i, _d, _dp]),
    "atus_sob_init": (_i, [_vp, _dp, _d]),
    "atus_sob_renormalize": (_i, [_vp]),
    "atus_sob_iterate": (_i, [_vp, _i, _dp, _dp]),
    "atus_sob_run": (_i, [_vp, _d, _i, C.POINTER(C.c_int), _dp]),
    "atus_sob_mu": (_i, [_vp, _dp]),
}

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libatus_gpu.so (built by ``python -m atus2_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with `python -m atus2_b200.build`")
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def grid_from_header(header) -> Grid:
    g = Grid()
    g.dim = int(header["nDims"])
    for a, ax in enumerate("XYZ"):
        g.n[a] = int(header[f"nDim{ax}"]) if a < g.dim else 1
    for a, ax in enumerate("xyz"):
        g.d[a] = float(header[f"d{ax}"]) if a < g.dim else 0.0
        g.dk[a] = float(header[f"dk{ax}"]) if a < g.dim else 0.0
    g.t = float(header["t"])
    return g


class Solver:
    """One GPU context holding ``ncomp`` fields on the grid of ``header``."""

    def __init__(self, header, ncomp: int, precision: int = PREC_FP64):
        self._L = load_library()
        self.dim = int(header["nDims"])
        self.shape = tuple(int(header[f"nDim{a}"]) for a in "XYZ"[: self.dim])
        self.npts = int(np.prod(self.shape))
        self.ncomp = ncomp
        self.precision = precision
        self._c = C.c_void_p()
        g = grid_from_header(header)
        r = self._L.atus_create(C.byref(g), ncomp, precision, C.byref(self._c))
        if r != ATUS_OK:
            raise AtusError(f"atus_create failed: {_ERRORS.get(r, r)} (grid {self.shape}, ncomp {ncomp})")

    def close(self):
        if getattr(self, "_c", None) and self._c.value:
            self._L.atus_destroy(self._c)
            self._c = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, r: int, what: str):
        if r != ATUS_OK:
            msg = self._L.atus_last_error(self._c)
            raise AtusError(f"{what}: {_ERRORS.get(r, r)}: {msg.decode() if msg else ''}")

    # ------------------------------------------------------------ state
    def set_psi(self, comp: int, data) -> None:
        a = np.ascontiguousarray(np.asarray(data, dtype=np.complex128).reshape(self.shape))
        self._ok(self._L.atus_upload_psi(self._c, comp, a.ctypes.data_as(_dp)), "upload_psi")

    def psi(self, comp: int) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.complex128)
        self._ok(self._L.atus_download_psi(self._c, comp, out.ctypes.data_as(_dp)), "download_psi")
        return out

    def upload_from(self, comp: int, host_ptr: int) -> None:
        """Upload N complex128 values from a host address (e.g. pinned memory)."""
        self._ok(self._L.atus_upload_psi(self._c, comp, C.cast(C.c_void_p(host_ptr), _dp)), "upload_psi")

    def download_to(self, comp: int, host_ptr: int) -> None:
        self._ok(self._L.atus_download_psi(self._c, comp, C.cast(C.c_void_p(host_ptr), _dp)), "download_psi")

    def profile_passes(self, kind: int, reps: int = 10):
        """[(ms per launch, launches per Strang step, field bytes per launch)] per fused pass."""
        ms, lps, by = np.zeros(8), np.zeros(8), np.zeros(8)
        n = C.c_int()
        self._ok(self._L.atus_profile_passes(self._c, int(kind), int(reps), _dptr(ms), _dptr(lps), _dptr(by), C.byref(n)),
                 "profile_passes")
        return [(float(ms[i]), float(lps[i]), float(by[i])) for i in range(n.value)]

    def device_ptr(self, comp: int) -> int:
        p = C.c_void_p()
        self._ok(self._L.atus_device_psi(self._c, comp, C.byref(p)), "device_psi")
        return p.value

    @property
    def t(self) -> float:
        v = C.c_double()
        self._ok(self._L.atus_get_time(self._c, C.byref(v)), "get_time")
        return v.value

    @t.setter
    def t(self, v: float) -> None:
        self._ok(self._L.atus_set_time(self._c, float(v)), "set_time")

    @property
    def dt(self) -> float:
        v = C.c_double()
        self._ok(self._L.atus_get_dt(self._c, C.byref(v)), "get_dt")
        return v.value

    def set_dt(self, dt: float) -> None:
        self._ok(self._L.atus_set_dt(self._c, float(dt)), "set_dt")

    def set_alpha(self, comp: int, alpha) -> None:
        a = np.zeros(3)
        a[: len(alpha)] = alpha
        self._ok(self._L.atus_set_alpha(self._c, comp, _dptr(a)), "set_alpha")

    def set_gs(self, gs) -> None:
        a = np.ascontiguousarray(gs, dtype=np.float64).ravel()
        assert a.size == self.ncomp * self.ncomp
        self._ok(self._L.atus_set_gs(self._c, _dptr(a)), "set_gs")

    def set_potential(self, comp: int, V) -> None:
        if V is None:
            self._ok(self._L.atus_set_potential(self._c, comp, None), "set_potential")
            return
        a = np.ascontiguousarray(V, dtype=np.float64).ravel()
        if a.size != self.npts:
            raise ValueError("potential size does not match the grid")
        self._ok(self._L.atus_set_potential(self._c, comp, _dptr(a)), "set_potential")

    def set_bragg_stable(self, on: bool = True) -> None:
        """FP64 bragg_ad in the eigenvalue-free form instead of the reference's eigen-form."""
        self._ok(self._L.atus_set_bragg_stable(self._c, int(bool(on))), "set_bragg_stable")

    def set_wait_limits(self, wait_rounds: int = 1 << 22, drop_copies: bool = False) -> None:
        """Bounded waits of the TMA-fed passes (atus_set_wait_limits);
        drop_copies makes every wait run out (tests of the error path)."""
        self._ok(self._L.atus_set_wait_limits(self._c, int(wait_rounds), int(bool(drop_copies))), "set_wait_limits")

    def set_laser(self, laser: Laser) -> None:
        self._ok(self._L.atus_set_laser(self._c, C.byref(laser)), "set_laser")

    def set_species2(self, laser2: Laser, t_start: float = 0.0, durations=(math.inf, math.inf)) -> None:
        """Second species of the two-species programs (laser parameters
        Beta_2, Amp_2, laser_k_2, ...) and the pulse windows of their bragg_ad
        (species s couples while t + dt/2 - t_start <= durations[s])."""
        self._ok(self._L.atus_set_laser2(self._c, C.byref(laser2)), "set_laser2")
        d = np.ascontiguousarray(durations, dtype=np.float64)
        self._ok(self._L.atus_set_pulse_windows(self._c, float(t_start), _dptr(d)), "set_pulse_windows")

    def set_stream(self, stream_handle: int | None) -> None:
        self._ok(self._L.atus_set_stream(self._c, C.c_void_p(stream_handle or 0)), "set_stream")

    def synchronize(self) -> None:
        self._ok(self._L.atus_synchronize(self._c), "synchronize")

    @property
    def launches(self) -> int:
        v = C.c_int64()
        self._ok(self._L.atus_launch_count(self._c, C.byref(v)), "launch_count")
        return v.value

    # ------------------------------------------------------------ steps
    def ft(self, comp: int, isign: int) -> None:
        """cft_Nd::ft on component comp: transform over all axes (isign -1
        forward, +1 backward) with the reference's scale."""
        self._ok(self._L.atus_ft(self._c, int(comp), int(isign)), "ft")

    def ft_step(self, half: bool) -> None:
        self._ok(self._L.atus_ft_step(self._c, 1 if half else 0), "ft_step")

    def nl_step(self) -> None:
        self._ok(self._L.atus_nl_step(self._c, STEP_NL, 1.0), "nl_step")

    def nl_if_step(self, laser: Laser) -> None:
        self.set_laser(laser)
        self._ok(self._L.atus_nl_step(self._c, STEP_NL_IF, 1.0), "nl_if_step")

    def bragg_ad(self, laser: Laser, F: float = 1.0) -> None:
        self.set_laser(laser)
        self._ok(self._L.atus_nl_step(self._c, STEP_BRAGG_AD, float(F)), "bragg_ad")

    def block(self, nk: int, kind: int, laser: Laser | None = None, F=None) -> None:
        if laser is not None:
            self.set_laser(laser)
        Fa = None
        if F is not None:
            Fa = np.ascontiguousarray(F, dtype=np.float64)
            if Fa.size < nk:
                raise ValueError("F needs one amplitude per potential step")
        self._ok(self._L.atus_strang_block(self._c, int(nk), int(kind), None if Fa is None else _dptr(Fa)),
                 "strang_block")

    def block_rabi(self, nk: int, kind: int, comps, k0, thr: float, laser: Laser | None = None, F=None) -> np.ndarray:
        """block() that also returns the Rabi sums of its final state for
        components comps (one k0 list per component): shape (len(comps), n)."""
        if laser is not None:
            self.set_laser(laser)
        Fa = None if F is None else np.ascontiguousarray(F, dtype=np.float64)
        if Fa is not None and Fa.size < nk:
            raise ValueError("F needs one amplitude per potential step")
        cs = (C.c_int * len(comps))(*comps)
        k = np.ascontiguousarray(k0, dtype=np.float64).reshape(len(comps), -1, self.dim)
        out = np.zeros(k.shape[0] * k.shape[1])
        self._ok(self._L.atus_strang_block_rabi(self._c, int(nk), int(kind), None if Fa is None else _dptr(Fa),
                                                len(comps), cs, _dptr(k), k.shape[1], float(thr), _dptr(out)),
                 "strang_block_rabi")
        return out.reshape(k.shape[0], k.shape[1])

    # ------------------------------------------------------------ observables
    def particle_number(self, comp: int = 0) -> float:
        v = C.c_double()
        self._ok(self._L.atus_particle_number(self._c, comp, C.byref(v)), "particle_number")
        return v.value

    def expval_position(self, comp: int = 0) -> np.ndarray:
        out = np.zeros(3)
        self._ok(self._L.atus_expval_position(self._c, comp, _dptr(out)), "expval_position")
        return out[: self.dim]

    def expval_momentum(self, comp: int = 0) -> np.ndarray:
        out = np.zeros(3)
        self._ok(self._L.atus_expval_momentum(self._c, comp, _dptr(out)), "expval_momentum")
        return out[: self.dim]

    def setup_momentum(self, comp: int, p) -> None:
        a = np.zeros(3)
        a[: len(p)] = p
        self._ok(self._L.atus_setup_momentum(self._c, comp, _dptr(a)), "setup_momentum")

    def rabi_integrals(self, k0, thr: float, comp: int = 0) -> np.ndarray:
        k = np.ascontiguousarray(k0, dtype=np.float64).reshape(-1, self.dim)
        out = np.zeros(k.shape[0])
        self._ok(self._L.atus_rabi_integrals_comp(self._c, int(comp), _dptr(k), k.shape[0], float(thr),
                                                  _dptr(out)), "rabi_integrals")
        return out

    # ------------------------------------------------------------ Sobolev gradient
    def sob_init(self, alpha_per_comp, stepsize: float) -> None:
        a = np.ascontiguousarray(alpha_per_comp, dtype=np.float64)
        self._ok(self._L.atus_sob_init(self._c, _dptr(a), float(stepsize)), "sob_init")

    def sob_renormalize(self) -> None:
        self._ok(self._L.atus_sob_renormalize(self._c), "sob_renormalize")

    def sob_iterate(self, n_iter: int = 1):
        res = C.c_double()
        N = np.zeros(MAX_COMP)
        self._ok(self._L.atus_sob_iterate(self._c, int(n_iter), C.byref(res), _dptr(N)), "sob_iterate")
        return res.value, N[: self.ncomp]

    def sob_run(self, epsilon: float, max_iter: int):
        it = C.c_int()
        res = C.c_double()
        self._ok(self._L.atus_sob_run(self._c, float(epsilon), int(max_iter), C.byref(it), C.byref(res)), "sob_run")
        return it.value, res.value

    def guess_decode(self, comp: int, coef, scale) -> None:
        """Fill component comp with the Hermite expansion coef (64) at basis lengths scale (3)."""
        c = np.ascontiguousarray(coef, dtype=np.float64)
        sc = np.ascontiguousarray(scale, dtype=np.float64)
        self._ok(self._L.atus_guess_decode(self._c, comp, _dptr(c), _dptr(sc)), "guess_decode")

    def embed_from(self, small: "Solver", comp: int = 0, comp_small: int = 0) -> None:
        """Component comp := `small`'s component comp_small (same spacing,
        fewer points) centred in this grid, zero elsewhere (FP64)."""
        self._ok(self._L.atus_embed(small._c, int(comp_small), self._c, int(comp)), "embed")

    def sob_mu(self) -> np.ndarray:
        mu = np.zeros(MAX_COMP)
        self._ok(self._L.atus_sob_mu(self._c, _dptr(mu)), "sob_mu")
        return mu[: self.ncomp]


class Batch:
    """Many independent two-component bragg_ad runs advanced together
    (atus_batch_*): ``instances`` is a list of dicts with ``header`` (1D or
    square 2D .bin header), ``alpha``, ``gs`` (4 values), ``laser`` (a
    ``Laser``) and ``pulse`` = (tc, sigma) of AMP_T."""

    def __init__(self, instances, precision: int = PREC_MIXED, dt: float = 1e-3):
        self._L = load_library()
        arr = (BatchInstance * len(instances))()
        self.shapes = []
        for i, d in enumerate(instances):
            h = d["header"]
            arr[i].grid = grid_from_header(h)
            arr[i].alpha = float(d.get("alpha", 0.5))
            for q, g in enumerate(d["gs"]):
                arr[i].gs[q] = float(g)
            arr[i].laser = d["laser"]
            arr[i].pulse_tc, arr[i].pulse_sigma = (float(x) for x in d.get("pulse", (0.0, 0.0)))
            arr[i].bragg_stable = int(bool(d.get("bragg_stable", False)))
            dim = int(h["nDims"])
            self.shapes.append(tuple(int(h[f"nDim{a}"]) for a in "XYZ"[:dim]))
        self._b = C.c_void_p()
        r = self._L.atus_batch_create(arr, len(instances), int(precision), float(dt), C.byref(self._b))
        if r != ATUS_OK:
            raise AtusError(f"atus_batch_create failed: {_ERRORS.get(r, r)}")
        self.count = len(instances)

    def close(self):
        if getattr(self, "_b", None) and self._b.value:
            self._L.atus_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, r: int, what: str):
        if r != ATUS_OK:
            msg = self._L.atus_batch_last_error(self._b)
            raise AtusError(f"{what}: {_ERRORS.get(r, r)}: {msg.decode() if msg else ''}")

    def set_psi(self, i: int, comp: int, data) -> None:
        a = np.ascontiguousarray(np.asarray(data, dtype=np.complex128).reshape(self.shapes[i]))
        self._ok(self._L.atus_batch_upload_psi(self._b, i, comp, _dptr(a.view(np.float64))), "batch_upload_psi")

    def psi(self, i: int, comp: int) -> np.ndarray:
        out = np.empty(self.shapes[i], dtype=np.complex128)
        self._ok(self._L.atus_batch_download_psi(self._b, i, comp, _dptr(out.view(np.float64))), "batch_download_psi")
        return out

    def time(self, i: int) -> float:
        t = C.c_double()
        self._ok(self._L.atus_batch_get_time(self._b, i, C.byref(t)), "batch_get_time")
        return t.value

    def tune(self, probe_steps: int = 20) -> None:
        self._ok(self._L.atus_batch_tune(self._b, int(probe_steps)), "batch_tune")

    def run(self, nk: int) -> float:
        """One Strang block of nk steps for every instance; device ms of the graph launch."""
        ms = C.c_double()
        self._ok(self._L.atus_batch_run(self._b, int(nk), C.byref(ms)), "batch_run")
        return ms.value

    def schedule(self) -> str:
        buf = C.create_string_buffer(8192)
        self._ok(self._L.atus_batch_schedule(self._b, buf, len(buf)), "batch_schedule")
        return buf.value.decode()
