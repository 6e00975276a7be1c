"""ctypes front end of the oracle restatement (atus_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke`` and
by bench.py's CPU-baseline leg, never by the ``atus2_b200`` package.

``Oracle`` mirrors the state of one ``CRT_Base<T,dim,n>`` object (or of a
``CSOB_Base`` for the Sobolev routines): the fields, the kinetic tables, the
header time ``t``, and exposes the reference's step functions one by one plus
``block()`` (one outer iteration of run_sequence, include/CRT_Base.h:776-786).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle_atus.so")
REF_DIR = os.path.join(HERE, "_ref")

KIND_NL = 0  # CRT_Base::Do_NL_Step (rt_solver "freeprop")
KIND_NL_IF = 1  # CRT_Base_IF::Do_NL_Step (bragg "freeprop")
KIND_BRAGG_AD = 2  # Bragg_single::Do_Bragg_ad
KIND_DOUBLE_BRAGG_AD = 3  # Bragg_double::Do_Double_Bragg_ad (double_bragg)
KIND_NL_IF_2 = 4  # CRT_Base_IF_2::Do_NL_Step (two-species "freeprop")
KIND_BRAGG_DS_AD = 5  # Bragg_single::Do_Bragg_ad of bragg_ds


class Laser(C.Structure):
    """Mirror of the CRT_Base_IF laser members (include/CRT_Base_IF.h:65-77)."""

    _fields_ = [
        ("beta", C.c_double * 3),
        ("DeltaL", C.c_double * 4),
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
            if isinstance(v, (int, float)):
                if k == "chirp":
                    setattr(L, k, float(v))
                else:
                    f[0] = float(v)
            else:
                for i, x in enumerate(v):
                    f[i] = float(x)
        return L


_lib = None


def build(quiet: bool = True) -> None:
    """Compile the restatement (make -C oracle lib)."""
    subprocess.run(["make", "-C", HERE, "lib"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, dp, i, d = C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_double
        sig = {
            "orc_create": (vp, [i, i, C.POINTER(C.c_longlong), dp, dp]),
            "orc_destroy": (None, [vp]),
            "orc_psi": (dp, [vp, i]),
            "orc_npts": (C.c_long, [vp]),
            "orc_get_t": (d, [vp]),
            "orc_set_t": (None, [vp, d]),
            "orc_set_gs": (None, [vp, dp]),
            "orc_set_alpha": (None, [vp, i, dp]),
            "orc_set_potential": (None, [vp, i, dp]),
            "orc_set_dt": (None, [vp, d]),
            "orc_ft_step": (None, [vp, i]),
            "orc_nl_step": (None, [vp]),
            "orc_nl_if_step": (None, [vp, C.POINTER(Laser)]),
            "orc_bragg_ad": (None, [vp, C.POINTER(Laser), d]),
            "orc_block": (None, [vp, i, i, C.POINTER(Laser), dp]),
            "orc_particle_number": (d, [vp, i]),
            "orc_expval_position": (None, [vp, i, dp]),
            "orc_expval_momentum": (None, [vp, i, dp]),
            "orc_setup_momentum": (None, [vp, i, dp]),
            "orc_rabi_integrals": (None, [vp, dp, i, d, dp]),
            "orc_rabi_integrals_comp": (None, [vp, i, dp, i, d, dp]),
            "orc_set_species2": (None, [vp, C.POINTER(Laser), d, dp]),
            "orc_ft": (None, [vp, dp, i]),
            "orc_fft_raw": (None, [vp, dp, i]),
            "orc_sob_init": (None, [vp, dp, d]),
            "orc_sob_grad": (dp, [vp, i]),
            "orc_sob_renormalize": (None, [vp]),
            "orc_sob_iterate": (d, [vp, dp]),
            "orc_sob_run": (i, [vp, d, i, dp]),
            "orc_sob_mu": (None, [vp, dp]),
            "orc_set_threads": (None, [i]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """One solver state on a grid described by an ATUS-2 header."""

    def __init__(self, header, ncomp: int, threads: int = 1):
        L = lib()
        L.orc_set_threads(int(threads))
        self.dim = int(header["nDims"])
        self.shape = tuple(int(header[f"nDim{a}"]) for a in "XYZ"[: self.dim])
        n = (C.c_longlong * 3)(*(list(self.shape) + [1] * (3 - self.dim)))
        d = np.array([float(header[f"d{a}"]) for a in "xyz"], dtype=np.float64)
        dk = np.array([float(header[f"dk{a}"]) for a in "xyz"], dtype=np.float64)
        self.ncomp = ncomp
        self._c = L.orc_create(self.dim, ncomp, n, _dp(d), _dp(dk))
        if not self._c:
            raise ValueError("oracle: bad grid")
        self.npts = int(L.orc_npts(self._c))
        self.t = float(header["t"])

    def __del__(self):
        if getattr(self, "_c", None):
            lib().orc_destroy(self._c)
            self._c = None

    # state -------------------------------------------------------------
    def psi(self, comp: int) -> np.ndarray:
        """Live complex view of component ``comp`` (shape = grid)."""
        p = lib().orc_psi(self._c, comp)
        a = np.ctypeslib.as_array(p, shape=(self.npts * 2,))
        return a.view(np.complex128).reshape(self.shape)

    def set_psi(self, comp: int, data) -> None:
        self.psi(comp)[...] = np.asarray(data, dtype=np.complex128).reshape(self.shape)

    @property
    def t(self) -> float:
        return float(lib().orc_get_t(self._c))

    @t.setter
    def t(self, v: float) -> None:
        lib().orc_set_t(self._c, float(v))

    def set_gs(self, gs) -> None:
        a = np.ascontiguousarray(gs, dtype=np.float64).ravel()
        lib().orc_set_gs(self._c, _dp(a))

    def set_alpha(self, comp: int, alpha) -> None:
        a = np.zeros(3)
        a[: len(alpha)] = alpha
        lib().orc_set_alpha(self._c, comp, _dp(a))

    def set_potential(self, comp: int, V) -> None:
        if V is None:
            lib().orc_set_potential(self._c, comp, None)
        else:
            a = np.ascontiguousarray(V, dtype=np.float64).ravel()
            assert a.size == self.npts
            lib().orc_set_potential(self._c, comp, _dp(a))

    def set_dt(self, dt: float) -> None:
        lib().orc_set_dt(self._c, float(dt))

    # steps ---------------------------------------------------------------
    def ft_step(self, half: bool) -> None:
        lib().orc_ft_step(self._c, 1 if half else 0)

    def nl_step(self) -> None:
        lib().orc_nl_step(self._c)

    def nl_if_step(self, laser: Laser) -> None:
        lib().orc_nl_if_step(self._c, C.byref(laser))

    def bragg_ad(self, laser: Laser, F: float = 1.0) -> None:
        lib().orc_bragg_ad(self._c, C.byref(laser), float(F))

    def block(self, nk: int, kind: int, laser: Laser | None = None, F=None) -> None:
        laser = laser if laser is not None else Laser()
        Fa = None if F is None else np.ascontiguousarray(F, dtype=np.float64)
        if Fa is not None:
            assert Fa.size >= nk
        lib().orc_block(self._c, int(nk), int(kind), C.byref(laser), None if Fa is None else _dp(Fa))

    # observables ---------------------------------------------------------
    def particle_number(self, comp: int = 0) -> float:
        return float(lib().orc_particle_number(self._c, comp))

    def expval_position(self, comp: int = 0) -> np.ndarray:
        out = np.zeros(3)
        lib().orc_expval_position(self._c, comp, _dp(out))
        return out[: self.dim]

    def expval_momentum(self, comp: int = 0) -> np.ndarray:
        out = np.zeros(3)
        lib().orc_expval_momentum(self._c, comp, _dp(out))
        return out[: self.dim]

    def setup_momentum(self, comp: int, p) -> None:
        a = np.zeros(3)
        a[: len(p)] = p
        lib().orc_setup_momentum(self._c, comp, _dp(a))

    def rabi_integrals(self, k0, thr: float, comp: int = 0) -> np.ndarray:
        k = np.ascontiguousarray(k0, dtype=np.float64).reshape(-1, self.dim)
        out = np.zeros(k.shape[0])
        lib().orc_rabi_integrals_comp(self._c, int(comp), _dp(k), k.shape[0], float(thr), _dp(out))
        return out

    def set_species2(self, laser2: Laser, t_start: float = 0.0, durations=(np.inf, np.inf)) -> None:
        """Second species of CRT_Base_IF_2 and the pulse windows of bragg_ds's
        bragg_ad (seq.time and seq.duration[0..1])."""
        dur = np.ascontiguousarray(durations, dtype=np.float64)
        lib().orc_set_species2(self._c, C.byref(laser2), float(t_start), _dp(dur))

    def ft(self, data: np.ndarray, isign: int) -> None:
        """cft_Nd::ft on an external complex array (in place)."""
        assert data.dtype == np.complex128 and data.flags.c_contiguous and data.size == self.npts
        lib().orc_ft(self._c, data.ctypes.data_as(C.POINTER(C.c_double)), int(isign))

    def fft_raw(self, data: np.ndarray, isign: int) -> None:
        assert data.dtype == np.complex128 and data.flags.c_contiguous and data.size == self.npts
        lib().orc_fft_raw(self._c, data.ctypes.data_as(C.POINTER(C.c_double)), int(isign))

    # Sobolev gradient (CSOB_Base) ------------------------------------------
    def sob_init(self, alpha_per_comp, stepsize: float) -> None:
        a = np.ascontiguousarray(alpha_per_comp, dtype=np.float64)
        lib().orc_sob_init(self._c, _dp(a), float(stepsize))

    def sob_grad(self, comp: int) -> np.ndarray:
        p = lib().orc_sob_grad(self._c, comp)
        return np.ctypeslib.as_array(p, shape=(self.npts * 2,)).view(np.complex128).reshape(self.shape)

    def sob_renormalize(self) -> None:
        lib().orc_sob_renormalize(self._c)

    def sob_iterate(self):
        N = np.zeros(4)
        res = float(lib().orc_sob_iterate(self._c, _dp(N)))
        return res, N[: self.ncomp]

    def sob_run(self, epsilon: float, max_iter: int):
        res = np.zeros(1)
        it = int(lib().orc_sob_run(self._c, float(epsilon), int(max_iter), _dp(res)))
        return it, float(res[0])

    def sob_mu(self) -> np.ndarray:
        mu = np.zeros(4)
        lib().orc_sob_mu(self._c, _dp(mu))
        return mu[: self.ncomp]


def pulse_times(t0: float, dt: float, nk: int, nblocks: int = 1):
    """Header times at each potential step of ``nblocks`` run_sequence blocks.

    Replays the reference's float additions: half step t += 0.5*dt, full step
    t += dt (include/CRT_Base.h:361,391).  Returns (t at each potential step,
    t after the last block)."""
    t = t0
    out = []
    for _ in range(nblocks):
        t += 0.5 * dt
        for _j in range(2, nk + 1):
            out.append(t)
            t += dt
        out.append(t)
        t += 0.5 * dt
    return np.array(out), t
