"""ctypes access to the CPU oracle — TEST INFRASTRUCTURE ONLY.

* ``Oracle``: oracle/libgkm_oracle.so, the plain-C restatement of the
  reference algorithm (oracle/gkm_oracle.c).
* ``ReferenceRun``: oracle/_ref/libgkm_ref.so, the reference's own CPU sources
  compiled in place with a one-rank MPI stand-in (oracle/Makefile).  It keeps
  process-wide state (the reference uses globals), so use one run at a time per
  process.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
arm may import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libgkm_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libgkm_ref.so")

_dp = C.POINTER(C.c_double)


def build(ref: bool = True) -> None:
    """Build the oracle libraries (the reference one only where the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE] + ([] if ref else [os.path.join(HERE, "libgkm_oracle.so")]),
                   check=True)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


class OrcParams(C.Structure):
    _fields_ = [("n", C.c_int), ("nt", C.c_int), ("K", C.c_int), ("visc_law", C.c_int),
                ("gam", C.c_double), ("den0", C.c_double), ("p0", C.c_double), ("Mt", C.c_double),
                ("Re", C.c_double), ("mu0", C.c_double), ("t0", C.c_double),
                ("dx", C.c_double), ("T0", C.c_double), ("cfl", C.c_double)]


class OrcStats(C.Structure):
    _fields_ = [(k, C.c_double) for k in
                ("TKE", "Diss", "SijSij", "SKEWu", "SKEWv", "SKEWw", "KURTu", "KURTv", "KURTw",
                 "Prms", "Trms", "Vrms")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class OrcSpline(C.Structure):
    _fields_ = [("coefs", _dp), ("n", C.c_int * 3), ("periodic", C.c_int),
                ("start", C.c_double * 3), ("dinv", C.c_double * 3)]


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(ref=False)
        L = C.CDLL(path)
        self.L = L
        L.orc_params_init.argtypes = [C.POINTER(OrcParams), C.c_int] + [C.c_double] * 8
        L.orc_flux.argtypes = [_dp] * 10 + [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _dp]
        L.orc_weno.argtypes = [_dp] * 6 + [C.c_double, _dp, _dp]
        L.orc_step.argtypes = [C.POINTER(OrcParams), _dp * 5, _dp * 5, _dp * 5, _dp * 5, C.c_double]
        L.orc_timestep.argtypes = [C.POINTER(OrcParams), _dp * 5]
        L.orc_timestep.restype = C.c_double
        L.orc_max_wave_speed.argtypes = [C.POINTER(OrcParams), _dp * 5]
        L.orc_max_wave_speed.restype = C.c_double
        L.orc_halo.argtypes = [C.POINTER(OrcParams), _dp * 5]
        L.orc_sweep.argtypes = [C.POINTER(OrcParams), C.c_int, _dp * 5, _dp * 5, C.c_double]
        L.orc_run.argtypes = [C.POINTER(OrcParams), _dp * 5, C.c_int, C.c_int, C.c_long, _dp, _dp, _dp,
                              C.POINTER(OrcStats)]
        L.orc_run.restype = C.c_int
        L.orc_spline1d.argtypes = [_dp, C.c_long, C.c_int, C.c_int, _dp, C.c_long]
        L.orc_spline3d_build.argtypes = [_dp, C.c_int * 3, C.c_int, _dp, _dp]
        L.orc_spline3d_eval.argtypes = [C.POINTER(OrcSpline), C.c_double, C.c_double, C.c_double, C.c_int,
                                        _dp, _dp, _dp, _dp]
        L.orc_spline_pad.argtypes = [C.c_int]
        L.orc_spline_pad.restype = C.c_int
        L.orc_grid_natural_ghost3.argtypes = [C.POINTER(OrcParams), _dp, _dp]
        L.orc_grid_periodic.argtypes = [C.POINTER(OrcParams), _dp, _dp]
        L.orc_print_stats.argtypes = [C.POINTER(OrcParams), _dp * 5] + [C.POINTER(OrcSpline)] * 4 + [
            C.POINTER(OrcStats)]
        L.orc_particle_props.argtypes = [C.POINTER(OrcParams), _dp * 5, C.c_int, C.c_long, _dp, _dp]
        L.orc_particle_stats.argtypes = [_dp, C.c_long, _dp]

    # -- parameters ----------------------------------------------------------
    def params(self, P, cfl: float, visc_law: int = 0) -> OrcParams:
        p = OrcParams()
        self.L.orc_params_init(C.byref(p), P.n, P.gam, P.den0, P.Mt, P.Re, P.mu0, P.p0, P.t0, cfl)
        p.visc_law = visc_law
        return p

    @staticmethod
    def _w5(W: np.ndarray):
        return (_dp * 5)(*[_ptr(W[q]) for q in range(5)])

    # -- numerics --------------------------------------------------------------
    def flux(self, WL, WR, Wl, Wr, DWxl, DWxr, DWyl, DWyr, DWzl, DWzr, tau, dt, dx, gam, K=2):
        F = np.zeros(5)
        args = [np.ascontiguousarray(a, dtype=np.float64) for a in (WL, WR, Wl, Wr, DWxl, DWxr, DWyl, DWyr, DWzl, DWzr)]
        self.L.orc_flux(*[_ptr(a) for a in args], tau, dt, dx, gam, K, _ptr(F))
        return F

    def weno(self, s6x5: np.ndarray, gam: float):
        s = np.ascontiguousarray(s6x5, dtype=np.float64)
        Wl, Wr = np.zeros(5), np.zeros(5)
        self.L.orc_weno(*[_ptr(s[o]) for o in range(6)], gam, _ptr(Wl), _ptr(Wr))
        return Wl, Wr

    def halo(self, p: OrcParams, W: np.ndarray) -> None:
        self.L.orc_halo(C.byref(p), self._w5(W))

    def timestep(self, p: OrcParams, W: np.ndarray) -> float:
        return self.L.orc_timestep(C.byref(p), self._w5(W))

    def max_wave_speed(self, p: OrcParams, W: np.ndarray) -> float:
        return self.L.orc_max_wave_speed(C.byref(p), self._w5(W))

    def sweep(self, p: OrcParams, d: int, W: np.ndarray, dt: float) -> np.ndarray:
        F = np.zeros_like(W)
        self.L.orc_sweep(C.byref(p), d, self._w5(W), self._w5(F), dt)
        return F

    def step(self, p: OrcParams, W: np.ndarray, dt: float) -> None:
        """In place: evolveEulerian + HaloTransfer on W (5, nt, nt, nt)."""
        Fx, Fy, Fz = (np.zeros_like(W) for _ in range(3))
        self.L.orc_step(C.byref(p), self._w5(W), self._w5(Fx), self._w5(Fy), self._w5(Fz), dt)

    def run(self, p: OrcParams, W: np.ndarray, nsteps: int, spline_mode: int = 0, pos=None, stats=True):
        """Evolve's loop body nsteps times, in place on W.  pos: (np, 3) in (y, x, z) order.
        Returns dict(dt, U, pos, stats)."""
        npart = 0 if pos is None else len(pos)
        pos = np.zeros((0, 3)) if pos is None else np.ascontiguousarray(pos, dtype=np.float64).copy()
        U = np.zeros_like(pos)
        dts = np.zeros(max(nsteps, 1))
        st = (OrcStats * (nsteps // 10 + 2))()
        ns = self.L.orc_run(C.byref(p), self._w5(W), nsteps, spline_mode, npart,
                            _ptr(pos) if npart else None, _ptr(U) if npart else None, _ptr(dts),
                            st if stats else None)
        return {"dt": dts[:nsteps], "pos": pos, "U": U, "stats": [st[i].as_dict() for i in range(ns)]}

    def particle_props(self, p: OrcParams, W: np.ndarray, pos: np.ndarray, spline_mode: int = 0) -> np.ndarray:
        """getParticleProp with the eight splines of W (ghosts valid): (np, 41) property table."""
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        out = np.zeros((len(pos), 41))
        self.L.orc_particle_props(C.byref(p), self._w5(W), spline_mode, len(pos), _ptr(pos), _ptr(out))
        return out

    def particle_stats(self, props: np.ndarray) -> np.ndarray:
        """GetParticleStats on a property table: TKE, SijSij, SKEWu, SKEWw."""
        props = np.ascontiguousarray(props, dtype=np.float64)
        out = np.zeros(4)
        self.L.orc_particle_stats(_ptr(props), len(props), _ptr(out))
        return out

    # -- splines ---------------------------------------------------------------
    def spline1d(self, f: np.ndarray, periodic: int) -> np.ndarray:
        f = np.ascontiguousarray(f, dtype=np.float64)
        c = np.zeros(len(f) + self.L.orc_spline_pad(periodic))
        self.L.orc_spline1d(_ptr(f), 1, len(f), periodic, _ptr(c), 1)
        return c

    def spline3d(self, data: np.ndarray, periodic: int, start, dinv):
        data = np.ascontiguousarray(data, dtype=np.float64)
        P = self.L.orc_spline_pad(periodic)
        coefs = np.zeros(tuple(s + P for s in data.shape))
        n = (C.c_int * 3)(*data.shape)
        self.L.orc_spline3d_build(_ptr(data), n, periodic, _ptr(coefs), None)
        s = OrcSpline()
        s.coefs = _ptr(coefs)
        s.n = n
        s.periodic = periodic
        s.start = (C.c_double * 3)(*([start] * 3 if np.isscalar(start) else start))
        s.dinv = (C.c_double * 3)(*([dinv] * 3 if np.isscalar(dinv) else dinv))
        s._keep = coefs
        return s, coefs

    def eval(self, s: OrcSpline, a: float, b: float, c: float, what: int = 3):
        val = np.zeros(1)
        g = np.zeros(3)
        l = np.zeros(1)
        h = np.zeros(9)
        self.L.orc_spline3d_eval(C.byref(s), a, b, c, what, _ptr(val), _ptr(g), _ptr(l), _ptr(h))
        return val[0], g, l[0], h

    def grid(self, p: OrcParams, periodic: int):
        s, d = C.c_double(), C.c_double()
        fn = self.L.orc_grid_periodic if periodic else self.L.orc_grid_natural_ghost3
        fn(C.byref(p), C.byref(s), C.byref(d))
        return s.value, d.value


class ReferenceRun:
    """The reference CPU build (oracle/_ref) on one IC directory."""

    def __init__(self, icdir: str, cfl: float, with_particles: bool = True, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: build it with `make -C oracle` where the reference tree exists")
        L = C.CDLL(path)
        self.L = L
        L.gkmref_setup.argtypes = [C.c_char_p, C.c_double, C.c_int]
        L.gkmref_setup.restype = C.c_int
        L.gkmref_nt.restype = C.c_int
        for f in ("gkmref_dt", "gkmref_dx", "gkmref_time"):
            getattr(L, f).restype = C.c_double
        L.gkmref_get_W.argtypes = [_dp]
        L.gkmref_set_W.argtypes = [_dp]
        L.gkmref_get_flux.argtypes = [C.c_int, _dp]
        L.gkmref_set_cfl.argtypes = [C.c_double]
        L.gkmref_set_dt.argtypes = [C.c_double]
        L.gkmref_run.argtypes = [C.c_int, _dp, _dp, C.c_int]
        L.gkmref_run.restype = C.c_int
        L.gkmref_stats.argtypes = [_dp]
        L.gkmref_get_particles.argtypes = [_dp, _dp, C.POINTER(C.c_int)]
        L.gkmref_get_particles.restype = C.c_int
        L.gkmref_time_steps.argtypes = [C.c_int, _dp, _dp]
        L.gkmref_flux.argtypes = [_dp] * 10 + [C.c_double] * 4 + [_dp]
        L.gkmref_weno.argtypes = [_dp, C.c_double, _dp, _dp]
        L.gkmref_particle_table.argtypes = [_dp, C.POINTER(C.c_int)]
        L.gkmref_particle_table.restype = C.c_int
        L.gkmref_particle_stats.argtypes = [_dp]
        L.gkmref_write_outputs.argtypes = [C.c_char_p]
        L.gkmref_write_outputs.restype = C.c_int
        rc = L.gkmref_setup(icdir.encode(), cfl, 1 if with_particles else 0)
        if rc != 0:
            raise RuntimeError(f"gkmref_setup failed ({rc})")
        self.nt = L.gkmref_nt()

    @property
    def dt(self) -> float:
        return self.L.gkmref_dt()

    def W(self) -> np.ndarray:
        out = np.zeros((5, self.nt, self.nt, self.nt))
        self.L.gkmref_get_W(_ptr(out))
        return out

    def run(self, nsteps: int):
        dts = np.zeros(max(nsteps, 1))
        st = np.zeros((nsteps // 10 + 2, 16))
        ns = self.L.gkmref_run(nsteps, _ptr(dts), _ptr(st), len(st))
        return dts[:nsteps], st[:ns]

    def eulerian_step(self) -> None:
        self.L.gkmref_eulerian_step()

    def particle_props(self) -> None:
        """getParticleProp at the current positions (U of the next iteration's predictor)."""
        self.L.gkmref_particle_props()

    def stats(self) -> np.ndarray:
        out = np.zeros(16)
        self.L.gkmref_stats(_ptr(out))
        return out

    def particles(self, max_count: int):
        pos = np.zeros((max_count, 3))
        U = np.zeros((max_count, 3))
        tags = np.zeros(max_count, dtype=np.int32)
        n = self.L.gkmref_get_particles(_ptr(pos), _ptr(U), tags.ctypes.data_as(C.POINTER(C.c_int)))
        return pos[:n], U[:n], tags[:n]

    def particle_table(self, max_count: int):
        """getParticleProp at the current positions: (count, 41) property table and tags."""
        out = np.zeros((max_count, 41))
        tags = np.zeros(max_count, dtype=np.int32)
        n = self.L.gkmref_particle_table(_ptr(out), tags.ctypes.data_as(C.POINTER(C.c_int)))
        return out[:n], tags[:n]

    def particle_stats(self) -> np.ndarray:
        """GetParticleStats after particle_table: part_TKE, part_SijSij, part_SKEWu, part_SKEWw."""
        out = np.zeros(4)
        self.L.gkmref_particle_stats(_ptr(out))
        return out

    def write_outputs(self, directory: str) -> None:
        """The reference's own writeField / WriteReInit / writeParticleData into directory."""
        for sub in ("Results/Field", "Results/Particles", "Results/Time", "InitialCondition"):
            os.makedirs(os.path.join(directory, sub), exist_ok=True)
        rc = self.L.gkmref_write_outputs(directory.encode())
        if rc != 0:
            raise RuntimeError(f"gkmref_write_outputs failed ({rc})")

    def time_steps(self, nsteps: int):
        te, tp = C.c_double(), C.c_double()
        self.L.gkmref_time_steps(nsteps, C.byref(te), C.byref(tp))
        return te.value, tp.value

    def flux(self, WL, WR, Wl, Wr, DWxl, DWxr, DWyl, DWyr, DWzl, DWzr, tau, dt, dx, gam):
        F = np.zeros(5)
        args = [np.ascontiguousarray(a, dtype=np.float64) for a in (WL, WR, Wl, Wr, DWxl, DWxr, DWyl, DWyr, DWzl, DWzr)]
        self.L.gkmref_flux(*[_ptr(a) for a in args], tau, dt, dx, gam, _ptr(F))
        return F

    def weno(self, s6x5, gam):
        s = np.ascontiguousarray(s6x5, dtype=np.float64)
        Wl, Wr = np.zeros(5), np.zeros(5)
        self.L.gkmref_weno(_ptr(s), gam, _ptr(Wl), _ptr(Wr))
        return Wl, Wr


def write_case(directory: str, n: int, Mt: float, Re: float, seed: int, nparticles: int):
    """Write one seeded case in the reference's input formats; returns (params, W_ghost, pos_yxz)."""
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    from dns_gkm_lpt_b200 import ic
    P, u, v, w, rho, p = ic.make_field(n, Mt, Re, seed)
    xyz = ic.make_particles(nparticles, seed) if nparticles else None
    ic.write_reference_inputs(directory, P, u, v, w, rho, p, xyz)
    W = ic.embed_ghost(ic.primitive_to_conserved(P, u, v, w, rho, p))
    pos = ic.particles_to_reference_order(xyz) if nparticles else None
    return P, W, pos


def tmpdir() -> str:
    return tempfile.mkdtemp(prefix="gkm_case_")
