"""Python host mirror of the reference's interface for the hot path.

The reference drives the step from C++ globals and free functions
(src/update.h:14-81, src/FlowField.h, src/ParticleTrack.h); ``Solver`` keeps
those names and argument meanings on top of the C ABI (include/gkm.h):

    reference                                   Solver
    GetParams / segment / MAKE5s / DevAlloc     Solver(params, cfl, ...)
    Initialize_DHIT(W)                          upload_state(W)
    evolve(W, dev, dt)            GPUupdate.h   evolve(W, dt)          (host arrays in/out)
    evolveEulerian + HaloTransfer update.cpp    evolve_eulerian(nsteps)
    timestep(W)                                 timestep()
    generateSplines (u, v, w)                   generate_splines()
    locateParticles / getParticleProp           particles_upload(pos, U=None)
    Evolve's loop body                          step(nsteps)
    PrintStats                                  print_stats()

Arrays follow the reference layout: W is (5, nt, nt, nt) float64 in (y, x, z)
order with 3 ghost layers; particle positions are (np, 3) as (y, x, z).
Errors raise GkmError carrying the gkm_status code.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from .ic import Params

_dp = C.POINTER(C.c_double)


class GkmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{_capi.STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _w5(W):
    """Five component pointers of a (5, nt, nt, nt) float64 array: a NumPy array
    (host) or a CUDA tensor (device; the C ABI copies either way)."""
    if hasattr(W, "data_ptr"):   # torch tensor
        import torch
        if W.dtype != torch.float64 or not W.is_contiguous() or W.dim() != 4 or W.shape[0] != 5:
            raise ValueError("W must be a contiguous float64 tensor of shape (5, nt, nt, nt)")
        return (_dp * 5)(*[C.cast(C.c_void_p(W[q].data_ptr()), _dp) for q in range(5)])
    if W.dtype != np.float64 or not W.flags.c_contiguous or W.ndim != 4 or W.shape[0] != 5:
        raise ValueError("W must be a C-contiguous float64 array of shape (5, nt, nt, nt)")
    return (_dp * 5)(*[_ptr(W[q]) for q in range(5)])


def make_config(params: Params, cfl: float = 0.10, visc_law: int = 0, spline_mode: int = 0,
                max_particles: int = 0, device: int = 0, use_graphs: bool = True,
                precision: int = 0, spline_build: int = 0, test_wait_probe: int = 0,
                spline_precision: int = 0) -> _capi.GkmConfig:
    L = _capi.lib()
    cfg = _capi.GkmConfig()
    L.gkm_config_default(C.byref(cfg))
    cfg.params = _capi.GkmParams(n=params.n, gam=params.gam, den0=params.den0, Mt=params.Mt, Re=params.Re,
                                 mu0=params.mu0, p0=params.p0, t0=params.t0)
    cfg.cfl = cfl
    cfg.visc_law = visc_law
    cfg.spline_mode = spline_mode
    cfg.device = device
    cfg.max_particles = max_particles
    cfg.use_graphs = 1 if use_graphs else 0
    cfg.precision = precision   # 0 FP64, 1 mixed (FP32 reconstruction + flux, FP64 state)
    cfg.spline_build = spline_build   # 0 auto, 1 one component per launch, 2 three components per launch
    cfg.test_wait_probe = test_wait_probe   # failure-detection test hook (gkm.h), 0 in normal use
    cfg.spline_precision = spline_precision   # 0 FP64 velocity-spline coefficients, 1 FP32 (same FP64 solves)
    return cfg


class Solver:
    def __init__(self, params: Params, cfl: float = 0.10, visc_law: int = 0, spline_mode: int = 0,
                 max_particles: int = 0, device: int = 0, use_graphs: bool = True, precision: int = 0,
                 spline_build: int = 0, test_wait_probe: int = 0, spline_precision: int = 0,
                 _member_handle=None):
        self.L = _capi.lib()
        self._owned = _member_handle is None
        if self._owned:
            cfg = make_config(params, cfl, visc_law, spline_mode, max_particles, device, use_graphs, precision,
                              spline_build, test_wait_probe, spline_precision)
            h = C.c_void_p()
            s = self.L.gkm_create(C.byref(cfg), C.byref(h))
            if s != 0:
                raise GkmError(s, "gkm_create failed (see stderr)")
        else:
            h = C.c_void_p(_member_handle)
        self.h = h
        self.params = params
        self.device = device
        self.n = params.n
        self.nt = self.L.gkm_nt(h)
        self.spline_mode = spline_mode
        self.np = 0

    # -- plumbing ----------------------------------------------------------
    def _check(self, s: int) -> None:
        if s != 0:
            raise GkmError(s, self.L.gkm_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            if self._owned:
                self.L.gkm_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- field ---------------------------------------------------------------
    def upload_state(self, W: np.ndarray) -> None:
        self._check(self.L.gkm_upload_state(self.h, _w5(W)))

    def download_state(self, out=None):
        """Current state (ghosts wrapped) into ``out`` (NumPy array or CUDA tensor) or a new NumPy array."""
        out = np.empty((5, self.nt, self.nt, self.nt)) if out is None else out
        self._check(self.L.gkm_download_state(self.h, _w5(out)))
        return out

    def device_state(self):
        """The current state in device memory as a CUDA tensor view (5, nt, nt, nt), no copy
        (gkm_device_state); valid until the next step, which writes the other buffer."""
        import torch

        p = C.POINTER(C.c_double)()
        self._check(self.L.gkm_device_state(self.h, C.byref(p)))
        view = type("DeviceState", (), {})()
        view.__cuda_array_interface__ = {"shape": (5, self.nt, self.nt, self.nt), "typestr": "<f8",
                                         "data": (C.cast(p, C.c_void_p).value, False), "version": 2}
        return torch.as_tensor(view, device=f"cuda:{self.device}")

    def timestep(self) -> float:
        dt = C.c_double()
        self._check(self.L.gkm_timestep(self.h, C.byref(dt)))
        return dt.value

    def set_dt(self, dt: float) -> None:
        self._check(self.L.gkm_set_dt(self.h, dt))

    def evolve_eulerian(self, nsteps: int = 1) -> None:
        self._check(self.L.gkm_evolve_eulerian(self.h, nsteps))

    def evolve(self, W: np.ndarray, dt: float) -> None:
        """The reference GPU plug point evolve(W, dev, dt): W updated in place."""
        self._check(self.L.gkm_evolve(self.h, _w5(W), dt))

    def set_pipeline(self, chunk_planes: int = 0, compute_streams: int = 2) -> None:
        """Shape of the evolve() pipeline used with pinned or device buffers."""
        self._check(self.L.gkm_set_pipeline(self.h, chunk_planes, compute_streams))

    def step(self, nsteps: int = 1) -> None:
        self._check(self.L.gkm_step(self.h, nsteps))

    def evolve_particles(self) -> None:
        """generateSplines + evolveParticles of the current state (the Lagrangian half of a step)."""
        self._check(self.L.gkm_evolve_particles(self.h))

    def step_timed(self, nsteps: int, with_particles: bool = True) -> dict:
        """nsteps with CUDA-event timing of each phase (milliseconds summed over the steps)."""
        ms = np.zeros(7)
        self._check(self.L.gkm_step_timed(self.h, nsteps, 1 if with_particles else 0, _ptr(ms)))
        keys = ("sweep_x", "sweep_y", "sweep_z", "halo", "splines", "particles", "total")
        return dict(zip(keys, ms.tolist()))

    def autotune(self, reps: int = 2) -> list:
        """Pick the fastest window and segment length per sweep direction on the current state."""
        self._check(self.L.gkm_autotune(self.h, reps))
        return self.sweep_config()

    def sweep_config(self) -> list:
        out = (C.c_int32 * 12)()
        self._check(self.L.gkm_sweep_config(self.h, out))
        return [{"dir": "xyz"[d], "variant": out[4 * d], "window": [out[4 * d + 1], out[4 * d + 2]],
                 "segment": out[4 * d + 3]} for d in range(3)]

    def set_sweep_config(self, shapes) -> None:
        """shapes: three (window variant, segment length) pairs for x, y, z."""
        arr = (C.c_int32 * 6)(*[int(x) for pair in shapes for x in pair])
        self._check(self.L.gkm_set_sweep_config(self.h, arr))

    def launch_count(self) -> int:
        n = C.c_int64()
        self._check(self.L.gkm_launch_count(self.h, C.byref(n)))
        return n.value

    def set_stream(self, stream_ptr: int | None) -> None:
        self._check(self.L.gkm_set_stream(self.h, stream_ptr))

    def clock(self):
        t, dt, it = C.c_double(), C.c_double(), C.c_int64()
        self._check(self.L.gkm_get_clock(self.h, C.byref(t), C.byref(dt), C.byref(it)))
        return t.value, dt.value, it.value

    def synchronize(self) -> None:
        self._check(self.L.gkm_synchronize(self.h))

    # -- particles -------------------------------------------------------------
    def particles_upload(self, pos_yxz: np.ndarray, U: np.ndarray | None = None) -> None:
        pos = np.ascontiguousarray(pos_yxz, dtype=np.float64)
        Up = None if U is None else _ptr(np.ascontiguousarray(U, dtype=np.float64))
        self._check(self.L.gkm_particles_upload(self.h, len(pos), _ptr(pos) if len(pos) else None, Up))
        self.np = len(pos)

    def particles_download(self):
        pos = np.empty((self.np, 3))
        U = np.empty((self.np, 3))
        self._check(self.L.gkm_particles_download(self.h, _ptr(pos), _ptr(U)))
        return pos, U

    # -- splines / stats -------------------------------------------------------
    def generate_splines(self) -> None:
        self._check(self.L.gkm_generate_splines(self.h))

    def spline_coefs(self, c: int) -> np.ndarray:
        N = self.nt if self.spline_mode == 0 else self.n
        M = N + (2 if self.spline_mode == 0 else 3)
        out = np.empty((M, M, M))
        self._check(self.L.gkm_spline_coefs(self.h, c, _ptr(out), out.size))
        return out

    def print_stats(self) -> dict:
        st = _capi.GkmStats()
        self._check(self.L.gkm_stats_compute(self.h, C.byref(st)))
        return st.as_dict()

    # -- particle properties and output files ------------------------------------
    def particle_props(self) -> np.ndarray:
        """getParticleProp for every particle: (np, 41), columns _capi.PROP_NAMES."""
        out = np.empty((self.np, _capi.PROP_COUNT))
        self._check(self.L.gkm_particle_props(self.h, _ptr(out) if self.np else None))
        return out

    def particle_stats(self) -> dict:
        """GetParticleStats: particle TKE, SijSij, SKEWu, SKEWw."""
        st = _capi.GkmParticleStats()
        self._check(self.L.gkm_particle_stats_compute(self.h, C.byref(st)))
        return st.as_dict()

    def write_field(self, path: str) -> None:
        self._check(self.L.gkm_write_field(self.h, path.encode()))

    def write_particles(self, path: str) -> None:
        self._check(self.L.gkm_write_particles(self.h, path.encode()))

    def write_time(self, path: str) -> None:
        self._check(self.L.gkm_write_time(self.h, path.encode()))

    def write_reinit(self, path: str) -> None:
        self._check(self.L.gkm_write_reinit(self.h, path.encode()))

    def write_outputs(self, directory: str, iteration: int, rank: int = 0) -> dict:
        """The files the reference writes at an output iteration, under its own names
        (Results/Field, Results/Particles, Results/Time, InitialCondition)."""
        import os
        paths = {"field": os.path.join(directory, "Results", "Field", f"Field_{rank}_{iteration}"),
                 "particles": os.path.join(directory, "Results", "Particles", f"P_{rank}_{iteration}"),
                 "time": os.path.join(directory, "Results", "Time", f"T_{iteration}"),
                 "reinit": os.path.join(directory, "InitialCondition", "Init000")}
        for p in paths.values():
            os.makedirs(os.path.dirname(p), exist_ok=True)
        self.write_field(paths["field"])
        self.write_reinit(paths["reinit"])
        self.write_particles(paths["particles"])
        self.write_time(paths["time"])
        return paths


class Ensemble:
    """Many independent cubes stepped together, one launch per stage (gkm_ensemble_*).

    ``members`` is a list of dicts with the keyword arguments of Solver
    (params, cfl, visc_law, spline_mode, max_particles); all share ``device``
    and ``precision``.  ``ens[m]`` is a Solver view of member m (upload_state,
    download_state, particles_upload, print_stats, clock, ... act on that
    member); the ensemble owns the members.
    """

    def __init__(self, members: list, device: int = 0, precision: int = 0):
        self.L = _capi.lib()
        cfgs = (_capi.GkmConfig * len(members))()
        for i, m in enumerate(members):
            cfgs[i] = make_config(m["params"], m.get("cfl", 0.10), m.get("visc_law", 0), m.get("spline_mode", 0),
                                  m.get("max_particles", 0), device, True, precision)
        h = C.c_void_p()
        s = self.L.gkm_ensemble_create(cfgs, len(members), C.byref(h))
        if s != 0:
            raise GkmError(s, "gkm_ensemble_create failed (see stderr)")
        self.h = h
        self.members = [Solver(m["params"], spline_mode=m.get("spline_mode", 0),
                               _member_handle=self.L.gkm_ensemble_member(h, i)) for i, m in enumerate(members)]

    def _check(self, s: int) -> None:
        if s != 0:
            raise GkmError(s, self.L.gkm_ensemble_last_error(self.h).decode())

    def __len__(self) -> int:
        return len(self.members)

    def __getitem__(self, m: int) -> Solver:
        return self.members[m]

    def close(self) -> None:
        if getattr(self, "h", None):
            for m in self.members:
                m.h = None
            self.L.gkm_ensemble_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, nsteps: int = 1, with_particles: bool = True) -> None:
        self._check(self.L.gkm_ensemble_step(self.h, nsteps, 1 if with_particles else 0))

    def step_timed(self, nsteps: int, with_particles: bool = True) -> dict:
        ms = np.zeros(7)
        self._check(self.L.gkm_ensemble_step_timed(self.h, nsteps, 1 if with_particles else 0, _ptr(ms)))
        keys = ("sweep_x", "sweep_y", "sweep_z", "halo", "splines", "particles", "total")
        return dict(zip(keys, ms.tolist()))

    def autotune(self, reps: int = 2) -> list:
        self._check(self.L.gkm_ensemble_autotune(self.h, reps))
        return self.sweep_config()

    def sweep_config(self) -> list:
        out = (C.c_int32 * 12)()
        self._check(self.L.gkm_ensemble_sweep_config(self.h, out))
        segs = self.segments()
        cfg = []
        for d in range(3):
            by_n = {}
            for m, L in enumerate(segs[d]):
                by_n[self.members[m].n] = L
            cfg.append({"dir": "xyz"[d], "variant": out[4 * d], "window": [out[4 * d + 1], out[4 * d + 2]],
                        "segment": out[4 * d + 3], "segment_by_grid_size": dict(sorted(by_n.items()))})
        return cfg

    def set_sweep_config(self, shapes) -> None:
        """shapes: three (window variant, segment length) pairs for x, y, z, one length for every member."""
        arr = (C.c_int32 * 6)(*[int(x) for pair in shapes for x in pair])
        self._check(self.L.gkm_ensemble_set_sweep_config(self.h, arr))

    def segments(self) -> list:
        """Segment length of every member, per sweep direction: [x list, y list, z list]."""
        nm = len(self)
        out = (C.c_int32 * (3 * nm))()
        self._check(self.L.gkm_ensemble_segments(self.h, out, 3 * nm))
        return [[out[d * nm + m] for m in range(nm)] for d in range(3)]

    def launch_count(self) -> int:
        n = C.c_int64()
        self._check(self.L.gkm_ensemble_launch_count(self.h, C.byref(n)))
        return n.value

    def synchronize(self) -> None:
        self._check(self.L.gkm_ensemble_synchronize(self.h))

    def stream(self) -> int:
        """The ensemble's cudaStream_t as an integer (torch.cuda.ExternalStream accepts it)."""
        p = C.c_void_p()
        self._check(self.L.gkm_ensemble_stream(self.h, C.byref(p)))
        return p.value or 0


def probe_fma_peak(device: int = 0):
    """(fp64, fp32) FMA throughput of the device in TFLOP/s."""
    L = _capi.lib()
    a, b = C.c_double(), C.c_double()
    s = L.gkm_probe_fma_peak(device, C.byref(a), C.byref(b))
    if s != 0:
        raise GkmError(s, "gkm_probe_fma_peak")
    return a.value, b.value


def flux_faces(inputs: np.ndarray, gam: float, dt: float, dx: float) -> np.ndarray:
    """flux() on independent faces: inputs (nf, 51) = WL WR Wl Wr DW[6x5] tau."""
    L = _capi.lib()
    a = np.ascontiguousarray(inputs, dtype=np.float64)
    F = np.zeros((len(a), 5))
    s = L.gkm_flux_faces(_ptr(a), len(a), gam, dt, dx, _ptr(F))
    if s != 0:
        raise GkmError(s, "gkm_flux_faces")
    return F


def weno_faces(stencils: np.ndarray, gam: float):
    """ApplyWENO on stencils (n, 6, 5) -> (Wl, Wr) each (n, 5)."""
    L = _capi.lib()
    a = np.ascontiguousarray(stencils, dtype=np.float64)
    Wl = np.zeros((len(a), 5))
    Wr = np.zeros((len(a), 5))
    s = L.gkm_weno_faces(_ptr(a), len(a), gam, _ptr(Wl), _ptr(Wr))
    if s != 0:
        raise GkmError(s, "gkm_weno_faces")
    return Wl, Wr
