"""ctypes binding of include/gkm.h (libgkm_b200.so).

The library is the product: there is no Python or CPU fallback.  If the
shared object is missing this module raises at import, so a run on a machine
without the built library fails loudly instead of silently computing
something else.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("GKM_B200_LIB", os.path.join(PKG, "lib", "libgkm_b200.so"))

GKM_OK, GKM_ERR_ARG, GKM_ERR_CONFIG, GKM_ERR_CUDA, GKM_ERR_NONFINITE, GKM_ERR_STATE, GKM_ERR_NOMEM = range(7)
STATUS_NAMES = {0: "GKM_OK", 1: "GKM_ERR_ARG", 2: "GKM_ERR_CONFIG", 3: "GKM_ERR_CUDA", 4: "GKM_ERR_NONFINITE",
                5: "GKM_ERR_STATE", 6: "GKM_ERR_NOMEM"}

# every entry point declared in include/gkm.h
EXPORTS = [
    "gkm_config_default", "gkm_create", "gkm_destroy", "gkm_last_error", "gkm_abi_version", "gkm_nt",
    "gkm_upload_state", "gkm_download_state", "gkm_timestep", "gkm_set_dt", "gkm_evolve_eulerian", "gkm_evolve",
    "gkm_step", "gkm_get_clock", "gkm_synchronize", "gkm_particles_upload", "gkm_particles_download",
    "gkm_generate_splines", "gkm_spline_coefs", "gkm_stats_compute", "gkm_flux_faces", "gkm_weno_faces",
    "gkm_set_stream", "gkm_device_state", "gkm_evolve_particles", "gkm_step_timed", "gkm_launch_count",
    "gkm_probe_fma_peak", "gkm_spline_build_noalloc", "gkm_autotune", "gkm_sweep_config",
    "gkm_ensemble_create", "gkm_ensemble_destroy", "gkm_ensemble_last_error", "gkm_ensemble_size",
    "gkm_ensemble_member", "gkm_ensemble_step", "gkm_ensemble_step_timed", "gkm_ensemble_autotune",
    "gkm_ensemble_sweep_config", "gkm_ensemble_launch_count", "gkm_ensemble_synchronize", "gkm_ensemble_stream",
    "gkm_particle_props", "gkm_particle_stats_compute", "gkm_write_field", "gkm_write_particles", "gkm_write_time",
    "gkm_write_reinit", "gkm_set_pipeline", "gkm_ensemble_segments", "gkm_set_sweep_config",
    "gkm_ensemble_set_sweep_config",
]

PROP_COUNT = 41
PROP_NAMES = (["rho"] + [f"grad_rho_{a}" for a in "yxz"] + ["u", "v", "w"]
              + [f"grad_{c}_{a}" for c in "uvw" for a in "yxz"] + ["p"] + [f"grad_p_{a}" for a in "yxz"]
              + [f"hess_p_{a}{b}" for a in "yxz" for b in "yxz"] + ["lap_u", "lap_v", "lap_w"]
              + [f"grad_lap_{c}_{a}" for c in "uvw" for a in "yxz"])


class GkmParams(C.Structure):
    _fields_ = [("n", C.c_int32), ("pad_", C.c_int32), ("gam", C.c_double), ("den0", C.c_double),
                ("Mt", C.c_double), ("Re", C.c_double), ("mu0", C.c_double), ("p0", C.c_double),
                ("t0", C.c_double)]


class GkmConfig(C.Structure):
    _fields_ = [("params", GkmParams), ("cfl", C.c_double), ("visc_law", C.c_int32), ("spline_mode", C.c_int32),
                ("precision", C.c_int32), ("device", C.c_int32), ("max_particles", C.c_int64),
                ("use_graphs", C.c_int32), ("spline_build", C.c_int32), ("test_wait_probe", C.c_int32),
                ("spline_precision", C.c_int32), ("reserved", C.c_int32 * 4)]


class GkmParticleStats(C.Structure):
    _fields_ = [("TKE", C.c_double), ("SijSij", C.c_double), ("SKEWu", C.c_double), ("SKEWw", C.c_double),
                ("count", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class GkmStats(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("t_over_t0", "TKE", "Diss", "SijSij", "SKEWu", "SKEWv", "SKEWw",
                                          "KURTu", "KURTv", "KURTw", "Prms", "Trms", "Vrms")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_dp = C.POINTER(C.c_double)
_h = C.c_void_p


def load(path: str = LIB_PATH) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(f"libgkm_b200.so not found at {path}: build it with `python -m dns_gkm_lpt_b200.build`")
    L = C.CDLL(path)
    st = C.c_int
    L.gkm_config_default.argtypes = [C.POINTER(GkmConfig)]
    L.gkm_config_default.restype = None
    L.gkm_create.argtypes = [C.POINTER(GkmConfig), C.POINTER(_h)]
    L.gkm_destroy.argtypes = [_h]
    L.gkm_last_error.argtypes = [_h]
    L.gkm_last_error.restype = C.c_char_p
    L.gkm_abi_version.argtypes = []
    L.gkm_nt.argtypes = [_h]
    L.gkm_upload_state.argtypes = [_h, _dp * 5]
    L.gkm_download_state.argtypes = [_h, _dp * 5]
    L.gkm_timestep.argtypes = [_h, _dp]
    L.gkm_set_dt.argtypes = [_h, C.c_double]
    L.gkm_evolve_eulerian.argtypes = [_h, C.c_int32]
    L.gkm_evolve.argtypes = [_h, _dp * 5, C.c_double]
    L.gkm_step.argtypes = [_h, C.c_int32]
    L.gkm_get_clock.argtypes = [_h, _dp, _dp, C.POINTER(C.c_int64)]
    L.gkm_synchronize.argtypes = [_h]
    L.gkm_particles_upload.argtypes = [_h, C.c_int64, _dp, _dp]
    L.gkm_particles_download.argtypes = [_h, _dp, _dp]
    L.gkm_generate_splines.argtypes = [_h]
    L.gkm_spline_coefs.argtypes = [_h, C.c_int32, _dp, C.c_int64]
    L.gkm_stats_compute.argtypes = [_h, C.POINTER(GkmStats)]
    L.gkm_flux_faces.argtypes = [_dp, C.c_int64, C.c_double, C.c_double, C.c_double, _dp]
    L.gkm_weno_faces.argtypes = [_dp, C.c_int64, C.c_double, _dp, _dp]
    L.gkm_set_stream.argtypes = [_h, C.c_void_p]
    L.gkm_device_state.argtypes = [_h, C.POINTER(_dp)]
    L.gkm_evolve_particles.argtypes = [_h]
    L.gkm_step_timed.argtypes = [_h, C.c_int32, C.c_int32, _dp]
    L.gkm_launch_count.argtypes = [_h, C.POINTER(C.c_int64)]
    L.gkm_probe_fma_peak.argtypes = [C.c_int32, _dp, _dp]
    L.gkm_autotune.argtypes = [_h, C.c_int32]
    L.gkm_sweep_config.argtypes = [_h, C.POINTER(C.c_int32)]
    L.gkm_set_sweep_config.argtypes = [_h, C.POINTER(C.c_int32)]
    L.gkm_spline_build_noalloc.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]
    L.gkm_ensemble_create.argtypes = [C.POINTER(GkmConfig), C.c_int32, C.POINTER(_h)]
    L.gkm_ensemble_destroy.argtypes = [_h]
    L.gkm_ensemble_last_error.argtypes = [_h]
    L.gkm_ensemble_last_error.restype = C.c_char_p
    L.gkm_ensemble_size.argtypes = [_h]
    L.gkm_ensemble_member.argtypes = [_h, C.c_int32]
    L.gkm_ensemble_member.restype = _h
    L.gkm_ensemble_step.argtypes = [_h, C.c_int32, C.c_int32]
    L.gkm_ensemble_step_timed.argtypes = [_h, C.c_int32, C.c_int32, _dp]
    L.gkm_ensemble_autotune.argtypes = [_h, C.c_int32]
    L.gkm_ensemble_sweep_config.argtypes = [_h, C.POINTER(C.c_int32)]
    L.gkm_ensemble_segments.argtypes = [_h, C.POINTER(C.c_int32), C.c_int64]
    L.gkm_ensemble_set_sweep_config.argtypes = [_h, C.POINTER(C.c_int32)]
    L.gkm_ensemble_launch_count.argtypes = [_h, C.POINTER(C.c_int64)]
    L.gkm_ensemble_synchronize.argtypes = [_h]
    L.gkm_ensemble_stream.argtypes = [_h, C.POINTER(C.c_void_p)]
    L.gkm_set_pipeline.argtypes = [_h, C.c_int32, C.c_int32]
    L.gkm_particle_props.argtypes = [_h, _dp]
    L.gkm_particle_stats_compute.argtypes = [_h, C.POINTER(GkmParticleStats)]
    for w in ("gkm_write_field", "gkm_write_particles", "gkm_write_time", "gkm_write_reinit"):
        getattr(L, w).argtypes = [_h, C.c_char_p]
    for name in EXPORTS:
        if name not in ("gkm_config_default", "gkm_last_error", "gkm_ensemble_last_error", "gkm_ensemble_member"):
            getattr(L, name).restype = st   # gkm_status, or int for gkm_abi_version / gkm_nt
    return L


_LIB = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = load()
    return _LIB
