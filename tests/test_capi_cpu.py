"""C-ABI checks that need no GPU: the library loads, exports every entry point
include/gkm.h declares, and rejects bad arguments before touching CUDA."""
import ctypes as C
import os
import re

import pytest

from dns_gkm_lpt_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "gkm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gkm_[a-z_0-9]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    L = _capi.lib()
    decl = declared_symbols()
    assert len(decl) >= 20
    for name in decl:
        assert hasattr(L, name), name
    assert sorted(_capi.EXPORTS) == decl


def test_abi_version_and_defaults():
    L = _capi.lib()
    assert L.gkm_abi_version() == 1
    cfg = _capi.GkmConfig()
    L.gkm_config_default(C.byref(cfg))
    assert cfg.cfl == 0.10 and cfg.visc_law == 0 and cfg.spline_mode == 0 and cfg.use_graphs == 1
    assert cfg.test_wait_probe == 0


def test_struct_layout_matches_header():
    # gkm_params: 2 ints + 7 doubles; gkm_config adds cfl, 4 ints, int64, 8 ints
    assert C.sizeof(_capi.GkmParams) == 8 + 7 * 8
    assert C.sizeof(_capi.GkmConfig) == C.sizeof(_capi.GkmParams) + 8 + 16 + 8 + 32
    assert C.sizeof(_capi.GkmStats) == 13 * 8


@pytest.mark.parametrize("field,value", [("n", 2), ("gam", 1.0), ("den0", 0.0), ("p0", -1.0)])
def test_create_rejects_bad_config_without_gpu(field, value):
    L = _capi.lib()
    cfg = _capi.GkmConfig()
    L.gkm_config_default(C.byref(cfg))
    cfg.params.n, cfg.params.gam, cfg.params.den0, cfg.params.p0, cfg.params.mu0 = 16, 1.4, 1.0, 86100.0, 1.0
    setattr(cfg.params, field, value)
    h = C.c_void_p()
    assert L.gkm_create(C.byref(cfg), C.byref(h)) == _capi.GKM_ERR_CONFIG
    assert not h.value


def test_create_rejects_bad_enums_and_null():
    L = _capi.lib()
    cfg = _capi.GkmConfig()
    L.gkm_config_default(C.byref(cfg))
    cfg.params.n, cfg.params.gam, cfg.params.den0, cfg.params.p0, cfg.params.mu0 = 16, 1.4, 1.0, 86100.0, 1.0
    h = C.c_void_p()
    for f, v in (("spline_mode", 7), ("visc_law", -1), ("precision", 3), ("precision", -1), ("test_wait_probe", 2),
                 ("test_wait_probe", -1)):
        c2 = _capi.GkmConfig.from_buffer_copy(cfg)
        setattr(c2, f, v)
        assert L.gkm_create(C.byref(c2), C.byref(h)) == _capi.GKM_ERR_CONFIG
    assert L.gkm_create(None, C.byref(h)) == _capi.GKM_ERR_ARG
    assert L.gkm_destroy(None) == _capi.GKM_ERR_ARG
    assert L.gkm_flux_faces(None, -1, 1.4, 1e-4, 0.1, None) == _capi.GKM_ERR_ARG
    assert L.gkm_flux_faces(None, 0, 1.4, 1e-4, 0.1, None) == _capi.GKM_OK


def test_null_handle_calls_fail_cleanly():
    L = _capi.lib()
    assert L.gkm_step(None, 1) == _capi.GKM_ERR_ARG
    assert L.gkm_timestep(None, None) == _capi.GKM_ERR_ARG
    assert L.gkm_last_error(None) == b"null handle"


def test_ensemble_and_new_entry_points_reject_bad_arguments_without_gpu():
    L = _capi.lib()
    h = C.c_void_p()
    assert L.gkm_ensemble_create(None, 1, C.byref(h)) == _capi.GKM_ERR_ARG
    cfgs = (_capi.GkmConfig * 2)()
    for c in cfgs:
        L.gkm_config_default(C.byref(c))
        c.params.n, c.params.gam, c.params.den0, c.params.p0, c.params.mu0 = 16, 1.4, 1.0, 86100.0, 1.0
    assert L.gkm_ensemble_create(cfgs, 0, C.byref(h)) == _capi.GKM_ERR_ARG
    cfgs[1].precision = 1   # members must share the precision
    assert L.gkm_ensemble_create(cfgs, 2, C.byref(h)) == _capi.GKM_ERR_CONFIG
    cfgs[1].precision = 0
    cfgs[1].device = 3      # and the device
    assert L.gkm_ensemble_create(cfgs, 2, C.byref(h)) == _capi.GKM_ERR_CONFIG
    assert L.gkm_ensemble_destroy(None) == _capi.GKM_ERR_ARG
    assert L.gkm_ensemble_step(None, 1, 1) == _capi.GKM_ERR_ARG
    assert L.gkm_ensemble_size(None) == 0
    assert L.gkm_ensemble_member(None, 0) is None
    assert L.gkm_ensemble_last_error(None) == b"null ensemble"
    for fn in ("gkm_write_field", "gkm_write_particles", "gkm_write_time", "gkm_write_reinit"):
        assert getattr(L, fn)(None, b"/dev/null") == _capi.GKM_ERR_ARG
    assert L.gkm_particle_props(None, None) == _capi.GKM_ERR_ARG
    assert L.gkm_particle_stats_compute(None, None) == _capi.GKM_ERR_ARG
    assert L.gkm_set_pipeline(None, 32, 2) == _capi.GKM_ERR_ARG
    assert L.gkm_spline_build_noalloc(None, 16, 0, 1, None, None) != _capi.GKM_OK


def test_reference_gpu_build_exports_the_plug_point():
    """The reference's -D UseGPU build linked with dns_gkm_lpt_b200/plug/GPUupdate_b200.cpp loads
    (its libgkm_b200.so dependency resolves) and defines evolve(ptype*[5], DevAlloc*, ptype) and
    DevAlloc's constructor and destructor (src/GPUupdate.h:33, src/GPUAlloc.h:8-26)."""
    import ctypes
    import subprocess
    so = os.path.join(ROOT, "oracle", "_ref", "libgkm_ref_gpu.so")
    if not os.path.exists(so):
        pytest.skip("oracle/_ref/libgkm_ref_gpu.so is built by `make -C oracle` where the reference tree exists")
    ctypes.CDLL(so)
    syms = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    for s in ("_Z6evolvePPdP8DevAllocd", "_ZN8DevAllocC1Ev", "_ZN8DevAllocD1Ev", "gkmrefgpu_setup", "gkmrefgpu_run"):
        assert f" {s}\n" in syms, s
