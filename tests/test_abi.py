"""The C ABI library: loads without a GPU, exports every declared symbol, and its
structs have the sizes the ctypes mirror assumes."""
import ctypes as C
import os
import re

import pytest

from pelemp_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "pmp_spray.h")).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(pmp_\w+)\s*\(", src, re.M)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for n in ("pmp_spray_create", "pmp_spray_update", "pmp_spray_update_host",
              "pmp_spray_set_particles", "pmp_spray_get_particles", "pmp_spray_setup"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from pelemp_b200 import spray
    L = spray.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert b"sm_100a" in L.pmp_spray_version()


def test_struct_sizes_match_c(oracle):
    sizes = oracle.abi_sizes()
    mirror = [capi.Geometry, capi.Box, capi.BoxView, capi.SprayComps, capi.SprayData,
              capi.SprayInputs, capi.Particles, capi.SprayConfig, capi.ErrorInfo, capi.Stats,
              capi.Mech, capi.LaunchConfig, capi.TuneReport, capi.LearnConfig, capi.LearnReport]
    assert len(sizes) == len(mirror)
    for s, m in zip(sizes, mirror):
        assert s == C.sizeof(m), m.__name__


def test_create_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from pelemp_b200 import spray
    with pytest.raises(spray.SprayError) as e:
        spray.SprayParticleContainer(["N2", "O2", "NC7H16"], 1)
    assert e.value.code == capi.PMP_ERR_NO_DEVICE


def test_invalid_arguments_rejected_without_gpu():
    from pelemp_b200 import spray
    L = spray.lib()
    assert L.pmp_spray_create(None, None) == capi.PMP_ERR_INVALID
    assert L.pmp_spray_set_host_source_in(None, 0) == capi.PMP_ERR_INVALID
    cfg = capi.SprayConfig()
    cfg.nfuel = 0
    cfg.nspec = 3
    h = C.c_void_p()
    assert L.pmp_spray_create(C.byref(cfg), C.byref(h)) == capi.PMP_ERR_INVALID
