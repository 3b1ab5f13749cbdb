"""The C-ABI library loads and exports every entry point declared in include/*.h."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(ymrt_[a-z_0-9]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    import ymrt_b200 as Y
    lib = Y.library()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert declared_symbols(), "no declarations found"
    assert not missing, f"missing exports: {missing}"


def test_render_setting_is_reference_layout():
    import ymrt_b200 as Y
    assert ctypes.sizeof(Y.RenderSetting) == 40
    assert Y.RenderSetting.indirect_limit.offset == 36
    assert Y.RenderSetting.enable_distant_light.offset == 28


def test_no_device_is_an_error_not_a_fallback():
    import ymrt_b200 as Y
    from conftest import cuda_available
    if cuda_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(Y.YmrtError) as e:
        Y.Context(0)
    assert e.value.code == -9


def test_compat_library_exports_the_reference_launchers():
    """libymrt_compat.so exports the seventeen extern "C" launchers the
    reference's RenderModule declares (src/core/RenderModule.cpp:14-46,
    without its two ImGui test hooks), so that module links against it."""
    import ctypes
    import ymrt_b200 as Y
    Y.library()
    names = ["AllocateRayCounter", "ReleaseRayCounter", "AllocateShadingRayData", "ReleaseShadingRayData",
             "AllocateHitData", "ReleaseHitData", "AllocateShadowRayData", "ReleaseShadowRayData",
             "RayGenerationEditorView", "RayTraceEditorView", "RayShadingEditorView", "RayGenerationPathTracing",
             "RayTracePathTracing", "RayShadingPathTracing", "AccumulateImagePathTracing", "PostProcessingEditorView",
             "PostProcessingPathTracing"]
    lib = ctypes.CDLL(os.path.join(ROOT, "ymrt_b200", "libymrt_compat.so"))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
