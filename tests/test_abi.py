"""C ABI checks that need no GPU: libsrcuda.so loads, exports every entry point
include/srcuda.h declares, and the ctypes mirrors have the C struct layouts."""
import ctypes
import os
import re
import subprocess

import pytest

from spatialrust_b200 import _native
from spatialrust_b200.csrc import build as csrc_build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "srcuda.h")


@pytest.fixture(scope="module")
def lib():
    csrc_build.build()
    return _native.load()


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(srcu_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "srcu_voxel_centroid" in names and "srcu_radius_normals" in names
    assert len(names) >= 12


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.check_output(["nm", "-D", "--defined-only", _native.library_path()], text=True)
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, f"not exported: {missing}"


def test_ctypes_signatures_cover_header(lib):
    assert set(declared_functions()) == set(_native.SIGNATURES)


def test_abi_version(lib):
    assert lib.srcu_abi_version() == 1


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "sizes.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "srcuda.h"\n'
        "int main(void){\n"
        'printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(srcu_cloud), sizeof(srcu_voxel_params),'
        " sizeof(srcu_voxel_out), sizeof(srcu_normal_params), sizeof(srcu_normal_out),"
        " sizeof(srcu_normal_stats), sizeof(srcu_frame_view), sizeof(srcu_server_config),"
        " sizeof(srcu_request_result), sizeof(srcu_server_stats));\n"
        'printf("%zu %zu %zu %zu %zu\\n", offsetof(srcu_cloud, n),'
        " offsetof(srcu_normal_params, include_self), offsetof(srcu_frame_view, n_attrs),"
        " offsetof(srcu_request_result, points), offsetof(srcu_server_stats, frame_p50_ms));\n"
        'printf("%zu %zu %zu %zu %zu\\n", sizeof(srcu_stream_voxel_params),'
        " sizeof(srcu_stream_voxel_info), sizeof(srcu_stream_voxel_out),"
        " offsetof(srcu_stream_voxel_params, run_points),"
        " offsetof(srcu_stream_voxel_out, on_device));\n"
        "return 0;}\n")
    exe = tmp_path / "sizes"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)])
    lines = subprocess.check_output([str(exe)], text=True).split("\n")
    sizes = [int(v) for v in lines[0].split()]
    offs = [int(v) for v in lines[1].split()]
    assert sizes == [ctypes.sizeof(t) for t in (
        _native.SrcuCloud, _native.SrcuVoxelParams, _native.SrcuVoxelOut, _native.SrcuNormalParams,
        _native.SrcuNormalOut, _native.SrcuNormalStats, _native.SrcuFrameView,
        _native.SrcuServerConfig, _native.SrcuRequestResult, _native.SrcuServerStats)]
    assert offs == [_native.SrcuCloud.n.offset, _native.SrcuNormalParams.include_self.offset,
                    _native.SrcuFrameView.n_attrs.offset, _native.SrcuRequestResult.points.offset,
                    _native.SrcuServerStats.frame_p50_ms.offset]
    stream = [int(v) for v in lines[2].split()]
    assert stream == [ctypes.sizeof(_native.SrcuStreamVoxelParams),
                      ctypes.sizeof(_native.SrcuStreamVoxelInfo),
                      ctypes.sizeof(_native.SrcuStreamVoxelOut),
                      _native.SrcuStreamVoxelParams.run_points.offset,
                      _native.SrcuStreamVoxelOut.on_device.offset]


def test_header_compiles_as_c_and_cxx(tmp_path):
    for comp, ext in (("gcc", "c"), ("g++", "cpp")):
        src = tmp_path / f"inc.{ext}"
        src.write_text('#include "srcuda.h"\nint main(void){ return srcu_abi_version() == 1 ? 0 : 1; }\n')
        subprocess.check_call([comp, "-c", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                               "-o", str(tmp_path / f"inc_{ext}.o"), str(src)])


def test_create_without_device_reports_no_device(lib):
    """On a machine without a B200 the context refuses cleanly (no abort)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = ctypes.c_void_p()
    st = lib.srcu_create(0, 0, ctypes.byref(h))
    assert st == _native.SRCU_ERR_NO_DEVICE
    assert not h.value
    assert lib.srcu_last_error(None) == b"no context"


def test_server_without_device_or_budget(lib):
    """The serving loop refuses cleanly: slots larger than the HBM budget, bad
    size relations, and (here) no device."""
    import torch
    cfg = _native.SrcuServerConfig()
    h = ctypes.c_void_p()
    cfg.hbm_budget_bytes = 1 << 20
    assert lib.srcu_server_create(ctypes.byref(cfg), ctypes.byref(h)) == _native.SRCU_ERR_OUT_OF_BUDGET
    cfg.hbm_budget_bytes = 0
    cfg.bulk_threshold_points = 2_000_000  # above frame_batch_points (1M default)
    assert (lib.srcu_server_create(ctypes.byref(cfg), ctypes.byref(h))
            == _native.SRCU_ERR_INVALID_ARGUMENT)
    assert lib.srcu_server_create(None, None) == _native.SRCU_ERR_INVALID_ARGUMENT
    if torch.cuda.is_available():
        return
    with pytest.raises(_native.NoDevice):
        _native.Server(0)
    assert not h.value
