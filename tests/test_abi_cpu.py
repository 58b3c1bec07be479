"""The C-ABI library loads and exports every entry point that
include/appearance_cuda.h declares; argument checks run without a GPU."""
import ctypes
import os
import re
import struct

import numpy as np

from appearance_b200 import _native, presets, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "appearance_cuda.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ap_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = _native.load()
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s
    assert set(_native.EXPORTS) <= set(syms)


def test_config_default_matches_reference_literals():
    c = _native.FrameConfig()
    _native.load().ap_frame_config_default(ctypes.byref(c))
    got = {k: getattr(c, k) for k, _ in _native.FrameConfig._fields_}
    for k, v in presets.FAITHFUL.items():
        assert abs(got[k] - v) < 1e-6, k


def test_null_handle_is_rejected_without_a_gpu():
    lib = _native.load()
    buf = ctypes.create_string_buffer(80)
    assert lib.ap_world_action(None, 0, buf, 80) == _native.AP_E_INVALID
    assert lib.ap_render_hdr(None, 4, 4, 0, 4, None, 0, None) == _native.AP_E_INVALID
    assert lib.ap_trace_rays(None, None, None, 0, 0, None) == _native.AP_E_INVALID
    assert lib.ap_last_error(None) == b"null handle"


def test_struct_layouts():
    assert ctypes.sizeof(_native.FrameConfig) == 20 * 4
    assert ctypes.sizeof(_native.Mesh) == 6 * 4
    assert scenes.MAT_FLOATS == 26


def test_camera_update_wire_format():
    from appearance_b200.renderer import PathTracer
    m = np.eye(4, dtype=np.float32)
    b = PathTracer.camera_update_bytes(m, 60.0, 0.1, 300.0)
    assert len(b) == 80  # CameraUpdateData: Mat4 + fov + near + far + pad
    assert struct.unpack_from("<fff", b, 64) == (60.0, np.float32(0.1), 300.0)


def _c_params(src, name):
    m = re.search(r"\b" + name + r"\s*\(([^)]*)\)", src, re.S)
    args = m.group(1).strip()
    return 0 if args in ("", "void") else len(args.split(","))


def test_rust_ffi_crate_declares_the_header():
    """ffi/appearance-path-tracer-cuda/src/ffi.rs (no Rust toolchain here to
    compile it) declares every entry point of the header with as many
    parameters, and its #[repr(C)] structs list the header's fields in order."""
    hdr = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "appearance_cuda.h")).read(), flags=re.S)
    rs = open(os.path.join(ROOT, "ffi", "appearance-path-tracer-cuda", "src", "ffi.rs")).read()
    rs_fns = dict(re.findall(r"pub fn (ap_[a-z0-9_]+)\(([^)]*)\)", rs, re.S))
    assert sorted(rs_fns) == declared_symbols()
    for name, args in rs_fns.items():
        n_rs = 0 if not args.strip() else len([a for a in args.split(",") if a.strip()])
        assert n_rs == _c_params(hdr, name), name
    for c_name, rs_name in (("ap_frame_config", "ApFrameConfig"), ("ap_material", "ApMaterial"),
                            ("ap_mesh", "ApMesh"), ("ap_frame_stats", "ApFrameStats"), ("ap_job", "ApJob"),
                            ("ap_job_result", "ApJobResult")):
        body = re.search(r"typedef struct " + c_name + r" \{(.*?)\} " + c_name, hdr, re.S).group(1)
        c_fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            names = decl.split(None, 1)[1] if decl.split()[0] not in ("const",) else decl.split(None, 2)[2]
            c_fields += [n.strip().lstrip("*").split("[")[0] for n in names.split(",")]
        rs_body = re.search(r"pub struct " + rs_name + r" \{(.*?)\n\}", rs, re.S).group(1)
        rs_fields = re.findall(r"pub ([a-z0-9_]+):", rs_body)
        assert rs_fields == c_fields, rs_name
