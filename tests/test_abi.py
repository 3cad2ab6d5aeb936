"""The C-ABI libraries load and export every symbol their headers declare."""
import ctypes
import os
import re

from conftest import ROOT
from flite3d_b200 import _abi


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\bint\s+(f(?:lite|p)_\w+)\s*\(", text)))


def test_gpu_library_exports_header():
    lib = _abi.gpu_lib()
    names = _declared("flite_gpu.h")
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_abi.GPU_SYMBOLS) | (set(names) - set(_abi.GPU_SYMBOLS))


def test_prepro_library_exports_header():
    lib = _abi.prepro_lib()
    for n in _declared("flite_prepro.h"):
        assert hasattr(lib, n), n


def test_struct_sizes_match_c():
    # sizeof(flite_controls) and sizeof(flite_level_desc) as compiled
    # five counts (+4 padding), 17 arrays, the engine side count (+4) and its two arrays
    assert ctypes.sizeof(_abi.LevelDesc) == 5 * 4 + 4 + 17 * 8 + 4 + 4 + 2 * 8


def test_create_rejects_unsupported_controls():
    from flite3d_b200 import Mesh, default_controls
    m = Mesh.bump_channel(4, 2, 2, 0.05, nlevels=1)
    lib = _abi.gpu_lib()
    h = ctypes.c_void_p()
    for bad in (dict(flowType=3), dict(flowType=2, physicalTimeStep=0.1, precision=1), dict(turbulenceModel=2),
                dict(movingwall=1),
                dict(ReynoldsNumber=0.0, multigridScheme=6)):
        c = default_controls(**bad)
        rc = lib.flite_create(ctypes.byref(c), m.nlevels, m.descs, ctypes.byref(h))
        assert rc == _abi.FLITE_EUNSUPPORTED, bad
        # the reason is kept for the calling thread, retrieved with a NULL context
        buf = ctypes.create_string_buffer(256)
        assert lib.flite_last_error(None, buf, len(buf)) == _abi.FLITE_OK
        assert buf.value, bad
    assert b"multigridScheme" in buf.value


def test_fortran_interface_module_matches_the_c_abi():
    # include/flite_gpu_mod.f90: its bind(C) names are exported symbols and
    # its flite_controls type lists the C struct's fields in order and kind
    text = open(os.path.join(ROOT, "include", "flite_gpu_mod.f90")).read()
    code = "\n".join(ln.split("!")[0] for ln in text.splitlines())
    code = code.replace("&\n", " ")
    lib = _abi.gpu_lib()
    names = re.findall(r'bind\(C,\s*name="(\w+)"\)', code)
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    body = re.search(r"type, bind\(C\) :: flite_controls\n(.*?)end type flite_controls", code, re.S).group(1)
    fields = []
    for ln in body.splitlines():
        m = re.match(r"\s*(real|integer)\(c_(\w+)\)\s*::\s*(.*)", ln)
        if not m:
            continue
        for item in m.group(3).split(","):
            item = item.strip()
            if not item:
                continue
            nm = re.match(r"(\w+)(?:\((\d+)\))?", item)
            fields.append((nm.group(1), m.group(2), int(nm.group(2) or 1)))
    want = []
    for name, typ in _abi.Controls._fields_:
        n = getattr(typ, "_length_", 1)
        base = typ._type_ if hasattr(typ, "_length_") else typ
        want.append((name, "double" if base is ctypes.c_double else "int", n))
    assert fields == want
