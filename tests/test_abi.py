"""The C-ABI library builds for sm_100a, loads, and exports every entry point
declared in include/ovs.h (CPU only; no compute call is made)."""
import ctypes
import re
from pathlib import Path

import numpy as np

from oversetdevfort_b200 import _ffi as F
from oversetdevfort_b200 import mesh as M

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    txt = (ROOT / "include" / "ovs.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(?:int|const char\*)\s+(ovs_\w+)\s*\(", txt)))


def test_header_declarations_exported(lib):
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"{n} declared in ovs.h but not exported"
    assert sorted(F.EXPORTS) == names, "ctypes signature table out of sync with ovs.h"


def test_library_is_sm100a_build(lib):
    # the fat binary carries sm_100a code only (checked on the object list)
    from oversetdevfort_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)
    assert build.LIB.exists()


def test_status_strings(lib):
    for s in (0, 1, -1, -2, -3, -4, -5, -6, -7, -8):
        assert lib.ovs_status_string(s)
    assert lib.ovs_version() >= 10000


def test_create_argument_errors(lib):
    h = ctypes.c_void_p()
    bad = F.OvsDims(0, 10, 4, 0)
    assert lib.ovs_create(ctypes.byref(h), ctypes.byref(bad)) == F.OVS_ERR_ARG
    bad = F.OvsDims(10, 10, 5, 0)
    assert lib.ovs_create(ctypes.byref(h), ctypes.byref(bad)) == F.OVS_ERR_ARG
    assert lib.ovs_destroy(None) == 0
    assert lib.ovs_assemble_async(None, F.OVS_ASM_NSVOF, 6, F.OVS_FP32) == F.OVS_ERR_ARG
    assert lib.ovs_assemble_wait(None, None) == F.OVS_ERR_ARG


def test_params_struct_layout():
    # 30 doubles then 4 ints: offsets must match the C struct
    assert ctypes.sizeof(F.OvsParams) == 30 * 8 + 4 * 4
    assert F.OvsParams.gravvec.offset == 27 * 8
    assert F.OvsParams.fluid_elm_id.offset == 30 * 8


def test_mesh_generator_counts():
    m = M.box_tet(4, 3, 2)
    assert m.nnode == 5 * 4 * 3 and m.nelem == 6 * 24
    assert m.ien.min() == 1 and m.ien.max() == m.nnode
    assert all(len(f) > 0 for f in m.faces)
    c = M.config1(n=4)
    assert c.ibc[:, :3].sum() > 0 and c.ibc[:, 3:].sum() == 0
    lid = c.mesh.faces[5]
    np.testing.assert_array_equal(c.state["ug"][lid, 0], 1.0)


def test_missing_library_fails_loudly(tmp_path):
    """No CPU fallback: loading a library that is not there raises, naming the
    build step."""
    import pytest
    with pytest.raises(OSError, match="oversetdevfort_b200.build"):
        F.load(tmp_path / "libovs_b200.so")


def test_context_without_device_raises(lib):
    """On a machine without a CUDA device the public API refuses to run
    (OVS_ERR_NODEVICE) instead of computing elsewhere."""
    import pytest
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from oversetdevfort_b200.api import Context
    with pytest.raises(Exception, match="(?i)device"):
        Context(8, 6, 4)


def test_product_code_never_imports_the_oracle():
    """The oracle is test infrastructure: nothing in the package imports it,
    and bench.py reaches it only from its CPU-baseline and reference legs."""
    pkg = ROOT / "oversetdevfort_b200"
    pat = re.compile(r"^\s*(from\s+oracle\b|import\s+oracle\b)", re.M)
    for f in pkg.rglob("*.py"):
        assert not pat.search(f.read_text()), f"{f} imports the oracle"
    for f in (pkg / "csrc").glob("*"):
        assert "ovs_oracle" not in f.read_text(), f"{f} refers to the oracle"
    bench = (ROOT / "bench.py").read_text()
    for m in re.finditer(r"^(\s*)(from\s+oracle\b|import\s+oracle\b).*$", bench, re.M):
        # every import sits inside a function whose name says it is a baseline leg
        head = bench[: m.start()]
        fn = re.findall(r"^def (\w+)\(", head, re.M)
        assert fn and ("cpu" in fn[-1] or "reference" in fn[-1] or "baseline" in fn[-1]), (fn[-1:], m.group(0))


def test_binding_covers_every_entry_point():
    """The Python binding's export list and signature table name exactly the
    entry points include/ovs.h declares."""
    declared = set(_declared())
    assert set(F.EXPORTS) == declared, (sorted(declared - set(F.EXPORTS)), sorted(set(F.EXPORTS) - declared))
    assert len(F.EXPORTS) == len(set(F.EXPORTS))


def test_smoke_needs_the_device():
    """__graft_entry__.smoke() runs the CUDA path only: without a device it
    raises instead of passing on the oracle."""
    import pytest
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import __graft_entry__ as g
    with pytest.raises(F.OvsError):
        g.smoke()


def test_every_kernel_launch_is_counted():
    """ovs_launch_count (and bench.py's gpu_launches from it) covers every
    kernel a context launches: each launch site in csrc/ is followed within
    a few lines by an increment of the context's counter.  The one exception
    is ovs_gmres_tem_noalloc, which has no context."""
    csrc = ROOT / "oversetdevfort_b200" / "csrc"
    missing = []
    for f in sorted(csrc.glob("*.cu*")):
        lines = f.read_text().splitlines()
        for i, ln in enumerate(lines):
            if "<<<" in ln and not ln.strip().startswith("//"):
                if "launches" not in "\n".join(lines[i:i + 9]) and f.name != "noalloc.cu":
                    missing.append(f"{f.name}:{i + 1}")
    assert not missing, missing


def test_enum_values_match_the_python_constants():
    """Every OVS_* constant the header defines (enums and #defines) has the
    same value in oversetdevfort_b200._ffi when the binding names it."""
    txt = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "ovs.h").read_text(), flags=re.S)
    values = {}
    for body in re.findall(r"enum\s*\{(.*?)\}", txt, flags=re.S):
        nxt = 0
        for item in body.split(","):
            item = item.strip()
            if not item:
                continue
            if "=" in item:
                name, val = (t.strip() for t in item.split("=", 1))
                nxt = int(val, 0)
            else:
                name = item
            values[name] = nxt
            nxt += 1
    for name, val in re.findall(r"#define\s+(OVS_\w+)\s+(-?\d+)", txt):
        values[name] = int(val)
    assert len(values) > 40
    checked = 0
    for name, val in values.items():
        if hasattr(F, name):
            assert getattr(F, name) == val, (name, getattr(F, name), val)
            checked += 1
    assert checked >= 30, checked
    # the nodal fields: OVS_F_<NAME> is FIELD_ID["<name>"] in the binding
    fields = {n[6:].lower(): v for n, v in values.items() if n.startswith("OVS_F_") and n != "OVS_F_COUNT"}
    assert fields == F.FIELD_ID and values["OVS_F_COUNT"] == len(F.FIELDS)


def test_struct_layouts_match_the_header(tmp_path):
    """Every ctypes structure of the binding has the size and field offsets
    of its C struct in include/ovs.h, as gcc lays it out (the program that
    prints them is generated from the ctypes field lists)."""
    import shutil
    import subprocess
    import pytest
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    pairs = [(F.OvsDims, "ovs_dims"), (F.OvsParams, "ovs_params"), (F.OvsGmresInfo, "ovs_gmres_info"),
             (F.OvsSolveInfo, "ovs_solve_info"), (F.OvsNewtonOpts, "ovs_newton_opts"),
             (F.OvsNewtonInfo, "ovs_newton_info"), (F.OvsBcSpec, "ovs_bc_spec")]
    body = []
    for cls, cname in pairs:
        body.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, *_ in cls._fields_:
            body.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "ovs.h"\nint main(void) {\n' + "\n".join(body)
                   + "\n  return 0;\n}\n")
    exe = tmp_path / "layout"
    res = subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines()
    got = {tuple(ln.split()[:2]): int(ln.split()[2]) for ln in out}
    for cls, cname in pairs:
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for fname, *_ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def test_ctypes_signatures_match_the_prototypes(lib):
    """Each entry point's ctypes argtypes has the parameter count of its
    prototype in include/ovs.h, and its result is a C int (or a string for
    ovs_status_string)."""
    txt = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "ovs.h").read_text(), flags=re.S)
    protos = dict(re.findall(r"\b(?:int|const char\*)\s+(ovs_\w+)\s*\(([^)]*)\)\s*;", txt))
    assert len(protos) == len(F.EXPORTS)
    for name, params in protos.items():
        params = params.strip()
        n = 0 if params in ("", "void") else params.count(",") + 1
        fn = getattr(lib, name)
        assert len(fn.argtypes) == n, (name, len(fn.argtypes), n)
        want = ctypes.c_char_p if name == "ovs_status_string" else ctypes.c_int
        assert fn.restype is want, name

