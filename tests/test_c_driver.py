"""The C ABI from plain C (tests/c/ovs_abi_driver.c, where the reference's
Fortran would call the library): include/ovs.h compiles as C99 and as C++
with every warning an error; the driver links libovs_b200.so and its
stateless and argument checks pass; the cavity mesh it builds for its GPU
mode is the Kuhn box of the Python mesh module, positively oriented, with
the closed-form pattern count that the oracle's genSparStruc gives (CPU)."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest
import torch

from oversetdevfort_b200 import build
from oversetdevfort_b200 import mesh as M

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "c" / "ovs_abi_driver.c"
WARN = ["-Wall", "-Wextra", "-Werror", "-pedantic"]


@pytest.fixture(scope="module")
def driver(tmp_path_factory, lib):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    exe = tmp_path_factory.mktemp("cdrv") / "ovs_abi_driver"
    libdir = build.LIB.parent
    cmd = ["gcc", "-std=c99", *WARN, "-O1", "-I", str(ROOT / "include"), str(SRC), "-o", str(exe),
           "-L", str(libdir), f"-l:{build.LIB.name}", f"-Wl,-rpath,{libdir}", "-lm"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


def test_header_compiles_as_c_and_cxx(tmp_path):
    if shutil.which("gcc") is None or shutil.which("g++") is None:
        pytest.skip("gcc/g++ not available")
    inc = ["-I", str(ROOT / "include")]
    unit = tmp_path / "unit.c"
    unit.write_text('#include "ovs.h"\nint main(void) { return OVS_OK; }\n')
    for comp, std in (("gcc", "-std=c99"), ("gcc", "-std=c11"), ("g++", "-std=c++11")):
        lang = ["-x", "c++"] if comp == "g++" else []
        res = subprocess.run([comp, std, *WARN, *inc, *lang, "-fsyntax-only", str(unit)],
                             capture_output=True, text=True)
        assert res.returncode == 0, f"{comp} {std}: {res.stderr}"


def test_abi_mode(driver):
    res = subprocess.run([str(driver), "abi"], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "abi checks: 0 failure(s)" in res.stdout
    assert ("device: none" in res.stdout) == (not torch.cuda.is_available())


def test_usage_errors(driver):
    assert subprocess.run([str(driver)], capture_output=True).returncode == 2
    assert subprocess.run([str(driver), "cavity", "0"], capture_output=True).returncode == 2
    assert subprocess.run([str(driver), "mesh", "0", "x"], capture_output=True).returncode == 2


@pytest.mark.skipif(torch.cuda.is_available(), reason="a device is present: the cavity mode would run")
def test_cavity_mode_reports_no_device(driver):
    res = subprocess.run([str(driver), "cavity", "2"], capture_output=True, text=True, timeout=120)
    assert res.returncode == 77 and "no CUDA device" in res.stdout


def _read_mesh(driver, n, tmp_path):
    path = tmp_path / f"mesh{n}.bin"
    res = subprocess.run([str(driver), "mesh", str(n), str(path)], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stderr
    fields = dict(kv.split("=") for kv in res.stdout.split()[1:])
    N, E = int(fields["N"]), int(fields["E"])
    raw = path.read_bytes()
    xg = np.frombuffer(raw[:24 * N], dtype=np.float64).reshape(3, N).T
    ien = np.frombuffer(raw[24 * N:], dtype=np.int32).reshape(4, E).T
    return xg, ien, int(fields["nnz"])


@pytest.mark.parametrize("n", [1, 2, 5])
def test_cavity_mesh_is_the_kuhn_box(driver, oracle, tmp_path, n):
    xg, ien, nnz = _read_mesh(driver, n, tmp_path)
    ref = M.box_tet(n, n, n)
    np.testing.assert_array_equal(xg, ref.xg)
    assert ien.shape == ref.ien.shape and ien.min() == 1 and ien.max() == ref.nnode
    assert sorted(map(tuple, np.sort(ien, axis=1))) == sorted(map(tuple, np.sort(ref.ien, axis=1)))
    x = xg[ien - 1]                                   # (E, 4, 3)
    det = np.linalg.det(np.stack([x[:, 0] - x[:, 3], x[:, 1] - x[:, 3], x[:, 2] - x[:, 3]], axis=1))
    assert np.all(det > 0.0)
    col, row = oracle.gen_spar_struc(np.asfortranarray(ien), xg.shape[0])
    assert len(row) == nnz


def test_closed_form_pattern_count_of_config1(driver, tmp_path):
    # 16^3 x 6 tets: 66,961 entries (4,913 nodes + both directions of 31,024 edges)
    _, _, nnz = _read_mesh(driver, 16, tmp_path)
    assert nnz == 66961
