"""The C ABI library loads and exports every function include/cp_prover.h declares."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_\s\*]*?\b(cp_[A-Za-z0-9_]+)\s*\(", text, re.M):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def libpath():
    from circlepacking_b200 import build

    return build.build()


def test_header_declares_functions():
    names = declared_functions()
    assert "cp_eval_boxes" in names and "cp_lattice_boxes" in names


def test_library_exports_all_declared(libpath):
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing


def test_library_loads_and_reports(libpath):
    import circlepacking_b200 as cp

    L = cp.lib()
    assert L.cp_family_dims(3) == 4 and L.cp_family_dims(1) == 3 and L.cp_family_dims(9) == -1
    assert L.cp_family_criteria(3) == 4
    assert L.cp_status_string(0) == b"ok"
    assert b"sm_100a" in L.cp_version()


def test_invalid_arguments_rejected_without_device(libpath):
    import circlepacking_b200 as cp

    L = cp.lib()
    # argument validation happens before any CUDA call
    assert L.cp_eval_boxes(7, 0, 0, None, None, 10, 10, None, None, None, None, None) == 1
    assert L.cp_eval_boxes(3, 5, 0, None, None, 10, 10, None, None, None, None, None) == 1
    assert L.cp_eval_boxes(3, 0, 0, None, None, 0, 0, None, None, None, None, None) == 0


def test_reference_prover_links_against_shim(libpath, tmp_path):
    """The reference's own prover.cpp links unchanged against the library (the
    C++ shim defines circlepacking::lane_packing::find_critical_intervals)."""
    ref = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref-dir"], capture_output=True,
                         text=True).stdout.strip()
    if not ref or not os.path.exists(os.path.join(ref, "prover.cpp")):
        pytest.skip("reference sources not present on this machine")
    out = tmp_path / "prover_b200"
    libdir = os.path.dirname(libpath)
    subprocess.run(["g++", "-std=c++17", f"-I{ref}/algcuda/cuda-cpp-wrapper/include", f"{ref}/prover.cpp",
                    f"-L{libdir}", "-lcp_b200", f"-Wl,-rpath,{libdir}", "-o", str(out)], check=True)
    assert out.exists()


def test_proof_defaults_without_device(libpath):
    """cp_proof_defaults needs no device: the seeds each family's proof uses."""
    import ctypes

    import circlepacking_b200 as cp

    L = cp.lib()
    L.cp_proof_defaults.argtypes = [ctypes.c_int, ctypes.POINTER(cp.ProofOpts)]
    o = cp.ProofOpts()
    assert L.cp_proof_defaults(9, ctypes.byref(o)) == 1  # CP_ERR_INVALID
    assert L.cp_proof_defaults(0, ctypes.byref(o)) == 0
    d = o.as_dict()
    assert d["slabs"] == 18 and d["geometric"] == 1 and d["seed_sizes"] == [1, 256, 256, 64]
    assert d["policy"] == 1 and d["engine"] == 1  # lambda-only split, graph engine
    # start: a radius lattice per slab; r1 the finest axis, growing toward lambda = 0.99
    sr = d["slab_radii"]
    assert all(0 < r[0] <= 256 and 0 < r[1] <= r[0] and r[2] >= 1 for r in sr[:18])
    assert sr[18:] == [[0, 0, 0]] * 14
    r1 = [r[0] for r in sr[:18]]
    assert r1 == sorted(r1)
    for f in (1, 3, 4, 5):
        assert L.cp_proof_defaults(f, ctypes.byref(o)) == 0
        assert o.slabs == 1 and o.seed_sizes[0] >= 32 and o.max_depth == 24
        assert all(list(r) == [0, 0, 0] for r in o.slab_radii)
    # start_end_3d: the start proof's geometric slabs, a radius lattice per slab
    assert L.cp_proof_defaults(2, ctypes.byref(o)) == 0
    assert o.slabs == 18 and o.geometric == 1 and o.seed_sizes[0] == 1
    assert all(r[0] > 0 and r[1] > 0 and r[2] > 0 for r in o.slab_radii[:18])
    L.cp_prove_family.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    assert L.cp_prove_family(None, None, None) == 1
