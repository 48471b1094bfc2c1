"""The Swift system-library target (k-wave-swift_b200/swift/) against the C ABI it binds.

Swift is not installed here, so the adapter cannot be compiled; these checks pin what a compile
would: every kw_* / KW_* name the Swift source uses is declared in include/kwave_cuda.h (and, when
the library is built, every function is exported by it), every descriptor field it sets exists
in that struct, and the module map links the library this repository builds.
"""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SWIFT = os.path.join(ROOT, "k-wave-swift_b200", "swift", "Sources")
ADAPTER = os.path.join(SWIFT, "KWave", "Solver", "KSpaceFirstOrderCUDA.swift")
HEADER = os.path.join(ROOT, "include", "kwave_cuda.h")
LIB = os.path.join(ROOT, "k-wave-swift_b200", "_build", "libkwave_cuda.so")


def _strip_comments(src: str) -> str:
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def _header():
    return _strip_comments(open(HEADER).read())


def _adapter():
    return _strip_comments(open(ADAPTER).read())


def _struct_fields(header: str, name: str) -> set[str]:
    m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), header, flags=re.S)
    assert m, name
    fields = set()
    for decl in m.group(1).split(";"):
        decl = decl.strip()
        if not decl:
            continue
        # "int nx, ny, nz" / "const float* data" / "kw_signal ux, uy, uz" / "void* user"
        decl = re.sub(r"\(\*(\w+)\)\(.*", r"\1", decl)   # function pointer typedef'd fields are plain here
        names = decl.split(",")
        first = names[0].split()
        fields.add(first[-1].lstrip("*"))
        fields.update(n.strip().lstrip("*") for n in names[1:])
    return fields


def test_adapter_uses_only_declared_names():
    h, s = _header(), _adapter()
    declared = set(re.findall(r"\b(kw_\w+|KW_\w+)\b", h))
    used = set(re.findall(r"\b(kw_\w+|KW_\w+)\b", s))
    assert used, "the adapter binds no ABI names"
    assert used <= declared, sorted(used - declared)


def test_adapter_functions_are_exported():
    if not os.path.exists(LIB):
        pytest.skip("library not built")
    h, s = _header(), _adapter()
    funcs = set(re.findall(r"KW_API\s+[\w\s\*]+?\b(kw_\w+)\s*\(", h))
    called = set(re.findall(r"\b(kw_\w+)\s*\(", s)) - {"kw_array", "kw_signal", "kw_sim_desc", "kw_adjoint_desc",
                                                      "kw_callbacks"}
    assert called <= funcs, sorted(called - funcs)
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\b(kw_\w+)\b", out))
    assert called <= exported, sorted(called - exported)


def test_adapter_descriptor_fields_exist():
    h, s = _header(), _adapter()
    for var, struct in (("d", "kw_sim_desc"), ("a", "kw_adjoint_desc"), ("cb", "kw_callbacks")):
        fields = _struct_fields(h, struct)
        used = set(re.findall(r"\b%s\.(\w+)\s*=" % var, s))
        assert used, var
        assert used <= fields, (struct, sorted(used - fields))


def test_module_map_links_the_built_library():
    mm = open(os.path.join(SWIFT, "CKWaveCUDA", "module.modulemap")).read()
    assert re.search(r'link\s+"kwave_cuda"', mm)
    assert re.search(r'header\s+"shim.h"', mm)
    shim = open(os.path.join(SWIFT, "CKWaveCUDA", "shim.h")).read()
    assert '#include "kwave_cuda.h"' in shim
