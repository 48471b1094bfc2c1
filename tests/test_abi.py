"""CPU tests of the C ABI boundary: the library loads, exports every symbol the header declares,
and the ctypes descriptor layout matches the C compiler's layout of include/kwave_cuda.h."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from kwave import abi
from kwave.runtime import LIB_PATH

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "kwave_cuda.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"^\s*(?:KW_API\s+)?(?:const\s+)?\w+[\s\*]+(kw_\w+)\s*\(", txt, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB_PATH):
        import importlib.util
        spec = importlib.util.spec_from_file_location("kwbuild", os.path.join(ROOT, "k-wave-swift_b200", "build.py"))
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        m.build()
    return C.CDLL(LIB_PATH)


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), f"missing export {n}"
    assert set(names) == set(abi.SIGNATURES), set(names) ^ set(abi.SIGNATURES)


def test_only_abi_symbols_exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    kw = {s for s in exported if s.startswith("kw_")}
    assert kw == set(declared_functions())


def test_descriptor_layout_matches_c(lib):
    fields = [f for f, _ in abi.kw_sim_desc._fields_]
    src = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void){",
           'printf("%zu\\n", sizeof(kw_sim_desc));']
    for f in fields:
        src.append(f'printf("%zu\\n", offsetof(kw_sim_desc, {f}));')
    src.append('printf("%zu %zu\\n", sizeof(kw_callbacks), sizeof(kw_array)); return 0; }')
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write("\n".join(src))
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", c, "-o", exe], check=True)
        vals = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert int(vals[0]) == C.sizeof(abi.kw_sim_desc)
    for i, f in enumerate(fields):
        assert int(vals[1 + i]) == getattr(abi.kw_sim_desc, f).offset, f
    assert int(vals[-2]) == C.sizeof(abi.kw_callbacks)
    assert int(vals[-1]) == C.sizeof(abi.kw_array)


def test_adjoint_descriptor_layout_matches_c(lib):
    fields = [f for f, _ in abi.kw_adjoint_desc._fields_]
    src = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void){",
           'printf("%zu\\n", sizeof(kw_adjoint_desc));']
    for f in fields:
        src.append(f'printf("%zu\\n", offsetof(kw_adjoint_desc, {f}));')
    src.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write("\n".join(src))
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", c, "-o", exe], check=True)
        vals = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert int(vals[0]) == C.sizeof(abi.kw_adjoint_desc)
    for i, f in enumerate(fields):
        assert int(vals[1 + i]) == getattr(abi.kw_adjoint_desc, f).offset, f
    abi.bind(lib)
    a = abi.kw_adjoint_desc()
    lib.kw_adjoint_desc_init(C.byref(a))
    assert a.abi_version == abi.KW_ABI_VERSION and a.policy == abi.KW_CHECKPOINT_SQRT


def test_desc_init_defaults(lib):
    abi.bind(lib)
    d = abi.kw_sim_desc()
    lib.kw_sim_desc_init(C.byref(d))
    assert d.abi_version == abi.KW_ABI_VERSION and d.pml_size == 20 and d.pml_alpha == 2.0
    assert d.smooth_p0 == 1 and d.p_mode == 1 and d.u_mode == 1 and d.record == 1
    assert lib.kw_abi_version() == abi.KW_ABI_VERSION
    assert b"sm_100a" in lib.kw_version()


def test_context_create_fails_cleanly_without_gpu(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    abi.bind(lib)
    h = C.c_void_p()
    st = lib.kw_context_create(0, C.byref(h))
    assert st == abi.KW_ERR_CUDA and not h
    assert lib.kw_last_error_message(None)
