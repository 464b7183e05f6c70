"""The C-ABI library loads and exports every symbol its headers declare.

No compute call here (no GPU needed): the library is loaded with ctypes and
every function declared in include/*.h must resolve.
"""
import ctypes
import glob
import os
import re

import pytest

import spc5_b200
from spc5_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(B.LIB):
        B.build()
    return ctypes.CDLL(B.LIB)


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        text = re.sub(r"#define[^\n]*", "", text)
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name in ("if", "sizeof", "return", "defined"):
                continue
            pre = text[: m.start()].rstrip()
            # a declaration: the identifier follows a type (not an operator or '(')
            if pre and pre[-1] not in "(,=+-*/&|!<>?:" or pre.endswith("*"):
                names.add(name)
    return sorted(names)


def test_header_declares_dropins():
    names = declared_functions()
    for r in (1, 2, 4, 8):
        for t in ("double", "float"):
            assert f"core_SPC5_{r}rVc_Spmv_{t}" in names


def test_every_declared_symbol_is_exported(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"missing exports: {missing}"


def test_python_symbol_list_matches_header():
    assert set(spc5_b200.EXPORTED_SYMBOLS) == set(declared_functions())


def test_status_strings(lib):
    lib.spc5cuda_status_string.restype = ctypes.c_char_p
    assert lib.spc5cuda_status_string(0) == b"ok"
    assert b"format" in lib.spc5cuda_status_string(4)


def test_library_is_sm100a(lib):
    # the fatbin of every object is built for sm_100a only
    flags = open(B.__file__).read()
    assert "arch=compute_100a,code=sm_100a" in flags
