"""CPU: the C-ABI shared library loads, exports every function that
include/*.h declares, and rejects invalid descriptors exactly where the
reference does (api/validate_problem.h:346-414) -- validation runs before any
device work, so these checks need no GPU. No compute call is made here."""
import ctypes as C
import glob
import os
import re

import pytest

import aoclfftz_b200
from aoclfftz_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        txt = re.sub(r"#define[^\n]*(\\\n[^\n]*)*", "", txt)
        for m in re.finditer(r"\b((?:aoclfftz|fftwf?)_\w+)\s*\(", txt):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    return aoclfftz_b200.load()


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version(lib):
    assert lib.aoclfftz_version().startswith(b"AOCL-FFTZ 6.0.0")


def test_null_handles(lib):
    assert lib.aoclfftz_execute(None) == abi.AOCLFFTZ_EXECUTION_FAILURE
    assert lib.aoclfftz_execute_io(None, None, None) == abi.AOCLFFTZ_EXECUTION_FAILURE
    lib.aoclfftz_destroy(None)
    assert lib.aoclfftz_gpu_num_launches(None) == -1


def _setup(lib, dims, vecs, in_=1, out=2, **kw):
    d, keep = abi.make_desc(in_, out, dims, vecs, **kw)
    return abi.setup(lib, d, "f32"), lib.aoclfftz_gpu_last_error().decode()


@pytest.mark.parametrize("dims,vecs,kw,msg", [
    ([(0, 1, 1)], [(1, 1, 1)], {}, "positive"),
    ([(8, 0, 1)], [(1, 8, 8)], {}, "positive"),
    ([(8, 1, -1)], [(1, 8, 8)], {}, "positive"),
    ([(8, 1, 1)], [(-1, 8, 8)], {}, "vector"),
    ([(8, 1, 1)], [(2, 0, 8)], {}, "vector"),
    ([(8, 1, 1)], [(1, 8, 8)], {"fft_type": 2}, "fft_type"),
    ([(8, 1, 1)], [(1, 8, 8)], {"direction": 2}, "fft_direction"),
    ([(8, 1, 1)], [(1, 8, 8)], {"placement": 2}, "fft_placement"),
])
def test_validation_rejects(lib, dims, vecs, kw, msg):
    h, err = _setup(lib, dims, vecs, **kw)
    assert not h
    assert msg in err


def test_placement_rules(lib):
    # out-of-place with in == out, in-place with in != out
    h, err = _setup(lib, [(8, 1, 1)], [(1, 8, 8)], in_=5, out=5, placement=1)
    assert not h and "cannot be the same" in err
    h, err = _setup(lib, [(8, 1, 1)], [(1, 8, 8)], in_=5, out=6, placement=0)
    assert not h and "must be the same" in err
    # in-place c2c needs equal strides
    h, err = _setup(lib, [(8, 1, 2)], [(1, 8, 8)], in_=5, out=5, placement=0)
    assert not h and "in_stride != out_stride" in err
    # in-place r2c: outer strides must differ by 2 (docs/rst/data_layout_conventions.rst)
    h, err = _setup(lib, [(8, 1, 1), (4, 10, 10)], [(1, 40, 20)], in_=5, out=5, placement=0, fft_type=1)
    assert not h and "factor of 2" in err


def test_storage_order_and_transpose_rejected(lib):
    d, keep = abi.make_desc(1, 2, [(8, 1, 1)], [(1, 8, 8)])
    d.flags.storage_order = 1
    assert not abi.setup(lib, d, "f32")
    d.flags.storage_order = 0
    d.flags.transpose_mode = 1
    assert not abi.setup(lib, d, "f64")
    d.flags.transpose_mode = 0
    d.vec_rank = 0
    assert not abi.setup(lib, d, "f32")
    d.vec_rank = 1
    d.dim_rank = 0
    assert not abi.setup(lib, d, "f32")


def test_abi_struct_layout():
    # the descriptor layout is the reference's (api/aoclfftz.h:174-311)
    assert C.sizeof(abi.Dim) == 12 and C.sizeof(abi.Dim64) == 24
    assert C.sizeof(abi.Flags) == 6
    assert abi.DescLP64.flags.offset == 40
    assert C.sizeof(abi.DescLP64) == 72
