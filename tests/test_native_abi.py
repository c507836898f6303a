"""The C ABI library loads and exports every function include/tccg_b200.h
declares; argument validation returns error codes without a GPU."""
import ctypes
import os
import re

from tccg_b200 import _native as N

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "tccg_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tccg_[a-z_0-9]+)\s*\(", src)))


def test_header_lists_the_boundary():
    fns = declared_functions()
    assert "tccg_plan_create" in fns and "tccg_plan_run" in fns and "tccg_group_run" in fns
    assert set(N.EXPORTED) == set(fns)


def test_library_exports_every_declared_symbol():
    L = N.lib()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_version_string():
    assert b"sm_100a" in N.lib().tccg_version()


def test_invalid_descriptor_is_an_error_code():
    L = N.lib()
    d = N.Desc()  # nm = nn = nk = 0
    h = ctypes.c_void_p()
    rc = L.tccg_plan_create(ctypes.byref(d), N.F32, N.PREC_FP32, None, ctypes.byref(h))
    assert rc == N.ERR_INVALID and not h.value
    assert b"mode counts" in L.tccg_last_error()


def test_bad_precision_dtype_pairs():
    L = N.lib()
    d = N.Desc()
    d.nm = d.nn = d.nk = 1
    d.m_ext[0] = d.n_ext[0] = d.k_ext[0] = 4
    h = ctypes.c_void_p()
    assert L.tccg_plan_create(ctypes.byref(d), N.F64, N.PREC_FP32, None, ctypes.byref(h)) == N.ERR_UNSUPPORTED
    assert L.tccg_plan_create(ctypes.byref(d), N.BF16, N.PREC_BF16X3, None, ctypes.byref(h)) == N.ERR_UNSUPPORTED
    assert L.tccg_plan_create(ctypes.byref(d), 7, N.PREC_FP32, None, ctypes.byref(h)) == N.ERR_INVALID


def test_null_arguments():
    L = N.lib()
    assert L.tccg_plan_run(None, None, None, None, 1.0, 0.0, None, 0, None) == N.ERR_INVALID
    assert L.tccg_plan_workspace(None, None) == N.ERR_INVALID
    assert L.tccg_group_create(None, 0, None) == N.ERR_INVALID
    assert L.tccg_group_run(None, None) == N.ERR_INVALID
    perm = (ctypes.c_int32 * 2)(0, 0)  # not a permutation
    size = (ctypes.c_int64 * 2)(2, 2)
    assert L.tccg_transpose(N.F32, 2, perm, size, None, None, 1.0, ctypes.c_void_p(8), 0.0,
                            ctypes.c_void_p(8), None) == N.ERR_INVALID


def test_tuning_struct_matches_the_header():
    """The ctypes mirror of tccg_tuning has the header's fields, in order,
    and its size (every field an int32_t)."""
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct tccg_tuning \{(.*?)\} tccg_tuning;", src, re.S).group(1)
    fields = re.findall(r"int32_t\s+([a-z_0-9]+)\s*;", body)
    assert len(fields) == len(re.findall(r";", body)), "tccg_tuning holds int32_t fields only"
    assert [f[0] for f in N.Tuning._fields_] == fields
    assert ctypes.sizeof(N.Tuning) == 4 * len(fields)


def test_extent_products_cannot_wrap():
    """Extents whose product passes 2^63 (or wraps to a small number) are
    rejected before any table is built: the running product is checked
    before each multiplication."""
    L = N.lib()
    h = ctypes.c_void_p()
    for exts in ([1 << 32, 1 << 32], [1 << 31, 2], [3, 1 << 30]):
        d = N.Desc()
        d.nm, d.nn, d.nk = len(exts), 1, 1
        for i, e in enumerate(exts):
            d.m_ext[i] = e
        d.n_ext[0] = d.k_ext[0] = 4
        rc = L.tccg_plan_create(ctypes.byref(d), N.F32, N.PREC_FP32, None, ctypes.byref(h))
        assert rc == N.ERR_UNSUPPORTED and not h.value, exts
        assert b"2^31" in L.tccg_last_error()
        rc = L.tccg_gett_bf16x3_noalloc(ctypes.byref(d), ctypes.c_void_p(16), ctypes.c_void_p(16),
                                        ctypes.c_void_p(16), 1.0, 0.0, None)
        assert rc == N.ERR_UNSUPPORTED, exts


def test_debug_trigger_validates_its_arguments():
    L = N.lib()
    assert L.tccg_debug_inject_timeout(-1, 100) == N.ERR_INVALID
    assert L.tccg_debug_inject_timeout(0, 0) == N.ERR_INVALID
    assert L.tccg_debug_inject_timeout(0, 5000) == N.ERR_INVALID
    assert L.tccg_gett_bf16x3_noalloc_status(None) == N.ERR_INVALID
