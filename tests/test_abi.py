"""The C ABI library loads, exports every symbol declared in include/*.h, and
reports errors as status codes (no GPU needed)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import terra_b200 as T

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(tn_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(T.LIB_PATH)
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert missing == []


def test_version_and_error_strings():
    L = T.load()
    assert b"sm_100a" in L.tn_version()
    # invalid level -> TN_ERR_ARG with a message, no crash
    coords = np.zeros((10, 3, 3, 3))
    rc = L.tn_mesh_generate_host(-1, 1, 0.55, 1.0, coords.ctypes.data, None, None, None, None)
    assert rc == -1
    assert L.tn_last_error().decode() != ""
    rc = L.tn_mesh_generate_host(2, 2, 1.0, 0.5, None, None, None, None, None)
    assert rc == -1 and b"r_min" in L.tn_last_error()


def test_null_arguments_rejected():
    L = T.load()
    assert L.tn_shell_create(2, 2, 1, 0.55, 1.0, None) == -1
    assert L.tn_operator_apply(None, None, None, None) == -1
    assert L.tn_vec_dot(None, 0, 0, 1, None, None, None, None) == -1


def test_vec_alloc_and_free_argument_errors():
    """tn_vec_alloc rejects a NULL shell or output array before touching the device; tn_vec_free skips a NULL
    array and NULL entries (nothing to release)."""
    L = T.load()
    out = (ctypes.c_void_p * 4)()
    assert L.tn_vec_alloc(None, 0, T.TN_F64, 3, out) == -1
    assert b"NULL" in L.tn_last_error()
    assert L.tn_vec_alloc(None, 0, T.TN_F64, 3, None) == -1
    L.tn_vec_free(3, None)
    L.tn_vec_free(4, (ctypes.c_void_p * 4)())


def test_shell_create_without_device_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    L = T.load()
    h = ctypes.c_void_p()
    rc = L.tn_shell_create(2, 2, 1, 0.55, 1.0, ctypes.byref(h))
    assert rc in (-2, -3)  # CUDA error / allocation failure, reported
    assert L.tn_last_error().decode() != ""
