"""The C ABI library loads and exports every symbol the header declares (CPU only: no
kernel launches, only calls that fail argument checks before touching a device)."""
import ctypes
import os
import re

import pytest

from nngpr_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, 'include', 'nngp_b200.h')


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(nngp_[a-z0-9_]+)\s*\(', text)))


def test_header_and_binding_agree():
    assert set(header_functions()) == set(_lib.EXPORTED)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    for name in header_functions():
        assert hasattr(L, name), name


def test_version_and_status_strings():
    L = _lib.lib()
    assert L.nngp_abi_version() == 3
    assert L.nngp_status_string(0) == b'NNGP_OK'
    assert L.nngp_status_string(3) == b'NNGP_ERR_WORKSPACE'


def test_invalid_arguments_fail_before_any_launch():
    L = _lib.lib()
    st = L.nngp_knn_f32(None, 10, None, 10, 0, None, 0, 4, 0, 0, None, None, None, 0, None)
    assert st == 1 and b'd <= 0' in L.nngp_last_error()
    st = L.nngp_knn_f32(None, 10, None, 10, 300, None, 0, 4, 0, 0, None, None, None, 0, None)
    assert st == 2
    with pytest.raises(NotImplementedError):
        _lib.check(st, 'probe')
    k = _lib.NngpKernel()
    k.n_ls = 2
    st = L.nngp_loglik_f32(None, None, 10, 3, 1, None, 4, ctypes.byref(k), 0, 1e-6, None, None, None, 0, None)
    assert st == 1  # out is null


def test_workspace_sizes_are_host_only():
    L = _lib.lib()
    assert L.nngp_knn_workspace_size_f32(1000, 1000, 3, 32) >= 1000 * 4 * 4
    assert L.nngp_knn_workspace_size_f64(1000, 500, 3, 100) >= 500 * 100 * 12
    assert L.nngp_loglik_workspace_size(1000, 3, 1, 32, 3) > 0
