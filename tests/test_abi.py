"""The C-ABI library loads and exports every symbol include/sinvb.h declares.

No compute calls: only entry points that fail host-side argument checks
before touching a device are called here.
"""

import ctypes
import os
import re

import pytest

from sinv_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(sinvb_\w+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from sinv_b200 import build
    build.build()
    return _lib.load()


def test_header_declares_entry_points():
    names = _declared_symbols()
    assert "sinvb_rgf_z" in names and "sinvb_workspace_status" in names


def test_every_declared_symbol_is_exported(lib):
    for name in _declared_symbols():
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, "python binding missing for %s" % name


def test_version_and_status_strings(lib):
    assert lib.sinvb_version() >= 100
    for code in (_lib.OK, _lib.EINVAL, _lib.EWORKSPACE, _lib.EUNSUPPORTED, _lib.STATUS_PIVOT,
                 _lib.STATUS_TIMEOUT):
        assert lib.sinvb_status_string(code)


def test_workspace_size_grows_with_problem(lib):
    small = lib.sinvb_rgf_workspace_size(10, 32, _lib.C128, _lib.SAVE_OFFDIAG)
    nosave = lib.sinvb_rgf_workspace_size(10, 32, _lib.C128, 0)
    big = lib.sinvb_rgf_workspace_size(64, 256, _lib.C128, _lib.SAVE_OFFDIAG)
    single = lib.sinvb_rgf_workspace_size(10, 32, _lib.C64, _lib.SAVE_OFFDIAG)
    assert 256 <= small < big
    assert nosave > small          # X / P blocks move into the workspace
    assert single > small          # widened copies of inputs and outputs
    assert small % 256 == 0
    assert lib.sinvb_rgf_workspace_size(0, 32, _lib.C128, 0) == 0
    assert lib.sinvb_rgf_workspace_size(4, 32, 9, 0) == 0


def test_host_side_argument_checks(lib):
    buf = (ctypes.c_char * 4096)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    null = None
    # null inputs / bad sizes are rejected before any device work
    assert lib.sinvb_rgf_z(null, null, null, 4, 8, 0, p, null, null, p, 4096, null) == _lib.EINVAL
    assert lib.sinvb_rgf_z(p, p, p, 0, 8, 0, p, null, null, p, 4096, null) == _lib.EINVAL
    assert lib.sinvb_rgf_z(p, p, p, 4, 0, 0, p, null, null, p, 4096, null) == _lib.EINVAL
    # off-diagonal outputs required when SAVE_OFFDIAG is set
    assert lib.sinvb_rgf_z(p, p, p, 4, 8, _lib.SAVE_OFFDIAG, p, null, null, p, 4096, null) == _lib.EINVAL
    # conflicting team flags
    assert lib.sinvb_rgf_z(p, p, p, 1, 8, _lib.FORCE_GRID | _lib.FORCE_CTA, p, null, null, p, 4096,
                           null) == _lib.EINVAL
    # workspace too small
    assert lib.sinvb_rgf_d(p, p, p, 4, 8, 0, p, null, null, p, 16, null) in (_lib.EWORKSPACE, _lib.EINVAL)
    assert lib.sinvb_workspace_status(null, null, None) == _lib.EINVAL


def test_product_path_has_no_cpu_fallback(monkeypatch, tmp_path):
    """Without the shared object the API raises instead of computing elsewhere."""
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(_lib.SinvbUnavailable):
        _lib.load(str(tmp_path / "missing.so"))
