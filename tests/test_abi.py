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


def test_psr_partition_rule_and_sizes(lib):
    # sinvb_psr_partitions: about sqrt(n/2), 3 <= P <= 32, n >= 3P (psr_utils.py:55-58)
    assert lib.sinvb_psr_partitions(64, 0) == 6
    assert lib.sinvb_psr_partitions(9, 0) == 3
    assert lib.sinvb_psr_partitions(2000, 0) == 32
    assert lib.sinvb_psr_partitions(8, 0) == -1
    assert lib.sinvb_psr_partitions(12, 4) == 4
    assert lib.sinvb_psr_partitions(12, 5) == -1 and lib.sinvb_psr_partitions(12, 2) == -1
    whole = lib.sinvb_psr_workspace_size(64, 256, 6, _lib.C128, 0)
    parts = [lib.sinvb_psr_part_workspace_size(64, 256, 6, k, _lib.C128) for k in range(6)]
    assert whole % 256 == 0 and all(p % 256 == 0 and p > 0 for p in parts)
    assert max(parts) < whole / 4            # a rank holds only its partition's rows
    assert parts[0] > parts[1] == parts[5]   # the first partition takes the remainder rows
    assert lib.sinvb_psr_workspace_size(64, 256, 6, _lib.C128, 1) == 0   # flags must be 0
    assert lib.sinvb_psr_part_workspace_size(64, 256, 6, 6, _lib.C128) == 0
    assert lib.sinvb_psr_workspace_size(64, 256, 6, _lib.F64, 0) < whole


def test_psr_and_bcr_batched_host_checks(lib):
    buf = (ctypes.c_char * 4096)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    null = None
    assert lib.sinvb_psr_z(null, p, p, 12, 4, 3, 0, p, p, p, p, 4096, null) == _lib.EINVAL
    assert lib.sinvb_psr_z(p, p, p, 12, 4, 5, 0, p, p, p, p, 4096, null) == _lib.EINVAL    # 12 < 3 * 5
    assert lib.sinvb_psr_z(p, p, p, 12, 4, 3, 1, p, p, p, p, 4096, null) == _lib.EINVAL    # flags
    assert lib.sinvb_psr_part_z(p, p, p, 12, 4, 3, 0, 2, p, p, p, p, p, 4096, null) == _lib.EINVAL  # stage
    assert lib.sinvb_psr_part_z(p, p, p, 12, 4, 3, 3, 0, p, p, p, p, p, 4096, null) == _lib.EINVAL  # part
    assert lib.sinvb_psr_part_z(p, p, p, 12, 4, 3, 0, 0, null, p, p, p, p, 4096, null) == _lib.EINVAL
    descs = (_lib.BatchDesc * 2)()
    descs[0] = _lib.BatchDesc(None, None, None, None, None, None, 3, 8)
    descs[1] = _lib.BatchDesc(None, None, None, None, None, None, 0, 8)
    cd = ctypes.cast(descs, ctypes.c_void_p)
    assert lib.sinvb_bcr_batched_workspace_size(cd, 2, _lib.C128, 0) == 0     # n < 1
    assert lib.sinvb_bcr_batched_workspace_size(cd, 1, _lib.C128, 0) > 0
    assert lib.sinvb_bcr_batched_workspace_size(cd, 0, _lib.C128, 0) == 256  # the header alone
    big = (ctypes.c_char * 8192)()
    aligned = ctypes.c_void_p((ctypes.addressof(big) + 255) & ~255)   # workspaces are 256-byte aligned
    assert lib.sinvb_bcr_batched_z(cd, 1, 0, aligned, 4096, null, null) == _lib.EINVAL   # null block pointers
    assert lib.sinvb_bcr_batched_z(cd, -1, 0, aligned, 4096, null, null) == _lib.EINVAL
    assert lib.sinvb_bcr_batched_z(cd, 1, 0, p if ctypes.addressof(buf) % 256 else None, 4096, null,
                                   null) in (_lib.EINVAL, _lib.EWORKSPACE)


def test_lesser_batched_host_checks(lib):
    """Argument checks of sinvb_rgf_lesser_batched_z run before any device
    call: distinct 16-byte aligned host ranges stand in for the blocks."""
    big = (ctypes.c_char * (1 << 16))()
    base = (ctypes.addressof(big) + 255) & ~255
    ws = ctypes.c_void_p(base)
    n, b = 3, 4
    blk = b * b * 16
    sizes = [n, n - 1, n - 1, n, n, n - 1, n - 1, n, n - 1]   # diag, upper, lower, sigma, G*, GL*
    offs, o = [], 4096
    for m in sizes:
        offs.append(base + o)
        o += m * blk
    names = ["diag", "upper", "lower", "sigma_lesser", "G_diag", "G_upper", "G_lower", "GL_diag", "GL_upper"]

    def desc(**change):
        f = dict(zip(names, offs))
        f.update(change)
        d = (_lib.LesserDesc * 1)()
        d[0] = _lib.LesserDesc(*(f[k] for k in names), n, b)
        return ctypes.cast(d, ctypes.c_void_p), d

    good, keep = desc()
    assert lib.sinvb_rgf_lesser_batched_z(good, 0, 0, ws, 4096, None, None) == _lib.EINVAL
    assert lib.sinvb_rgf_lesser_batched_z(None, 1, 0, ws, 4096, None, None) == _lib.EINVAL
    assert lib.sinvb_rgf_lesser_batched_z(good, 1, _lib.FORCE_GRID, ws, 4096, None, None) == _lib.EINVAL
    assert lib.sinvb_rgf_lesser_batched_z(good, 1, 0, ctypes.c_void_p(base + 16), 4096, None,
                                          None) == _lib.EWORKSPACE
    for change in ({"sigma_lesser": None}, {"GL_upper": None}, {"diag": offs[0] + 8},
                   {"G_diag": offs[0]},              # an output over an input
                   {"GL_upper": offs[5]}):           # two outputs over each other
        bad, keep2 = desc(**change)
        assert lib.sinvb_rgf_lesser_batched_z(bad, 1, 0, ws, 4096, None, None) == _lib.EINVAL, change
    # a valid descriptor: no GPU here (EUNSUPPORTED / ECUDA), or on a GPU a workspace too small
    assert lib.sinvb_rgf_lesser_batched_z(good, 1, 0, ws, 256, None, None) in (
        _lib.EUNSUPPORTED, _lib.ECUDA, _lib.EWORKSPACE)
    assert lib.sinvb_rgf_lesser_batched_workspace_size(good, 0, 0) == 0
