"""Host-side checks that need no GPU: the C-ABI library loads and exports every
symbol the headers declare; the product's shape plan and wire helpers agree
with the oracle (and so with the reference's derivation)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b((?:ipr|gpu)_[a-z0-9_]+)\s*\(", txt)))


@pytest.mark.parametrize("header", ["ipr_b200.h", "ipr_b200_compat.h"])
def test_library_exports_every_declared_symbol(pkg, header):
    names = _declared(header)
    assert len(names) > 10
    for n in names:
        assert hasattr(pkg.lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", pkg._LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (\S+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing


@pytest.mark.parametrize("header", ["ipr_b200.h", "ipr_b200_compat.h"])
def test_debug_library_exports_the_same_symbols_and_release_checks_nothing(pkg, header):
    """the bounds-checked debug build exports every declared symbol too and says what it is;
    in the release library the debug entry points refuse and the report is empty (no GPU)"""
    dbg = os.path.join(os.path.dirname(pkg._LIB_PATH), "libipr_b200_dbg.so")
    assert os.path.exists(dbg), "run make -C inspire-rs_b200 debug"
    out = subprocess.run(["nm", "-D", "--defined-only", dbg], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (\S+)", out))
    missing = [n for n in _declared(header) if n not in exported]
    assert not missing, missing
    d = ctypes.CDLL(dbg)
    assert d.ipr_bounds_checked_build() == 1
    if not pkg.BOUNDS_CHECK:
        assert pkg.bounds_checked_build() is False
        assert pkg.bounds_report() == (0, "")
        assert pkg.debug_cut_fold_extent(2048) == -7  # IPR_E_STATE: not a bounds-checked build
        assert pkg.debug_check_extent(0, 16) == -7


@pytest.mark.gpu
def test_library_is_sm100a(pkg):
    """the runtime reports the library's kernels as built for compute capability 10.0"""
    v = ctypes.c_int(0)
    f = pkg.lib.ipr_device_binary_version
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    assert f(0, ctypes.byref(v)) == 0
    assert v.value == 100


SHAPES = [
    (10_000, 32, 1184, None, None),
    (1_000_000, 32, 1184, 2_097_152, 2048),
    (4_000_000, 32, 800, 8_388_608, 8192),
    (1_000_000, 32, 1184, 2_097_152, 8192),
    (2_000_000, 32, 1568, 4_194_304, 8192),
    (5_000_000, 32, 1184, 8_388_608, 65_536),
    (5_000_000, 32, 1184, None, None),
    (3000, 16, 16, None, None),
    (700, 32, 1184, None, None),
]


@pytest.mark.parametrize("shape", SHAPES)
def test_plan_matches_oracle(pkg, orc, shape):
    p = pkg.plan_from_shape(*shape)
    o = orc.plan_from_shape(*[s or 0 for s in shape])
    assert o is not None
    for k, v in o.items():
        assert getattr(p, k) == v, k


def test_plan_rejections(pkg):
    with pytest.raises(pkg.IprError) as e:
        pkg.plan_from_shape(1_000_000, 32, 1184, 262_144, 2048)  # buckets < records
    assert e.value.status == -1
    with pytest.raises(pkg.IprError):
        pkg.plan_from_shape(10, 3, 0)
    with pytest.raises(pkg.IprError):
        pkg.plan_from_shape(0, 32, 1184)


def test_query_bytes(pkg, orc):
    for rows in (2048, 8192, 65536):
        for nq in (0, 1, 2, 5):
            assert pkg.query_bytes(rows, nq) == orc.query_bytes(rows, nq)
    assert pkg.query_bytes(2048, 2) == 286_721


def test_serialize_query_roundtrip(pkg, orc):
    rows = 2048
    q = orc.synth_query(5, rows, 2)
    y, z, qrows, gsw = orc.parse_query(q, rows)
    payload = pkg.KeywordQueryPayload(
        y_body=y.reshape(3, 2048), z_body=z.reshape(3, 2048),
        queries=[(qrows[i], gsw[i]) for i in range(2)])
    assert pkg.serialize_keyword_query(payload) == q


def test_response_framing_roundtrip(pkg):
    body = [bytes(range(7)) * 3, b"xyz"]
    stash = [b"k" * 5]
    buf = len(body).to_bytes(4, "little")
    for b in body:
        buf += len(b).to_bytes(4, "little") + b
    buf += len(stash).to_bytes(4, "little") + len(stash[0]).to_bytes(4, "little") + stash[0]
    r = pkg.deserialize_keyword_response(buf)
    assert r.responses == body and r.stash_entries == stash


def test_server_create_without_gpu_fails_loudly(pkg):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except ImportError:
        pass
    plan = pkg.plan_from_shape(10_000, 32, 1184)
    with pytest.raises(pkg.IprError) as e:
        pkg.KeywordServer.synthetic(plan, seed=1)
    assert e.value.status in (-2, -3)


def test_error_string_reports_status(pkg):
    with pytest.raises(pkg.IprError) as e:
        pkg.plan_from_shape(1_000_000, 32, 1184, 262_144, 2048)
    assert "IPR_E_ARGS" in str(e.value) and "buckets" in str(e.value)


def test_library_has_no_unresolved_symbols():
    """every symbol the library needs comes from a versioned system library (a missing
    definition would only show when the library is loaded on the GPU box)"""
    import subprocess
    lib = os.path.join(ROOT, "inspire-rs_b200", "libipr_b200.so")
    out = subprocess.run(["nm", "-D", "--undefined-only", lib], capture_output=True, text=True, check=True).stdout
    missing = [ln.split()[-1] for ln in out.splitlines() if ln.split() and ln.split()[0] == "U" and "@" not in ln]
    assert missing == []
