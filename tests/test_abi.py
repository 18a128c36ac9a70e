"""The C-ABI library loads, exports every declared symbol, and validates on the host.

No compute call is made here: every call below fails argument validation
before anything is launched, so these run without a GPU.
"""

from __future__ import annotations

import ctypes
import pathlib
import re

import numpy as np
import pytest

from aprict_b200 import _lib
from aprict_b200 import _structs as S

HEADER = pathlib.Path(__file__).resolve().parents[1] / "include" / "aprict_b200.h"


def declared_symbols() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"APRICT_API[^;(]*?\b(aprict_b200_\w+)\s*\(", text)))


def test_header_declares_entry_points() -> None:
    syms = declared_symbols()
    assert "aprict_b200_project_siddon" in syms
    assert "aprict_b200_backproject" in syms
    assert len(syms) >= 10


def test_library_exports_every_declared_symbol() -> None:
    lib = _lib.lib()
    for name in declared_symbols():
        assert hasattr(lib, name), f"{name} declared in include/aprict_b200.h but not exported"


def test_binding_covers_every_declared_symbol() -> None:
    assert set(declared_symbols()) <= set(_lib.SIGNATURES), set(declared_symbols()) - set(_lib.SIGNATURES)


def test_struct_layouts_match_c() -> None:
    lib = _lib.lib()
    for name, dt in S.ABI_STRUCTS.items():
        assert lib.aprict_b200_struct_size(name.encode()) == dt.itemsize, name
    assert lib.aprict_b200_struct_size(b"no_such_struct") == 0


def test_status_strings() -> None:
    lib = _lib.lib()
    assert lib.aprict_b200_status_string(0) == b"ok"
    assert lib.aprict_b200_status_string(1) == b"invalid argument"
    assert lib.aprict_b200_status_string(999) == b"unknown status"
    assert lib.aprict_b200_version().decode().count(".") == 2


def _fake(n: int = 1 << 20) -> int:
    """A host address standing in for a device pointer; never dereferenced because validation fails first."""
    return 0x10000000


@pytest.mark.parametrize(
    ("field", "value", "expect"),
    [("ssu", 0, ValueError), ("ssv", 100, ValueError), ("multiply_before_adding", np.inf, ValueError)],
)
def test_project_rejects_bad_config(field: str, value: float, expect: type) -> None:
    lib = _lib.lib()
    cfg = np.array((1.0, 1.0, 1, 1), dtype=S.project_config)
    cfg[field] = value
    pd = _lib.proj_desc((2, 4, 4), (16, 4, 1))
    vd = _lib.vol_desc((4, 4, 4), "C", 1.0, np.zeros(3))
    rc = lib.aprict_b200_project_siddon(_fake(), _lib.ptr(pd), _fake(), None, _lib.ptr(vd), _fake(), _lib.ptr(cfg), None, None)
    with pytest.raises(expect):
        _lib.check(rc, "project")


def test_project_rejects_bad_volume() -> None:
    lib = _lib.lib()
    cfg = np.array((1.0, 1.0, 1, 1), dtype=S.project_config)
    pd = _lib.proj_desc((2, 4, 4), (16, 4, 1))
    for vd in (
        _lib.vol_desc((0, 4, 4), "C", 1.0, np.zeros(3)),
        _lib.vol_desc((4, 4, 4), "C", -1.0, np.zeros(3)),
        _lib.vol_desc((4, 4, 4), "C", 1.0, np.array([np.nan, 0, 0])),
    ):
        rc = lib.aprict_b200_project_siddon(_fake(), _lib.ptr(pd), _fake(), None, _lib.ptr(vd), _fake(), _lib.ptr(cfg), None, None)
        assert rc == 1
    # unaligned volume pointer
    vd = _lib.vol_desc((4, 4, 4), "C", 1.0, np.zeros(3))
    rc = lib.aprict_b200_project_siddon(_fake(), _lib.ptr(pd), _fake(), None, _lib.ptr(vd), _fake() + 2, _lib.ptr(cfg), None, None)
    assert rc == 1
    assert b"aligned" in lib.aprict_b200_last_error()


def test_project_empty_is_a_no_op() -> None:
    lib = _lib.lib()
    cfg = np.array((1.0, 1.0, 1, 1), dtype=S.project_config)
    vd = _lib.vol_desc((4, 4, 4), "C", 1.0, np.zeros(3))
    pd = _lib.proj_desc((0, 4, 4), (16, 4, 1))
    assert lib.aprict_b200_project_siddon(None, _lib.ptr(pd), None, None, _lib.ptr(vd), _fake(), _lib.ptr(cfg), None, None) == 0


def test_backproject_validation() -> None:
    lib = _lib.lib()
    from aprict_b200.cb import flatpanel as fp

    pd = _lib.proj_desc((2, 4, 4), (16, 4, 1))
    vd = _lib.vol_desc((4, 4, 4), "C", 1.0, np.zeros(3))
    # multiplier flag without a multiplier
    cfg = fp.ConfigBackproject(apply_summand_multiplier=True).contents
    rc = lib.aprict_b200_backproject(_fake(), _lib.ptr(pd), _fake(), _lib.ptr(vd), _fake(), None, _lib.ptr(cfg), None, None)
    assert rc == 1
    # weighting preset 7 (GBC) has its own entry point
    cfg = fp.ConfigBackproject(backproj_weighting_preset=7).contents
    rc = lib.aprict_b200_backproject(_fake(), _lib.ptr(pd), _fake(), _lib.ptr(vd), _fake(), None, _lib.ptr(cfg), None, None)
    assert rc == 2
    with pytest.raises(NotImplementedError):
        _lib.check(rc, "backproject")
    gbc = fp.ConfigBackproject(fast_approx=True, backproj_weighting_preset=7, Z_on_val_factor_val=100.0,
                               soft_vartheta_v=0.2, soft_vartheta_v_softspan=0.05, soft_vartheta_h=0.4,
                               soft_vartheta_h_softspan=0.05).contents
    bad = [
        (fp.ConfigBackproject(fast_approx=True).contents, _fake() + 4096),       # preset 0
        (fp.ConfigBackproject(backproj_weighting_preset=7, Z_on_val_factor_val=100.0).contents, _fake() + 4096),  # exact
        (gbc, None),                                                             # no weight-sum volume
        (gbc, _fake()),                                                          # aliases the volume
        (gbc, _fake() + 2),                                                      # unaligned
    ]
    for c, ws in bad:
        rc = lib.aprict_b200_backproject_gbc(_fake(), _lib.ptr(pd), _fake(), _lib.ptr(vd), _fake(), ws, None,
                                             _lib.ptr(c), None, None)
        assert rc in (1, 2)
    assert lib.aprict_b200_conebeam_spectral(_fake(), 4, 4, 4, ctypes.c_double(1.0), ctypes.c_double(4.0),
                                             ctypes.c_double(0.1), None) == 1  # cone angle > pi
    assert lib.aprict_b200_gbc_weight_integral(_fake(), 3, _fake(), 1, 10, _lib.ptr(gbc), None) == 1  # num_z < 2
    assert lib.aprict_b200_vol_div_softzero(None, _fake(), _fake(), 10, ctypes.c_float(1e-6), None) == 1


def test_volops_validation() -> None:
    lib = _lib.lib()
    assert lib.aprict_b200_vol_fill(None, 0, ctypes.c_float(1.0), None) == 0
    assert lib.aprict_b200_vol_fill(None, 10, ctypes.c_float(1.0), None) == 1
    assert lib.aprict_b200_vol_fill(_fake(), -1, ctypes.c_float(1.0), None) == 1
    vd = _lib.vol_desc((4, 4, 4), "C", 1.0, np.zeros(3))
    assert lib.aprict_b200_vol_softmask_cylinder(_fake(), _lib.ptr(vd), ctypes.c_float(1.5), None) == 1


def test_ramp_fft_tables_validate_on_the_host() -> None:
    lib = _lib.lib()
    # 32 bytes per point of the transform, N = 2^p >= 2 nu - 1, for 128 <= nu <= 2048
    assert lib.aprict_b200_ramp_fft_tables_bytes(127) == 0
    assert lib.aprict_b200_ramp_fft_tables_bytes(2049) == 0
    assert lib.aprict_b200_ramp_fft_tables_bytes(128) == 32 * 256
    assert lib.aprict_b200_ramp_fft_tables_bytes(129) == 32 * 512
    assert lib.aprict_b200_ramp_fft_tables_bytes(1024) == 32 * 2048
    assert lib.aprict_b200_ramp_fft_tables_bytes(2048) == 32 * 4096
    assert lib.aprict_b200_ramp_fft_tables(_fake(), 100, _fake(), None) == 2
    assert lib.aprict_b200_ramp_fft_tables(None, 256, _fake(), None) == 1
    assert lib.aprict_b200_ramp_fft_tables(_fake(), 256, _fake() + 8, None) == 1
    din = _lib.proj_desc((3, 300, 2), (600, 2, 1))
    dout = _lib.proj_desc((3, 300, 3), (900, 3, 1))
    dshort = _lib.proj_desc((3, 100, 2), (200, 2, 1))
    args = (None, 0, 0, ctypes.c_float(1.0), None)
    src, dst = _fake(), _fake() + (1 << 24)
    assert lib.aprict_b200_ramp_filter_fft(_lib.ptr(din), src, _lib.ptr(dout), dst, _fake(), *args) == 1
    assert lib.aprict_b200_ramp_filter_fft(_lib.ptr(din), src, _lib.ptr(din), src, _fake(), *args) == 1
    assert lib.aprict_b200_ramp_filter_fft(_lib.ptr(dshort), src, _lib.ptr(dshort), dst, _fake(), *args) == 2
    assert lib.aprict_b200_ramp_filter_fft(_lib.ptr(din), src, _lib.ptr(din), dst, None, *args) == 1
    assert lib.aprict_b200_ramp_filter_fft(_lib.ptr(din), src, _lib.ptr(din), dst, _fake() + 8, *args) == 1


def test_tuning_knobs_validate_and_round_trip() -> None:
    lib = _lib.lib()
    saved = [lib.aprict_b200_get_tuning(k) for k in range(8)]
    try:
        for key, good, bad in [(0, (0, 8, 16, 32), (7, 64, -1)), (1, (0, 2, 4, 8), (1, 3, 16)), (2, (0, 1, 16), (-1, 17)),
                               (3, (0, 8, 16, 32), (4, 64)), (4, (0, 1, 2, 4), (3, 8, -1)), (5, (0, 1, 2, 4), (3, 8)),
                               (6, (0, 1), (2, -1)), (7, (0, 1), (2, -1))]:
            for v in good:
                assert lib.aprict_b200_set_tuning(key, v) == 0
                assert lib.aprict_b200_get_tuning(key) == v
            for v in bad:
                with pytest.raises(ValueError):
                    _lib.check(lib.aprict_b200_set_tuning(key, v), "set_tuning")
        with pytest.raises(ValueError):
            _lib.check(lib.aprict_b200_set_tuning(8, 0), "set_tuning")
        assert lib.aprict_b200_get_tuning(99) == 0
    finally:
        for k, v in enumerate(saved):
            lib.aprict_b200_set_tuning(k, v)


def test_batch_plan_validates_on_the_host() -> None:
    lib = _lib.lib()
    assert lib.aprict_b200_batch_plan_bytes(0, 0) == 0
    assert lib.aprict_b200_batch_plan_bytes(7, 3) == 0
    n1, n96, n97 = (lib.aprict_b200_batch_plan_bytes(1, k) for k in (1, 96, 97))
    assert 0 < n1 < n96 < n97
    assert lib.aprict_b200_batch_plan_bytes(0, 3) > 0
    raw = np.zeros(n97 + 256, np.uint8)
    buf = raw[(-raw.ctypes.data) % 256 :]
    scans = np.zeros(2, S.scan)
    for i, order in enumerate(("C", "F")):
        scans[i]["specs_dev"] = _fake()
        scans[i]["projs"] = _lib.proj_desc((2, 4, 4), (16, 4, 1))
        scans[i]["projs_dev"] = _fake()
        scans[i]["vol"] = _lib.vol_desc((4, 4, 4), order, 1.0, np.zeros(3))
        scans[i]["vol_dev"] = _fake()
    cfgs = np.zeros(2, S.backproject_config)
    cfgs["ssx"] = cfgs["ssy"] = cfgs["ssz"] = 1
    cap = lib.aprict_b200_batch_plan_bytes(1, 2)
    # unknown op, too small a buffer, misaligned buffer, mixed volume order
    for op, c, ptr in [(5, cap, buf.ctypes.data), (1, cap - 1, buf.ctypes.data), (1, cap, buf.ctypes.data + 4),
                       (1, cap, buf.ctypes.data)]:
        with pytest.raises(ValueError):
            _lib.check(lib.aprict_b200_batch_plan(op, _lib.ptr(scans), 2, _lib.ptr(cfgs), ptr, c), "batch_plan")
    assert "same volume order" in lib.aprict_b200_last_error().decode()
    # a bad scan is reported with its index
    scans[1]["vol"] = _lib.vol_desc((4, 4, 4), "C", -1.0, np.zeros(3))
    with pytest.raises(ValueError, match="scan 1"):
        _lib.check(lib.aprict_b200_batch_plan(1, _lib.ptr(scans), 2, _lib.ptr(cfgs), buf.ctypes.data, cap), "batch_plan")
    # running something that is not a plan
    with pytest.raises(ValueError):
        _lib.check(lib.aprict_b200_batch_run(buf.ctypes.data, buf.ctypes.data, None), "batch_run")


def test_batch_records_keep_the_c_layout() -> None:
    from aprict_b200.batch import _packed

    recs = _packed([np.zeros((), S.scan)] * 3, S.scan)
    assert recs.dtype.itemsize == _lib.lib().aprict_b200_struct_size(b"aprict_scan") == 120
