"""CPU-side checks of the C-ABI library: it loads, exports every symbol the
header declares, and validates inputs (no GPU needed: validation runs before
any device call)."""

import ctypes as C
import os
import re

import pytest

from goav1_b200 import abi, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def L():
    import goav1_b200

    return goav1_b200.lib()


def test_header_symbols_exported(L):
    hdr = open(os.path.join(ROOT, "include", "goav1pf.h")).read()
    declared = set(re.findall(r"\b(pf_[a-z_]+)\s*\(", hdr))
    assert declared == set(abi.EXPORTED_SYMBOLS)
    for name in declared:
        assert hasattr(L, name), name


def test_struct_sizes_match_header(L):
    # Spot-check layouts that cross the boundary by value.
    assert C.sizeof(abi.pf_lr_unit) == 10
    assert C.sizeof(abi.pf_plane) == 32
    assert C.sizeof(abi.pf_frame) == 16 + 3 * 32
    assert C.sizeof(abi.pf_lf_record) == 32 and abi.lf_record_dtype().itemsize == 32
    assert abi.pf_lf_record.tx_split.offset == 24 and abi.pf_lf_record.delta_lf.offset == 19
    assert C.sizeof(abi.pf_lf_levels) == 20 + 8 * 4 * 2


def test_status_strings(L):
    assert L.pf_status_string(0) == b"ok"
    assert b"cdef" in L.pf_status_string(abi.PF_ERR_INVALID_CDEF)
    assert b"batch" in L.pf_status_string(abi.PF_ERR_INVALID_BATCH)


def _valid(L, fr, si, disp=None):
    return L.pf_frame_validate(C.byref(fr.pf()), C.byref(si.side), C.byref(disp.pf()) if disp else None)


def test_validate_ok_config0(L):
    fr, si = synth.make_frame(0, 1)
    assert _valid(L, fr, si) == abi.PF_OK


def test_validate_rejects_bad_inputs(L):
    fr, si = synth.make_frame(0, 1)
    si.side.cdef.damping = 9
    assert _valid(L, fr, si) == abi.PF_ERR_INVALID_CDEF
    fr, si = synth.make_frame(0, 1)
    si.side.cdef.y_strength[0] = 0x40
    assert _valid(L, fr, si) == abi.PF_ERR_INVALID_CDEF
    fr, si = synth.make_frame(0, 1)
    si.side.lf.mi_cols += 2
    assert _valid(L, fr, si) == abi.PF_ERR_INVALID_FILTER
    fr, si = synth.make_frame(0, 1)
    si.side.lf.sharpness = 8
    assert _valid(L, fr, si) == abi.PF_ERR_INVALID_FILTER
    fr, si = synth.make_frame(0, 1)
    si.side.stages |= 1 << 7
    assert _valid(L, fr, si) == abi.PF_ERR_UNSUPPORTED
    fr, si = synth.make_frame(0, 1)
    pf = fr.pf()
    pf.plane[1].alloc_height = 8
    assert L.pf_frame_validate(C.byref(pf), C.byref(si.side), None) == abi.PF_ERR_SHORT_BUFFER


def test_validate_rejects_bad_restoration_and_grain(L):
    fr, si = synth.make_frame(1, 2, width=256, height=192)
    disp = fr.like()
    assert _valid(L, fr, si, disp) == abi.PF_OK
    units = (abi.pf_lr_unit * si.side.lr.unit_count[0]).from_address(si.side.lr.units[0])
    units[0].type, units[0].wiener_v[1] = abi.PF_LR_WIENER, 20
    assert _valid(L, fr, si, disp) == abi.PF_ERR_INVALID_PLAN
    fr, si = synth.make_frame(1, 2, width=256, height=192)
    si.side.fg.scaling_shift = 7
    assert _valid(L, fr, si, disp) == abi.PF_ERR_INVALID_FORMAT
    fr, si = synth.make_frame(1, 2, width=256, height=192)
    assert _valid(L, fr, si, None) == abi.PF_ERR_INVALID_ARG
    # The display picture may not share memory with the frame.
    assert _valid(L, fr, si, fr) == abi.PF_ERR_INVALID_ARG
    half = fr.like()
    half.planes[2] = fr.planes[1]
    assert _valid(L, fr, si, half) == abi.PF_ERR_INVALID_ARG


def test_runner_without_device_raises():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from goav1_b200 import postfilter

    with pytest.raises(postfilter.ErrNoDevice):
        postfilter.PostFilterRunner()


def test_library_has_no_undefined_project_symbols():
    """Every pf:: function the library calls is defined in it (a missing one
    only shows up when the library is loaded)."""
    import subprocess

    import goav1_b200

    out = subprocess.run(["nm", "-D", "--undefined-only", goav1_b200.LIB_PATH], capture_output=True, text=True).stdout
    assert "_ZN2pf" not in out, out
