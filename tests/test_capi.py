"""C ABI checks that need no GPU: the library loads, exports every entry
point include/ctstereo.h declares, and rejects bad arguments with status codes
(never exceptions across the ABI, never a device call)."""
import ctypes as C

import pytest


def test_library_loads_and_versions(ct):
    assert "sm_100a" in ct.version()


def test_every_declared_symbol_is_exported(ct):
    names = ct.exported_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(ct.lib(), n)]
    assert not missing, missing


def test_generator_is_its_own_library(ct):
    """ct_synth_pair lives in libctsynth.so (include/ctsynth.h), not in the
    matcher library."""
    names = ct.exported_symbols("ctsynth.h")
    assert names == ["ct_synth_pair"]
    assert all(hasattr(ct.synth_lib(), n) for n in names)
    assert not hasattr(ct.lib(), "ct_synth_pair")


def test_create_destroy_each_kind(ct):
    for cls in (ct.CensusTransform, ct.BlockMatcherCensus, ct.BlockMatcherSAD1, ct.BlockMatcherNCC,
                ct.BlockMatcherAW, ct.CrossCheckDisparityMaps):
        d = cls()
        d.close()
        d.close()  # idempotent


def test_null_arguments_are_rejected(ct):
    L = ct.lib()
    assert L.ct_census_create(None) == ct.CT_EINVAL
    h = C.c_void_p()
    assert L.ct_census_create(C.byref(h)) == ct.CT_OK
    assert L.ct_census_configure(h, 0, None, None) == ct.CT_EINVAL
    assert b"null" in L.ct_last_error_string()
    # wrong handle kind
    assert L.ct_bm_census_process(h, None, None, None, None) == ct.CT_ESTATE
    assert L.ct_destroy(h) == ct.CT_OK
    assert L.ct_destroy(None) == ct.CT_OK


def test_parameter_validation_before_any_device_call(ct):
    m = ct.BlockMatcherCensus()
    with pytest.raises(ct.CtError) as e:
        m.configure(0, 640, 480, disp_count=0)
    assert e.value.code == ct.CT_EINVAL
    with pytest.raises(ct.CtError) as e:
        m.configure(0, 640, 480, disp_count=64, agg_radius=3)
    assert e.value.code == ct.CT_EINVAL
    with pytest.raises(ct.CtError) as e:
        m.configure(0, 4, 4, disp_count=64)
    assert e.value.code == ct.CT_EINVAL
    # process before configure
    L = ct.lib()
    img = ct.ct_image(1 << 20, 640, 640, 480, ct.CT_PIX_U8, 0)
    rc = L.ct_bm_census_process(m._h, C.byref(img), C.byref(img), C.byref(img), None)
    assert rc == ct.CT_ESTATE


def test_synth_rejects_bad_kind(ct):
    assert ct.synth_lib().ct_synth_pair(9, 1, 16, 16, 8, None, None, None, None) == ct.CT_EINVAL


def test_stream_argument_checks(ct):
    """ct_census_stream_*: state and argument errors before any device call."""
    L = ct.lib()
    h = C.c_void_p()
    assert L.ct_census_stream_create(C.byref(h)) == ct.CT_OK
    k = C.c_int64()
    buf = C.create_string_buffer(64)
    assert L.ct_census_stream_submit(h, buf, 8, buf, 8, buf, 8, C.byref(k)) == ct.CT_ESTATE
    assert L.ct_census_stream_wait(h, 0) == ct.CT_ESTATE
    assert L.ct_census_stream_timer_start(h) == ct.CT_ESTATE
    fmt = ct.ct_format(64, 32, ct.CT_PIX_U8)
    p = ct.ct_census_match_params(64, 2, 1, 0)
    assert L.ct_census_stream_configure(h, 0, C.byref(fmt), C.byref(p), -1, ct.CT_PIX_U8) == ct.CT_EINVAL
    assert L.ct_census_stream_configure(h, 0, C.byref(fmt), C.byref(p), 1, ct.CT_PIX_F32) == ct.CT_ETYPE
    p300 = ct.ct_census_match_params(256, 2, 1, 0)
    assert L.ct_census_stream_configure(h, 0, C.byref(fmt), C.byref(p300), 1, ct.CT_PIX_U8) == ct.CT_ETYPE
    assert L.ct_census_stream_configure(h, 0, None, C.byref(p), 1, ct.CT_PIX_U8) == ct.CT_EINVAL
    assert L.ct_destroy(h) == ct.CT_OK
