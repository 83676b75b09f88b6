"""Host-side handling of the device status words (no GPU needed).

The persistent pass's grid barrier sets XPBD_STATUS_BARRIER_TIMEOUT when a
wait gives up and the bit is sticky: every later barrier of later launches
gives up early too.  The tile passes set XPBD_STATUS_ACC_RANGE when a tet's
corrections leave the fixed-point range (or are not finite).  The engine
copies the words behind every frame and raises at the next frame or
synchronising read; these tests pin which bits are fatal.
"""
from rlmusclev2_b200 import _capi as capi
from rlmusclev2_b200.engine import status_error


def test_clean_words_pass():
    assert status_error(0, 0) is None


def test_dcd_overflow_bits_are_warnings_only():
    warn = capi.STATUS_PAIR_OVERFLOW | capi.STATUS_CONTACT_OVERFLOW | capi.STATUS_STACK_OVERFLOW
    assert status_error(0, warn) is None


def test_barrier_timeout_is_fatal():
    msg = status_error(capi.STATUS_BARRIER_TIMEOUT)
    assert msg is not None and "grid barrier" in msg and "cleared" in msg


def test_accumulator_range_is_fatal():
    msg = status_error(capi.STATUS_ACC_RANGE)
    assert msg is not None and "fixed-point" in msg


def test_dcd_sort_timeout_is_fatal():
    msg = status_error(0, capi.STATUS_BARRIER_TIMEOUT)
    assert msg is not None and "DCD" in msg


def test_all_fatal_bits_reported_together():
    msg = status_error(capi.STATUS_BARRIER_TIMEOUT | capi.STATUS_ACC_RANGE, capi.STATUS_BARRIER_TIMEOUT)
    assert msg.count(";") == 2
