"""Launch-shape wisdom text on the host (no GPU): `ffcm_wisdom_import` /
`ffcm_wisdom_export`, the analogue of FFTW's exported wisdom for the
reference's `fft_planning = :measure` (src/config.jl:416-423). Parsing and
the store live on the host, so these run without a device."""
import ctypes

import pytest

LINE_A = "ffcm-wisdom-2 7 4 96 96 96 148 2 8 148 3 8 148 0"
LINE_B = "ffcm-wisdom-2 7 8 48 96 32 148 1 4 296 0 2 0 0"


def test_import_then_export_round_trip(ffcm):
    ffcm.wisdom_import(LINE_A + "\n\n" + LINE_B + "\n")
    text = ffcm.wisdom_export()
    lines = text.splitlines()
    assert LINE_A in lines and LINE_B in lines
    # re-importing the export is idempotent
    ffcm.wisdom_import(text)
    assert ffcm.wisdom_export() == text


def test_import_replaces_the_same_key(ffcm):
    ffcm.wisdom_import("ffcm-wisdom-2 7 4 96 96 96 148 0 4 0 0 4 0 0")
    lines = ffcm.wisdom_export().splitlines()
    assert "ffcm-wisdom-2 7 4 96 96 96 148 0 4 0 0 4 0 0" in lines
    assert LINE_A not in lines


@pytest.mark.parametrize("bad", [
    "ffcm-wisdom-2 7 4 96 96 96 148 2 8 148 3 8 148",          # a field short
    "ffcm-wisdom-2 7 4 96 96 96 148 2 8 148 3 8 148 0 5",      # a field too many
    "ffcm-wisdom-1 7 4 96 96 96 2 8 148 3 8 148 0",            # the format without the SM count
    "ffcm-wisdom-2 7 6 96 96 96 148 2 8 148 3 8 148 0",        # element size 6
    "ffcm-wisdom-2 7 4 96 0 96 148 2 8 148 3 8 148 0",         # empty grid axis
    "ffcm-wisdom-2 7 4 96 96 96 148 2 8 -1 3 8 148 0",         # negative grid
    "ffcm-wisdom-2 7 4 96 96 96 0 2 8 148 3 8 148 0",          # no SMs
    "ffcm-wisdom-2 7 4 96 96 96 148 2 8 2147483647 3 8 148 0", # a y grid no GPU runs
    "ffcm-wisdom-2 7 4 96 96 96 148 2 8 148 3 8 999999 0",     # a z grid no GPU runs
])
def test_malformed_text_imports_nothing(ffcm, bad):
    before = ffcm.wisdom_export()
    fresh = "ffcm-wisdom-2 9 4 64 64 64 148 0 8 0 0 8 0 0"
    with pytest.raises(ffcm.ArgumentError):
        ffcm.wisdom_import(fresh + "\n" + bad + "\n")
    assert ffcm.wisdom_export() == before      # not even the valid first line


def test_export_truncates_to_the_buffer_and_reports_the_length(ffcm):
    lib = ffcm._lib.load()
    full = ffcm.wisdom_export().encode()
    n = lib.ffcm_wisdom_export(None, 0)
    assert n == len(full)
    buf = ctypes.create_string_buffer(11)
    assert lib.ffcm_wisdom_export(buf, 11) == len(full)
    assert buf.value == full[:10]
