"""The autotuner's table format, on the CPU (host code of the library only).

The table maps (knob, element bytes, block edge, AMR level, fill kind) to a
launch-shape choice; sfm_tune_save / sfm_tune_load carry it as text.  These
checks cover parsing, the canonical form written back, and the rejection of
malformed or out-of-range entries without touching a GPU.
"""
import ctypes as C

import pytest

from code_only_b200 import abi


@pytest.fixture(scope="module")
def lib(sfmg_lib):
    return sfmg_lib


def check(lib, text, cap=4096):
    out = C.create_string_buffer(cap)
    rc = lib.sfm_tune_text_check(text.encode(), out, cap)
    return rc, out.value.decode()


def test_roundtrip_is_canonical_and_stable(lib):
    text = ("# a comment\n\nghost_fill 4 8 2 -1 1\nrelax_threads 4 8 -1 -1 512\n"
            "resid_bpc 8 8 -1 -1 4\n   ghost_fill 4 2 3 0 0\n")
    rc, out = check(lib, text)
    assert rc == 4
    lines = [ln for ln in out.splitlines() if ln and not ln.startswith("#")]
    assert lines == ["ghost_fill 4 2 3 0 0", "ghost_fill 4 8 2 -1 1", "relax_threads 4 8 -1 -1 512",
                     "resid_bpc 8 8 -1 -1 4"]
    rc2, out2 = check(lib, out)
    assert rc2 == 4 and out2 == out


def test_later_entry_wins_and_empty_table(lib):
    rc, out = check(lib, "resid_bpc 4 8 -1 -1 1\nresid_bpc 4 8 -1 -1 2\n")
    assert rc == 1 and "resid_bpc 4 8 -1 -1 2" in out
    assert check(lib, "")[0] == 0
    assert check(lib, "# only comments\n")[0] == 0


@pytest.mark.parametrize("bad", [
    "ghost_fill 4 8 2 -1 2",          # not a candidate
    "relax_threads 4 8 -1 -1 384",
    "resid_bpc 4 8 -1 -1 3",
    "unknown_knob 4 8 -1 -1 1",
    "ghost_fill 2 8 2 -1 1",          # element size
    "ghost_fill 4 12 2 -1 1",         # block edge not a power of two
    "ghost_fill 4 8 2 -2 1",          # fill kind
    "ghost_fill 4 8 2 -1",            # missing field
    "ghost_fill 4 8 2 -1 1 7",        # extra field
    "ghost_fill four 8 2 -1 1",
    "base_ctas 8 32 -1 -1 3",          # not a cluster size offered
    "base_wide 8 32 -1 -1 8",
    "fused_sweeps 4 8 -1 -1 4",
    "local_sweeps 4 8 -1 -1 4",
])
def test_malformed_entries_are_rejected(lib, bad):
    assert check(lib, "ghost_fill 4 8 0 -1 1\n" + bad + "\n")[0] == abi.SFM_EINVAL


def test_small_output_buffer(lib):
    rc, _ = check(lib, "ghost_fill 4 8 0 -1 1\n", cap=8)
    assert rc == abi.SFM_ESIZE


def test_base_grid_knobs_parse(lib):
    rc, out = check(lib, "base_ctas 8 32 -1 -1 8\nbase_wide 8 32 -1 -1 16\nbase_ctas 4 16 -1 -1 1\n")
    assert rc == 3 and "base_ctas 8 32 -1 -1 8" in out and "base_wide 8 32 -1 -1 16" in out


def test_fused_sweep_knob_parses(lib):
    rc, out = check(lib, "fused_sweeps 4 8 -1 -1 1\nfused_sweeps 4 16 -1 -1 0\nfused_sweeps 4 4 -1 -1 3\n")
    assert rc == 3 and "fused_sweeps 4 8 -1 -1 1" in out and "fused_sweeps 4 16 -1 -1 0" in out
    assert "fused_sweeps 4 4 -1 -1 3" in out


def test_smoother_cta_sizes_parse(lib):
    rc, out = check(lib, "relax_threads 4 8 -1 -1 288\nrelax_threads 4 8 -1 1 544\nrelax_threads 8 16 -1 -1 512\n")
    assert rc == 3 and "relax_threads 4 8 -1 1 544" in out and "relax_threads 4 8 -1 -1 288" in out


def test_local_sweeps_parse(lib):
    rc, out = check(lib, "local_sweeps 4 8 -1 -1 2\nfused_sweeps 4 8 -1 -1 1\n")
    assert rc == 2 and "local_sweeps 4 8 -1 -1 2" in out
