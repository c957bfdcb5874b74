"""Host side of the outer driver's ice history (no GPU): the --ice-seq grammar and the --times
checks of the reference (run_outer.py:156-183, npyio.py:180-193), restated as expectations."""

import numpy as np
import pytest

from slevolve_b200.icehist import IceHistory, parse_ice_seq, read_times, step_lengths


def test_parse_ice_seq_entries():
    assert parse_ice_seq("0, 1:2:0.25\n3,,") == [(0,), (1, 2, 0.25), (3,)]
    assert parse_ice_seq(" 4 ") == [(4,)]
    assert parse_ice_seq("") == []
    assert parse_ice_seq("-1,0:-1:1e-3") == [(-1,), (0, -1, 1e-3)]


def test_parse_ice_seq_from_file(tmp_path):
    f = tmp_path / "seq.txt"
    f.write_text("0\n0:1:0.5\n1\n")
    assert parse_ice_seq("@" + str(f)) == [(0,), (0, 1, 0.5), (1,)]
    assert parse_ice_seq("@virtual", read_file=lambda p: "2,1:0:0.75") == [(2,), (1, 0, 0.75)]


@pytest.mark.parametrize("bad", ["1:2", "1:2:0.5:3", "a", "1:b:0.5", "1:2:x"])
def test_parse_ice_seq_rejects_malformed_entries(bad):
    with pytest.raises(ValueError):
        parse_ice_seq(bad)


def test_read_times_and_step_lengths(tmp_path):
    f = tmp_path / "t.txt"
    f.write_text("-1000\n-800\n-500\n-100\n")
    t = read_times(str(f))
    assert t.tolist() == [-1000.0, -800.0, -500.0, -100.0]
    assert read_times(str(f), nsteps=2).tolist() == [-1000.0, -800.0, -500.0]
    assert step_lengths(t, 4).tolist() == [200.0, 300.0, 400.0]
    with pytest.raises(ValueError):
        step_lengths(t, 5)
    with pytest.raises(ValueError):
        read_times(str(f), nsteps=4)
    for bad in ([0.0], [0.0, 0.0], [1.0, 0.5], [0.0, np.inf], [0.0, np.nan]):
        with pytest.raises(ValueError):
            read_times(np.array(bad))


def test_history_indices_checked():
    stack = np.zeros((3, 4, 8))
    h = IceHistory(stack, parse_ice_seq("0,0:2:0.5,-1"))
    assert len(h) == 3 and h.nsteps == 2 and h.shape == (4, 8)
    assert IceHistory(stack).items == [(0,), (1,), (2,)]
    with pytest.raises(IndexError):
        IceHistory(stack, [(3,)])
    with pytest.raises(IndexError):
        IceHistory(stack, [(0, 5, 0.5)])


def test_blend_argument_checks_before_any_device_call():
    from slevolve_b200 import _lib

    lib = _lib.lib()
    assert lib.sle_ice_blend(None, None, None, 0.5, -1, None) == _lib.SLE_ERR_BAD_ARG
    assert lib.sle_ice_blend(None, None, None, 0.5, 16, None) == _lib.SLE_ERR_BAD_ARG
    assert b"sle_ice_blend" in lib.sle_last_error()
    with pytest.raises(ValueError):
        _lib.check(lib.sle_ice_blend(None, None, None, 0.5, -1, None), "sle_ice_blend")
    assert lib.sle_ice_blend(None, None, None, 0.5, 0, None) == _lib.SLE_OK
