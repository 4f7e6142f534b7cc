"""The command-line driver (fg2_b200/cli.py): the reference's argument semantics
(src/main.cpp:36-58, src/misc.cpp:23-55) on the host, and on the GPU a fresh run and a
continuation from a dumped frame that write the same frames as the handle API."""
import os
import subprocess
import sys

import numpy as np
import pytest

from fg2_b200.cli import frame_number, parse

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_defaults():
    c = parse([])
    assert (c["input"], c["n0"], c["n1"], c["n2"], c["l0"], c["d"]) == ("default", 10, 1024, 1024, 1.0, 0)
    assert c["l1"] is None and c["p1"] is None and c["c"] is None and c["para"] == []


def test_options_take_one_to_three_values():
    c = parse(["-n", "5", "256", "-l", "0.5", "2", "3", "-b", "p", "x", "KH", "gamma=1.4", "-c", "0.3"])
    assert (c["n0"], c["n1"], c["n2"]) == (5, 256, 256)
    assert (c["l0"], c["l1"], c["l2"]) == (0.5, 2.0, 3.0)
    assert (c["p1"], c["p2"]) == (True, False)
    assert c["input"] == "KH" and c["para"] == ["gamma=1.4"] and c["c"] == 0.3
    c = parse(["-n", "3", "64", "128", "-l", "1", "-b", "P", "-d", "1"])
    assert (c["n0"], c["n1"], c["n2"], c["l1"], c["p1"], c["p2"], c["d"]) == (3, 64, 128, None, True, None, 1)


def test_values_convert_like_atof_and_atoi():
    # the parser is greedy, as the reference's: a name after an option's first value is taken
    # as its next value (atof("KH") == 0)
    c = parse(["-l", "0.002", "KH"])
    assert c["l0"] == 0.002 and c["l1"] == 0.0 and c["input"] == "default"
    c = parse(["-n", "3x", "1e3"])
    assert c["n0"] == 3 and c["n1"] == 1


def test_a_value_may_be_negative_but_not_an_option():
    # '-' followed by a digit is a value, '-' followed by a letter the next option (src/main.cpp:24-25)
    c = parse(["-l", "-1", "-n", "2"])
    assert c["l0"] == -1.0 and c["n0"] == 2


@pytest.mark.parametrize("argv", [["-n"], ["-x", "3"], ["-l", "-n", "2"], ["--help"]])
def test_bad_options_print_the_usage(argv):
    with pytest.raises(SystemExit):
        parse(argv)


def test_frame_number_is_the_first_number_of_the_name():
    assert frame_number("0012.raw") == 12 and frame_number("KH") == 0 and frame_number("run2/0012.raw") == 2


def _cli(args, cwd):
    env = dict(os.environ, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    return subprocess.run([sys.executable, "-m", "fg2_b200.cli", *args], cwd=cwd, env=env, capture_output=True,
                          text=True, timeout=600)


@pytest.mark.gpu
def test_fresh_run_and_continuation_match_the_api(tmp_path, cuda):
    import fg2_b200
    a, b = tmp_path / "cli", tmp_path / "api"
    a.mkdir()
    b.mkdir()
    r = _cli(["hydro", "KH", "gamma=1.4", "-l", "0.002", "-n", "2", "64"], a)
    assert r.returncode == 0, r.stdout + r.stderr
    r = _cli(["hydro", "0002.raw", "gamma=1.4", "-l", "0.001", "-n", "1", "64"], a)
    assert r.returncode == 0, r.stdout + r.stderr
    assert sorted(os.listdir(a)) == ["0000.raw", "0001.raw", "0002.raw", "0003.raw"]
    with fg2_b200.Sim(64, 64) as s:
        assert s.para("gamma=1.4") is not None
        s.config()
        s.init("KH")
        s.dump(str(b / "0000.raw"), 0.0)
        assert s.solve(0.0, 0.002, 0, 2, str(b))[0] == 0
    with fg2_b200.Sim(64, 64) as s:
        assert s.para("gamma=1.4") is not None
        t = s.load(str(b / "0002.raw"))
        s.config()
        assert s.solve(t, t + 0.001, 2, 3, str(b))[0] == 0
    for f in ("0000.raw", "0001.raw", "0002.raw", "0003.raw"):
        assert (a / f).read_bytes() == (b / f).read_bytes(), f
