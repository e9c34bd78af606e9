"""The C++ host program end to end on the GPU: period_search_in in,
period_search_out out, through the C ABI -- the same lines as the Python
driver over the same library, and an interrupted run resumed from its
checkpoint giving the same file as an uninterrupted one."""
import os
import subprocess

import pytest

from conftest import synth_text

pytestmark = pytest.mark.gpu


def _run(args, cwd):
    from ps_claude_opt_b200 import native

    r = subprocess.run([native.HOST_PROGRAM, *args], cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r


@pytest.mark.parametrize("kind", ["tiny", "mixed"])
def test_host_program_matches_python_driver(kind, tmp_path):
    from ps_claude_opt_b200 import native, objects

    text, _ = synth_text(kind, 11)
    (tmp_path / "period_search_in").write_text(text)
    _run(["--max-freq", "6"], tmp_path)            # default file names in the working directory
    got = (tmp_path / "period_search_out").read_text()
    obj = objects.parse_input(text)
    lines, conw_r = native.run_object(obj, max_freq=6)
    assert got == native.format_lines(lines)
    n, new_conw, cw = (tmp_path / "period_search_state").read_text().split()
    assert int(n) == 6 and float(cw) == conw_r


def test_host_program_resumes_from_checkpoint(tmp_path):
    text, _ = synth_text("tiny", 11)
    (tmp_path / "in").write_text(text)
    _run(["-s", "full_state", "--max-freq", "6", "in", "full_out"], tmp_path)
    # interrupted after the first chunk of 2 frequencies
    _run(["-s", "state", "--chunk", "2", "--stop-after", "1", "--max-freq", "6", "in", "out"], tmp_path)
    assert len((tmp_path / "out").read_text().splitlines()) == 2
    assert (tmp_path / "state").read_text().split()[0] == "2"
    # a line written after the last checkpoint is dropped on resume
    with open(tmp_path / "out", "a") as f:
        f.write("0.0  0.0  0.0  0.0    0    0\n")
    _run(["-s", "state", "--chunk", "2", "--max-freq", "6", "in", "out"], tmp_path)
    assert (tmp_path / "out").read_text() == (tmp_path / "full_out").read_text()
    assert (tmp_path / "state").read_text().split()[0] == "6"
