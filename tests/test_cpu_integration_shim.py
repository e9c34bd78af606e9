"""The binding INTEGRATION.md gives a PeriodSearch maintainer
(ps_claude_opt_b200/host/start_b200.cpp) compiles against the reference's own
headers and links against libps_b200.so: oracle/refapp/build.sh builds the
reference's unchanged host program (period_search_BOINC.cpp and its setup
sources) with that file in place of start_CUDA.cu, as refapp_b200shim.

Without a GPU the program still reads its input through the reference's own
reader and calls the reference's CUDAPrepare -- here the binding -- which
must reach the C ABI and report the missing device through ps_last_error
(exit 2, the reference's own failure code for CUDAPrepare) instead of
crashing.  The GPU run of the same program is in test_gpu_refapp_parity.py.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "oracle", "_ref", "refapp_b200shim")
LIB = os.path.join(ROOT, "ps_claude_opt_b200", "_lib", "libps_b200.so")
ENTRY_POINTS = ["ps_gpu_prepare", "ps_gpu_precalc", "ps_gpu_start", "ps_gpu_unprepare"]


def _undefined(path):
    out = subprocess.run(["nm", "-D", "--undefined-only", path], capture_output=True, text=True, check=True).stdout
    return {l.split()[-1] for l in out.splitlines() if l.strip()}


def _defined(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {l.split()[-1] for l in out.splitlines() if l.strip()}


@pytest.fixture(scope="module")
def shim():
    if not os.path.exists(SHIM):
        pytest.skip("refapp_b200shim not built (needs the reference source tree: oracle/refapp/build.sh)")
    return SHIM


def test_shim_binds_the_four_entry_points(shim):
    need = {s for s in _undefined(shim) if s.startswith("ps_")}
    assert set(ENTRY_POINTS) <= need
    assert need <= _defined(LIB), "symbols the binding needs that libps_b200.so does not export"
    needed = subprocess.run(["readelf", "-d", shim], capture_output=True, text=True, check=True).stdout
    assert "libps_b200.so" in needed


def test_shim_reaches_the_c_abi_without_a_gpu(shim, tmp_path):
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present: the GPU test runs this program for real")
    except ImportError:
        pass
    from ps_claude_opt_b200 import synth

    text, _ = synth.generate(synth.SynthConfig(n_freq=3), 1000003)
    (tmp_path / "period_search_in").write_text(text + synth.NEUTRAL_WEIGHT_LINE)
    r = subprocess.run([shim, "--device", "0"], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode == 2, (r.returncode, r.stderr[-2000:])
    assert "ps_gpu_prepare:" in r.stderr
    assert "20  Number of light curves" in r.stdout   # the reference's own reader ran
