import functools
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    # temporary files of the tests stay inside the repository tree
    if config.option.basetemp is None:
        config.option.basetemp = os.path.join(ROOT, ".pytest_tmp")


@functools.lru_cache(maxsize=None)
def synth_text(kind: str, seed: int):
    from ps_claude_opt_b200 import synth

    cfgs = {
        # tiny: seconds on the oracle
        "tiny": synth.SynthConfig(l_max=3, m_max=3, nrows=4, n_dense=4, dense_pts=(24, 24), n_freq=6),
        # C1 shape (lmax 3, nrows 6, 20 x 60 relative points), 8 trial frequencies
        "c1": synth.SynthConfig(n_freq=8),
        # mixed relative + calibrated, lmax 4 (ia[1] fitted)
        "mixed": synth.SynthConfig(l_max=4, m_max=4, nrows=5, n_dense=6, dense_pts=(20, 40), n_sparse=60,
                                   sparse_curves=2, n_freq=6),
        # C2 shape (lmax 6, nrows 8, 40 dense + 400 calibrated points), few frequencies
        "c2": synth.SynthConfig(l_max=6, m_max=6, nrows=8, n_dense=40, dense_pts=(50, 120), n_sparse=400,
                                sparse_curves=2, n_freq=4),
        # the largest model: lmax 8 (81 coefficients, ma 89), 800 facets, calibrated data
        # (ia[1] fitted -> 88 fitted parameters: 12 x 12 blocks of J^T W J)
        "lmax8": synth.SynthConfig(l_max=8, m_max=8, nrows=10, n_dense=4, dense_pts=(30, 40), n_sparse=40,
                                   sparse_curves=1, n_freq=3),
        # lmax 8, relative data only (87 fitted parameters)
        "lmax8rel": synth.SynthConfig(l_max=8, m_max=8, nrows=10, n_dense=5, dense_pts=(30, 40), n_freq=3),
        # stop condition < 1: fits run until the rms improves by less than 0.005
        # (at least 10, at most 60 iterations)
        "conv": synth.SynthConfig(l_max=3, m_max=3, nrows=5, n_dense=8, dense_pts=(30, 40), n_freq=4,
                                  stop_condition=0.005),
        # calibrated data only: no relative curve, no renormalisation
        "calonly": synth.SynthConfig(l_max=4, m_max=4, nrows=6, n_dense=0, n_sparse=150, sparse_curves=3, n_freq=3),
        # ragged: relative curves of 1 to 3 points beside one calibrated curve
        "ragged": synth.SynthConfig(l_max=3, m_max=3, nrows=5, n_dense=12, dense_pts=(1, 3), n_sparse=40,
                                    sparse_curves=1, n_freq=3),
        # the largest input: 199 lightcurves (200 with the pseudo-curve, the
        # reference's MAX_LC) of 100 points = 19 900 points, lmax 8, 800 facets
        "maxsize": synth.SynthConfig(l_max=8, m_max=8, nrows=10, n_dense=199, dense_pts=(100, 100), n_freq=2),
    }
    text, truth = synth.generate(cfgs[kind], seed)
    return text, truth


def prepared(kind: str, seed: int = 11, setup="oracle"):
    from ps_claude_opt_b200 import objects

    text, _ = synth_text(kind, seed)
    if setup == "oracle":
        import oracle

        return objects.parse_input(text, setup_fn=oracle.setup_shape)
    return objects.parse_input(text)
