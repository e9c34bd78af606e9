"""The host program's screened-scan control flow (ps_claude_opt_b200/host/
screen_flow.h, compiled here into tests/screen_flow_driver.cpp) against the
Python one (ps_claude_opt_b200.screen: select_parts, plan_scan,
polish_plan) on the same synthetic rms landscapes: the same core and audit
sample, the same fit calls in the same order, the same expansions, probes,
fallbacks and FP64 refits, and the same best line.  No GPU: the fits are
lookups in the landscape."""
import json
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

F0, DF = 0.5, 2.0 ** -13   # the grid freq_start - i freq_step (0.5 .. 0.134), exact in binary


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("flow") / "screen_flow_driver")
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "ps_claude_opt_b200", "host"),
                        os.path.join(HERE, "screen_flow_driver.cpp"), "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _landscape(n, rng, best, depth=0.4, width=3.0, base=0.03):
    i = np.arange(n)
    rms = base * (1 + 0.05 * rng.random(n))
    rms *= 1 - depth * np.exp(-0.5 * ((i - best) / width) ** 2)
    return rms


def _cases():
    """(name, scores, first-pass rms, FP64 rms, top, halo, audit, seed)."""
    out = []
    n = 3000
    for k in range(6):                                   # well-ranked, noisy scores
        rng = np.random.default_rng(100 + k)
        best = int(rng.integers(50, n - 50))
        rms = _landscape(n, rng, best)
        score = np.log(rms) + 0.05 * rng.standard_normal(n)
        out.append(("ranked%d" % k, score, rms, rms * (1 + 1e-4 * rng.standard_normal(n)), 0.034, 1, 0.02, k))
    rng = np.random.default_rng(7)
    rms = _landscape(n, rng, 1500, depth=0.1)            # ranked dip at 0.027-0.028 ...
    rms[1501:1506] = np.linspace(0.024, 0.020, 5)        # ... falling past the ranked run
    rms[1506] = 0.01                                     # deepest beyond the ranked run: expansions
    score = np.full(n, 5.0)
    score[1498:1501] = -5.0
    out.append(("edge", score, rms, rms, 0.0015, 1, 0.0005, 3))
    rng = np.random.default_rng(8)
    rms = _landscape(n, rng, 700, depth=0.05)            # a dip within the noise of the rest ...
    score = -np.log(rms)                                 # ... and a ranking that puts it last
    out.append(("inverted", score, rms, rms, 0.034, 1, 0.05, 1))   # the audit contradicts: fallback
    rms = np.linspace(1.0, 0.5, 600)                     # runaway edge: fallback after the expansions
    score = np.zeros(600)
    score[:3] = -1.0
    out.append(("runaway", score, rms, rms, 0.002, 0, 0.002, 2))
    # a double-peaked curve: the doubled period wins in the first pass (the
    # probe finds the true one), or only in mixed precision (the FP64
    # refits restore the true one)
    freqs = F0 - DF * np.arange(n)
    for name, first_pass_alias_wins in (("alias_probe", False), ("alias_mixed", True)):
        rng = np.random.default_rng(9)
        true_i = 1200
        alias_i = int(round((F0 - 0.5 * freqs[true_i]) / DF))
        rms64 = _landscape(n, rng, true_i, depth=0.3)
        rms64[alias_i] = rms64[true_i] * (1.002 if first_pass_alias_wins else 1.05)
        rms = rms64 * (1 + 1e-4 * np.cos(np.arange(n)))
        if first_pass_alias_wins:
            rms[alias_i] = rms64[true_i] * 0.999
        score = np.full(n, 5.0)
        score[alias_i - 1:alias_i + 2] = -5.0
        score[true_i - 1:true_i + 2] = -4.0 if first_pass_alias_wins else 5.0
        out.append((name, score, rms, rms64, 0.003 if first_pass_alias_wins else 0.0015, 1, 0.0005, 4))
    rng = np.random.default_rng(10)                      # NaN lines never win
    rms = _landscape(n, rng, 2000)
    rms[rng.choice(n, 300, replace=False)] = np.nan
    rms[2000] = np.nan
    out.append(("nan", np.nan_to_num(np.log(rms), nan=0.0), rms, rms, 0.034, 1, 0.02, 5))
    return out


def _python(score, rms, rms64, top, halo, audit, seed, polish):
    from ps_claude_opt_b200 import screen

    n = len(score)
    freqs = F0 - DF * np.arange(n)
    calls = []

    def fit(idx):
        calls.append(idx.tolist())
        return rms[idx]

    def fit64(idx):
        calls.append(idx.tolist())
        return rms64[idx]

    core, aud = screen.select_parts(score, top, halo, audit, seed)
    plan = screen.plan_scan(score, fit, top, halo, audit, seed, freqs=freqs)
    best_plan = plan.best()
    if polish:
        screen.polish_plan(plan, fit64, freqs)
    return dict(core=sorted(core), audit=sorted(aud), fitted=plan.fitted, calls=calls, initial=plan.initial,
                expansions=plan.expansions, alias_probes=plan.alias_probes, fallback=plan.fallback,
                reason=plan.reason, best_plan=best_plan, best=plan.best(), polished=plan.polished,
                polish_rounds=plan.polish_rounds)


def _cpp(driver, score, rms, rms64, top, halo, audit, seed, polish):
    n = len(score)
    text = "%d %.17g %d %.17g %d %.17g %.17g %d\n" % (n, top, halo, audit, seed, F0, DF, int(polish))
    text += " ".join("%.9g" % x for x in score) + "\n"
    text += " ".join("%.17g" % x for x in rms) + "\n"
    text += " ".join("%.17g" % x for x in rms64) + "\n"
    r = subprocess.run([driver], input=text, capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout)


def test_flow_constants_agree():
    from ps_claude_opt_b200 import screen

    src = open(os.path.join(ROOT, "ps_claude_opt_b200", "host", "screen_flow.h")).read()
    for name, value in (("kAuditMargin", screen.AUDIT_MARGIN), ("kEdge", screen.EDGE_WIDTH),
                        ("kMaxExpansions", screen.MAX_EXPANSIONS), ("kPolishMinima", screen.POLISH_MINIMA),
                        ("kPolishRounds", screen.POLISH_ROUNDS)):
        line = next(l for l in src.splitlines() if l.lstrip().startswith("constexpr") and name + " =" in l)
        assert float(line.split("=")[1].split(";")[0]) == value, name


@pytest.mark.parametrize("polish", [False, True])
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_host_flow_equals_python_flow(driver, case, polish):
    name, score, rms, rms64, top, halo, audit, seed = case
    score = np.asarray(score, dtype=np.float32)
    py = _python(score, rms, rms64, top, halo, audit, seed, polish)
    cc = _cpp(driver, score, rms, rms64, top, halo, audit, seed, polish)
    for key in py:
        assert cc[key] == py[key], (name, key)


def test_cases_cover_every_branch(driver):
    """The landscapes reach each branch of the flow: expansions, a probe that
    moves the best line, both fallbacks, and FP64 refits that move it."""
    seen, first = {}, {}
    for name, score, rms, rms64, top, halo, audit, seed in _cases():
        seen[name] = _python(np.asarray(score, dtype=np.float32), rms, rms64, top, halo, audit, seed, True)
        first[name] = rms
    assert seen["edge"]["expansions"] >= 1 and not seen["edge"]["fallback"]
    assert seen["inverted"]["fallback"] and seen["inverted"]["reason"] == "audit"
    assert seen["runaway"]["fallback"]
    assert seen["alias_probe"]["alias_probes"] >= 1 and seen["alias_probe"]["best"] == 1200
    assert seen["alias_mixed"]["best_plan"] != 1200 and seen["alias_mixed"]["best"] == 1200
    assert np.isfinite(first["nan"][seen["nan"]["best_plan"]]) and seen["nan"]["best_plan"] != 2000
