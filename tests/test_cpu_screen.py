"""CPU checks of the screening restatement (oracle/screen_ref.py) that the
GPU tests compare the kernels with: BF16 rounding, the fold statistics on a
known periodic signal, and the network's backward pass against finite
differences."""
import numpy as np

from oracle import screen_ref


def test_bf16_round():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 3.0e38, 0.0], dtype=np.float32)
    r = screen_ref.bf16_round(x)
    assert list(r[:4]) == [1.0, 1.0, 1.0 + 2 * 2.0 ** -7, -2.5]   # ties go to the even neighbour
    assert r[5] == 0.0
    u = r.view(np.uint32)
    assert np.all(u & 0xFFFF == 0)


def test_fold_statistics_of_a_double_peaked_curve():
    rng = np.random.default_rng(0)
    f0 = 3.7                                            # rotations per day
    t = np.sort(rng.uniform(0.0, 40.0, 600))
    br = 1.0 + 0.2 * np.cos(2 * np.pi * 2 * f0 * t + 0.3) + 0.002 * rng.standard_normal(600)
    lens = [300, 300]
    at = screen_ref.features(t, br, lens, [f0, 1.2345])
    # at the rotation frequency: little dispersion, power in the second harmonic
    theta64_all = at[0, 64 + 0]
    h2_all = at[0, 64 + 5]
    assert theta64_all < 0.05 and h2_all > 0.9
    # at an unrelated frequency the fold explains little
    assert at[1, 64 + 3] > 0.5 and at[1, 64 + 0] > 10 * theta64_all
    assert at.shape == (2, 88)


def test_network_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    sizes = (6, 5, 4, 1)
    W = [rng.standard_normal((n, k)) * 0.7 for k, n in zip(sizes[:-1], sizes[1:])]
    b = [rng.standard_normal(n) * 0.1 for n in sizes[1:]]
    x = rng.standard_normal((9, 6))
    y = rng.standard_normal(9)
    loss, _, gW, gb = screen_ref.mlp_forward_backward(x, y, W, b, round_bf16=False)
    h = 1e-6
    for l in range(len(W)):
        for (i, j) in [(0, 0), (W[l].shape[0] - 1, W[l].shape[1] - 1)]:
            Wp = [w.copy() for w in W]
            Wp[l][i, j] += h
            lp = screen_ref.mlp_forward_backward(x, y, Wp, b, round_bf16=False)[0]
            Wp[l][i, j] -= 2 * h
            lm = screen_ref.mlp_forward_backward(x, y, Wp, b, round_bf16=False)[0]
            assert abs((lp - lm) / (2 * h) - gW[l][i, j]) < 1e-6 * max(1.0, abs(gW[l][i, j]))
        bp = [v.copy() for v in b]
        bp[l][0] += h
        lp = screen_ref.mlp_forward_backward(x, y, W, bp, round_bf16=False)[0]
        bp[l][0] -= 2 * h
        lm = screen_ref.mlp_forward_backward(x, y, W, bp, round_bf16=False)[0]
        assert abs((lp - lm) / (2 * h) - gb[l][0]) < 1e-6 * max(1.0, abs(gb[l][0]))


def test_model_file_round_trip_and_errors(tmp_path):
    from ps_claude_opt_b200 import screen

    rng = np.random.default_rng(2)
    state = {"sizes": np.array([88, 7, 1])}
    state["W0"], state["b0"] = rng.standard_normal((7, 88)).astype(np.float32), rng.standard_normal(7).astype(np.float32)
    state["W1"], state["b1"] = rng.standard_normal((1, 7)).astype(np.float32), rng.standard_normal(1).astype(np.float32)
    p = tmp_path / "m.bin"
    screen.save_model(str(p), state)
    sizes, params, back = screen.read_model(str(p))
    assert list(sizes) == [88, 7, 1] and params.size == 88 * 7 + 7 + 7 + 1
    for k in ("W0", "b0", "W1", "b1"):
        assert np.array_equal(back[k], state[k])
    p.write_bytes(p.read_bytes()[:-4])                     # truncated
    import pytest
    with pytest.raises(ValueError):
        screen.read_model(str(p))
    sizes, _, _ = screen.read_model()                       # the committed model
    assert list(sizes) == [88, 256, 256, 256, 1]


def test_selection_is_deterministic_and_bounded():
    from ps_claude_opt_b200 import screen

    pred = np.random.default_rng(5).standard_normal(5000)
    a, b = screen.select(pred), screen.select(pred)
    assert np.array_equal(a, b)
    assert len(a) <= 0.122 * 5000 + 1
    top = np.argsort(pred, kind="stable")[:170]
    assert set(top.tolist()) <= set(a.tolist())
    assert np.all(np.diff(a) > 0)


def _landscape(n, best, depth=0.5, base=0.05, seed=0):
    """Best rms per frequency: noise around `base`, a dip of `depth` at `best`."""
    rng = np.random.default_rng(seed)
    r = base * (1.0 + 0.2 * rng.random(n))
    r[best] = base * depth
    return r


def _plan(pred, rms, **kw):
    from ps_claude_opt_b200 import screen

    calls = []

    def fit(idx):
        calls.append(len(idx))
        return rms[idx]

    return screen.plan_scan(pred, fit, **kw), calls


def test_plan_keeps_a_well_screened_scan_small():
    n = 2000
    rms = _landscape(n, best=777)
    pred = np.log(rms)                     # a perfect ranking
    plan, calls = _plan(pred, rms)
    assert not plan.fallback and plan.expansions == 0
    assert plan.best() == 777 and len(plan.fitted) == plan.initial <= 0.122 * n + 1
    assert len(calls) == 1


def test_plan_expands_around_a_best_line_at_a_run_edge():
    from ps_claude_opt_b200 import screen

    n = 2000
    rms = _landscape(n, best=1000)
    rms[1001:1006] = np.linspace(0.024, 0.020, 5)   # the minimum is wide, falling ...
    rms[1006] = 0.01                                 # ... to its deepest beyond the screened run
    pred = np.full(n, 5.0)
    pred[998:1001] = -5.0                             # the network ranks only 998..1000 first
    plan, _ = _plan(pred, rms, top=0.0015, halo=1, audit=0.0005)
    assert not plan.fallback and plan.expansions == 3
    assert plan.best() == 1006 and {1005, 1007} <= set(plan.fitted)
    assert len(plan.fitted) < 0.05 * n


def test_plan_falls_back_when_the_audit_contradicts_the_ranking():
    n = 2000
    rms = _landscape(n, best=300)
    pred = -np.log(rms)                     # an inverted ranking: the screen misses the dip
    pred[300] = 10.0
    plan, _ = _plan(pred, np.where(np.arange(n) == 300, 0.025, rms), audit=0.05)
    # the top-ranked frequencies all sit near base rms; random audit frequencies
    # reach within 10 % of them, so the scan falls back to the whole grid
    assert plan.fallback and plan.reason == "audit"
    assert plan.fitted == list(range(n)) and plan.best() == 300


def test_plan_falls_back_after_too_many_expansions():
    n = 500
    rms = np.linspace(1.0, 0.5, n)           # monotone: the best keeps moving to the right edge
    pred = np.zeros(n)
    pred[:3] = -1.0
    plan, _ = _plan(pred, rms, top=0.002, halo=0, audit=0.002, max_expansions=3)
    assert plan.fallback and plan.reason in ("edge", "audit") and len(plan.fitted) == n
    assert plan.best() == n - 1


def test_plan_probes_the_period_doubling_partner():
    """A double-peaked curve fits almost as well at twice its period: the
    ranking puts the doubled period first, the probe of the best line's
    partners (twice and half its frequency) finds the true one."""
    from ps_claude_opt_b200 import screen

    n = 2000
    freqs = 0.30 - 1e-4 * np.arange(n)          # 1/h, decreasing like the reference's grid
    true_i = 400                                  # f = 0.26
    alias_i = int(round((0.30 - 0.13) / 1e-4))    # half the frequency: the doubled period
    rms = _landscape(n, best=true_i, depth=0.3)
    rms[alias_i] = rms[true_i] * 1.05
    pred = np.full(n, 5.0)
    pred[alias_i - 1:alias_i + 2] = -5.0          # the network ranks only the alias first
    plan, _ = _plan(pred, rms, top=0.0015, halo=1, audit=0.0005, freqs=freqs)
    assert plan.alias_probes >= 1 and plan.best() == true_i and not plan.fallback
    assert len(plan.fitted) < 0.02 * n
    # without the grid the probe is off and the alias stays the answer
    plan0, _ = _plan(pred, rms, top=0.0015, halo=1, audit=0.0005)
    assert plan0.best() == alias_i and plan0.alias_probes == 0


def test_judgement_summary_counts_hits_fallbacks_and_aliases():
    """screen_train.summarize on hand-made judgement rows: hit rate with its
    one-sided 95 % Clopper-Pearson lower bound, fallbacks, and the period
    ratio of a miss (2.0: the screened scan ended at twice the period)."""
    from ps_claude_opt_b200 import screen_train

    def row(seed, ok, scr_p=10.0, fallback=False, fitted=520):
        return dict(seed=seed, ok=ok, ok_fp64_screen=ok, fallback=fallback, fitted=fitted, n_freq=5000,
                    expansions=1, alias_probes=2, screened_s=2.0, full_s_per_object=26.0,
                    full_line="10.00000000  0.020000  1.000000  1.0  100   20",
                    screened_line="%.8f  0.020000  1.000000  1.0  100   20" % scr_p)

    rows = [row(i, True) for i in range(9)] + [row(9, False, scr_p=20.0, fallback=True, fitted=5000)]
    s = screen_train.summarize(rows)
    assert s["objects"] == 10 and s["hits"] == 9 and s["fallbacks"] == 1
    assert abs(s["hit_rate"] - 0.9) < 1e-12
    # Clopper-Pearson: 9 of 10 -> P(X >= 9 | p) = 0.05 at p = 0.6058
    assert abs(s["hit_rate_lower95"] - 0.6058) < 1e-3
    assert s["fitted_max"] == 5000 and abs(s["fitted_mean"] - (9 * 520 + 5000) / 10) < 1e-9
    assert len(s["misses"]) == 1 and abs(s["misses"][0]["ratio"] - 2.0) < 1e-12
    assert screen_train.summarize([]) == {"objects": 0}
    # all hits: 200 of 200 -> lower bound 0.05 ** (1 / 200)
    s = screen_train.summarize([row(i, True) for i in range(200)])
    assert abs(s["hit_rate_lower95"] - 0.05 ** (1 / 200)) < 1e-9


def test_polish_refits_candidates_and_lets_the_fp64_line_win():
    """Mixed-precision rms puts the doubled period (the alias) just below
    the true one; the FP64 refits of the candidates -- the best line, its
    period-doubling partners, the lowest local minima -- restore the true
    line, and frequencies outside those neighbourhoods keep their mixed rms."""
    from ps_claude_opt_b200 import screen

    n = 2000
    freqs = 0.30 - 1e-4 * np.arange(n)
    true_i = 400
    alias_i = int(round((0.30 - 0.13) / 1e-4))
    rms64 = _landscape(n, best=true_i, depth=0.3)
    rms64[alias_i] = rms64[true_i] * 1.002                 # FP64: the true line wins
    rms_mixed = rms64 * (1.0 + 1e-4 * np.cos(np.arange(n)))
    rms_mixed[alias_i] = rms64[true_i] * 0.999             # mixed: the alias wins
    pred = np.full(n, 5.0)
    pred[alias_i - 1:alias_i + 2] = -5.0
    pred[true_i - 1:true_i + 2] = -4.0
    plan, _ = _plan(pred, rms_mixed, top=0.003, halo=1, audit=0.0005, freqs=freqs)
    assert plan.best() == alias_i
    refits = []

    def fit64(idx):
        refits.append(idx.tolist())
        return rms64[idx]

    before = dict(plan.rms)
    screen.polish_plan(plan, fit64, freqs)
    assert plan.best() == true_i
    done = {i for r in refits for i in r}
    assert {alias_i, true_i} <= done and plan.polished == len(done)
    assert 1 <= plan.polish_rounds <= screen.POLISH_ROUNDS
    assert len(done) <= 5 + 10 + 3 * screen.POLISH_MINIMA + 5 * 2 * (screen.POLISH_ROUNDS - 1)
    for i in set(before) - done:
        assert plan.rms[i] == before[i]
    for i in done:
        assert plan.rms[i] == rms64[i]
    # a second pass over the polished plan keeps the FP64 best line
    screen.polish_plan(plan, fit64, freqs)
    assert plan.best() == true_i
