"""The learned form's CPU oracle (oracle/mlp_oracle.py): gradient against
central differences, bf16 rounding against known values, the parameter
layout against the library's count, and the library's host code of the
targets' baseline (terms, nested evaluation, ridge solve) against the
oracle's restatement (no GPU call)."""
import numpy as np

from oracle import mlp_oracle as M


def test_bf16_round_known_values():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -7, -2.5,
                  3.0e38, np.inf, 0.0], np.float32)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties to even -> 1;
    # 1 + 3*2^-8 is halfway between 1 + 2^-7 and 1 + 2^-6: ties to even -> 1 + 2^-6
    want = [1.0, 1.0, 1.0 + 2.0 ** -6, 1.0 + 2.0 ** -7, -2.5, 2.9983e38, np.inf, 0.0]
    got = M.bf16_round(x)
    assert np.allclose(got[:5], want[:5], rtol=0, atol=0)
    assert abs(got[5] / 3.0e38 - 1) < 2.0 ** -8
    assert got[6] == np.inf and got[7] == 0.0


def test_gradient_against_central_differences():
    rng = np.random.default_rng(3)
    p = M.random_params(7).astype(np.float64)
    x = rng.standard_normal((40, M.N_IN))
    y = rng.standard_normal((40, M.N_OUT))
    _, g = M.loss_and_grad(p, x, y)
    # every bias plus a sample of weights from every matrix
    idx = [o + k for name, (o, s) in M.OFF.items() for k in
           (range(s) if name.startswith("b") else rng.choice(s, 24, replace=False))]
    h = 1e-6
    worst = 0.0
    for i in idx:
        if name_of(i) in ("W1",) and (i - M.OFF["W1"][0]) % 16 >= M.N_IN:
            continue
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (M.loss_and_grad(pp, x, y)[0] - M.loss_and_grad(pm, x, y)[0]) / (2 * h)
        worst = max(worst, abs(fd - g[i]) / max(1e-6, abs(g[i]) + abs(fd)))
    assert worst < 1e-5, worst
    # padding columns / rows carry no gradient
    W1g = M.unpack(g)["W1"]
    assert np.all(W1g[:, M.N_IN:] == 0)
    W4g = M.unpack(g)["W4"]
    assert np.all(W4g[M.N_OUT:] == 0)


def name_of(i):
    for name, (o, s) in M.OFF.items():
        if o <= i < o + s:
            return name
    raise IndexError(i)


def test_param_count_matches_library():
    from pelemp_b200.spray import learn_param_count
    assert learn_param_count() == M.N_PARAM == 9928


def test_quantised_forward_is_close_to_fp64():
    rng = np.random.default_rng(5)
    p = M.random_params(2)
    x = rng.standard_normal((200, M.N_IN))
    a, _ = M.forward(p, x, quant=False)
    b, _ = M.forward(p, x, quant=True)
    c = M.infer(p, x)
    scale = np.sqrt(np.mean(a * a))
    assert np.sqrt(np.mean((a - b) ** 2)) < 2e-2 * scale
    assert np.sqrt(np.mean((b - c) ** 2)) < 1e-2 * scale


def test_baseline_terms_and_nested_evaluation():
    """The library's host code of the targets' baseline (the code the kernels
    run): its terms equal the oracle's restatement exactly, and its FP32
    nested evaluation equals the dense polynomial within FP32 rounding."""
    from pelemp_b200.spray import learn_base_terms, learn_debug_base
    assert learn_base_terms() == M.BASE_TERMS
    rng = np.random.default_rng(5)
    for _ in range(20):
        xn = rng.standard_normal(M.N_IN).astype(np.float32)
        ell = np.float32(rng.uniform(0, 3))
        g = np.float32(rng.uniform(-1, 3))
        coef = rng.standard_normal(M.BASE_TERMS).astype(np.float32)
        feats, value = learn_debug_base(xn, ell, g, coef)
        want = M.base_features(xn.astype(np.float64), float(ell), float(g))[0]
        assert np.array_equal(feats, want)
        dense = float(want @ coef.astype(np.float64))
        assert abs(value - dense) <= 1e-6 * float(np.abs(want * coef).sum())


def test_baseline_solve_matches_numpy():
    """The library's host solve of the baseline fit, from normal equations in
    the accumulator layout of its GPU kernel, against numpy's ridge solve."""
    from pelemp_b200.spray import learn_debug_solve_baseline
    rng = np.random.default_rng(6)
    n = 20000
    xn = rng.standard_normal((n, M.N_IN))
    xn[:, 5] = 0.0   # a feature that never varies (one fuel) gets no weight
    ell = rng.uniform(0, 3, n)
    g = rng.uniform(-1, 3, n)
    F = M.base_features(xn, ell, g)
    true = rng.standard_normal((M.N_OUT, M.BASE_TERMS))
    true[:, 1 + len(M.BASE_Q) + 2] = 0.0
    Y = F @ true.T + 1e-3 * rng.standard_normal((n, M.N_OUT))
    coef = learn_debug_solve_baseline(M.normal_equations(F, Y))
    want = M.solve_baseline(F, Y)
    assert np.max(np.abs(coef - want)) <= 1e-5 * np.max(np.abs(want))
    assert np.max(np.abs(coef - true)) <= 1e-3
