"""The learned barostat's CPU oracle: BF16 rounding and the analytic gradient of the
network checked against finite differences (no GPU)."""
import numpy as np

from oracle import surrogate as sg


def test_bf16_rounding_is_round_to_nearest_even():
    one = np.float32(1.0)
    half_ulp = np.float32(2.0 ** -8)  # BF16 spacing at 1.0 is 2^-7
    cases = {
        float(one): 1.0,
        float(one + half_ulp): 1.0,                       # tie -> even (1.0)
        float(one + np.float32(3) * half_ulp): 1.015625,  # tie -> even (1 + 2^-6)
        float(one + half_ulp + np.float32(2.0 ** -20)): 1.0078125,  # above the tie
        -2.5: -2.5,
        0.0: 0.0,
    }
    got = sg.bf16_round(np.array(list(cases), np.float32))
    assert np.array_equal(got, np.array(list(cases.values()), np.float32))
    assert sg.bf16_round(np.float32(3.0e38)).dtype == np.float32


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(4)
    params = sg.random_parameters(seed=4).astype(np.float64)
    x = rng.normal(size=(24, 8))
    t = rng.normal(size=24) * 0.3
    loss, grad = sg.loss_and_gradients(params, x, t, bf16=False)
    picks = np.concatenate([rng.choice(np.arange(sg.W1, sg.B1), 6), rng.choice(np.arange(sg.B1, sg.W2), 3),
                            rng.choice(np.arange(sg.W2, sg.B2), 8), rng.choice(np.arange(sg.B2, sg.W3), 3),
                            rng.choice(np.arange(sg.W3, sg.B3), 4), [sg.B3]])
    eps = 1e-6
    for k in picks:
        up, dn = params.copy(), params.copy()
        up[k] += eps
        dn[k] -= eps
        fd = (sg.loss_and_gradients(up, x, t, bf16=False)[0] - sg.loss_and_gradients(dn, x, t, bf16=False)[0]) / (2 * eps)
        assert abs(fd - grad[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, grad[k])
    assert loss > 0


def test_bf16_forward_is_close_to_fp32():
    rng = np.random.default_rng(1)
    params = sg.random_parameters(seed=1)
    x = rng.normal(size=(16, 8))
    y16 = sg.forward(params, x, bf16=True)[0]
    y32 = sg.forward(params, x, bf16=False)[0]
    assert np.max(np.abs(y16 - y32)) < 0.05 * max(1.0, np.max(np.abs(y32)))
