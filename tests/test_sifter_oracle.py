"""The sifter's CPU oracle (tests/sifter_oracle.py) against finite differences of its own loss: the
backward formulas the GPU kernels implement are the gradient of the mean binary cross-entropy."""

import numpy as np

import sifter_oracle as SO


def test_backward_formulas_match_finite_differences():
    rng = np.random.default_rng(0)
    n = 12
    p = np.concatenate([rng.normal(0, np.sqrt(2.0 / 1728), 256 * 1728), rng.normal(0, 0.1, 256),
                        rng.normal(0, np.sqrt(2.0 / 256), 128 * 256), rng.normal(0, 0.1, 128),
                        rng.normal(0, np.sqrt(2.0 / 128), 128), [0.05]])
    x = rng.normal(0, 1.0, (n, 1728))
    y = (rng.random(n) < 0.5).astype(np.float64)
    _, g = SO.gradients(p, x, y, emulate=False)
    offs = np.cumsum([0] + [int(np.prod(s)) for s in SO.SHAPES])
    for blk in range(6):
        idx = rng.integers(offs[blk], offs[blk + 1], 6)
        for i in idx:
            h = 1e-6
            pp, pm = p.copy(), p.copy()
            pp[i] += h
            pm[i] -= h
            fd = (SO.loss(pp, x, y) - SO.loss(pm, x, y)) / (2 * h)
            assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (blk, i, fd, g[i])


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.0e-3, 65504.0], dtype=np.float32)
    r = SO.bf16(v)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties to even gives 1
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] + 3.0e-3) < 2e-5 and r[4] == 65536.0
