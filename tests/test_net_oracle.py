"""The CPU oracle of the learned preconditioner network (oracle/net_oracle.py)
against finite differences of its own loss, in FP64 (no BF16 rounding): the
hand-derived backward pass that the GPU kernels restate must be the gradient
of the forward pass.  Parameters are sampled from every layer; relative
agreement <= 1e-4 where the gradient is not negligible."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), ".."))
from oracle import net_oracle as N  # noqa: E402


def random_params(rng):
    w = np.zeros(N.n_params())
    o = 0
    for ci, co, k in N.LAYERS:
        nw = co * ci * k ** 3
        w[o:o + nw] = rng.standard_normal(nw) * np.sqrt(2.0 / (ci * k ** 3))
        o += nw
        w[o:o + co] = 0.1 * rng.standard_normal(co)
        o += co
    return w


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159265, 0.0], dtype=np.float32)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even -> 1.0
    assert list(N.bf16(x)) == [1.0, 1.0, np.float32(1.0078125), np.float32(-3.140625), 0.0]


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    w = random_params(rng)
    xin = rng.standard_normal((4, 8, 8, 8))
    t = rng.standard_normal((3, 8, 8, 8))
    mask = rng.uniform(size=t.shape) < 0.8
    loss, g, _ = N.loss_and_grads(w, xin, t, mask, bf=False)
    assert loss > 0
    offs, o = [], 0
    for ci, co, k in N.LAYERS:
        offs.append(o)
        o += co * ci * k ** 3 + co
    checked = 0
    for li, (ci, co, k) in enumerate(N.LAYERS):
        # the centre tap of a few (co, ci) pairs and one bias of every layer
        cand = [offs[li] + (a * ci + b) * k ** 3 + (k ** 3) // 2
                for a, b in [(0, 0), (co - 1, ci - 1), (co // 2, ci // 2)]]
        cand.append(offs[li] + co * ci * k ** 3 + co // 2)
        for i in cand:
            h = 1e-5
            wp, wm = w.copy(), w.copy()
            wp[i] += h
            wm[i] -= h
            fd = (N.loss_and_grads(wp, xin, t, mask, bf=False)[0] -
                  N.loss_and_grads(wm, xin, t, mask, bf=False)[0]) / (2 * h)
            if abs(fd) < 1e-9 and abs(g[i]) < 1e-9:
                continue
            assert abs(g[i] - fd) <= 1e-4 * max(abs(fd), 1e-6), (li, i, g[i], fd)
            checked += 1
    assert checked >= 20
