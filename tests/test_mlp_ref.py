"""The CPU reference network (the gradient oracle of the GPU kernels) is itself checked:
its FP64 backward pass against central finite differences of its forward pass."""
import numpy as np

import mlp_ref


def test_reference_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = np.zeros(sum(n for _, n in mlp_ref.SIZES))
    P = mlp_ref.unpack(p)
    P["W1"][:84] = rng.normal(0, 0.3, (84, 128))
    P["W2"] = rng.normal(0, 0.1, (128, 128))
    P["W3"] = rng.normal(0, 0.1, (128, 128))
    P["W4"][:, :2] = rng.normal(0, 0.1, (128, 2))
    for b in ("b1", "b2", "b3"):
        P[b] = rng.normal(0, 0.1, 128)
    P["b4"][:2] = rng.normal(0, 0.1, 2)
    p = mlp_ref.pack(P)
    X = rng.normal(size=(7, 84)).astype(np.float32)
    T = rng.normal(size=(7, 2))
    xm, xs = np.zeros(96, np.float32), np.ones(96, np.float32)
    _, loss, g = mlp_ref.forward_backward(p, xm, xs, X, T, bf=False)
    offs = np.cumsum([0] + [n for _, n in mlp_ref.SIZES])
    picks = [offs[0] + 5, offs[0] + 130, offs[1] + 3, offs[2] + 777, offs[3] + 9, offs[4] + 1234, offs[5] + 100,
             offs[6] + 8 * 17 + 1, offs[7] + 1]
    for i in picks:
        e = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += e
        pm[i] -= e
        fd = (mlp_ref.forward_backward(pp, xm, xs, X, T, bf=False)[1] -
              mlp_ref.forward_backward(pm, xm, xs, X, T, bf=False)[1]) / (2 * e)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5], dtype=np.float32)
    r = mlp_ref.bf16(x)
    # 1 + 2^-8 is the tie between 1 and 1 + 2^-7: ties go to the even significand (1.0)
    assert list(r) == [1.0, 1.0, 1.0, 1.0078125, -2.5]
