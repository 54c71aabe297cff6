"""The CPU oracle of the learned preconditioner (oracle/nn_oracle.py): its
hand-written backward pass against central finite differences of its own FP64
forward pass (the network has no reference counterpart)."""
import numpy as np

import oracle.nn_oracle as NN


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    grid = (6, 5, 4)
    N = 120
    P = rng.normal(0, 0.3, NN.n_params())
    R = rng.normal(size=(2, N))
    V = rng.normal(size=N)
    Y = rng.normal(size=(2, N))
    loss, g = NN.loss_and_grad(P, grid, R, V, 2.0, Y, exact=True)
    # one weight and one bias of every layer, plus random indices
    offs = [0, 864, 880, 7792, 7808, 14720, 14736, 15168]
    idx = sorted(set(offs + list(rng.integers(0, NN.n_params(), 12))))
    h = 1e-6
    for i in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        fd = (NN.loss_and_grad(Pp, grid, R, V, 2.0, Y, exact=True)[0] -
              NN.loss_and_grad(Pm, grid, R, V, 2.0, Y, exact=True)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_oracle_zero_last_layer_gives_zero_correction():
    rng = np.random.default_rng(4)
    P = rng.normal(0, 0.3, NN.n_params())
    P[-(16 * 27 + 1):] = 0.0
    out = NN.apply(P, (4, 4, 4), rng.normal(size=(1, 64)), rng.normal(size=64), 1.0)
    assert np.all(out == 0.0)
