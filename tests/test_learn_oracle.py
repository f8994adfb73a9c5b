"""CPU checks of the learned-weight oracle (oracle/hzgnn_oracle.c):
the loss gradient dL/domega against central finite differences, and the
network's backward pass against torch autograd of the same network (FP64,
BF16 rounding switched off in the oracle)."""
import numpy as np
import pytest

import oracle
from hazmath_b200 import problems as P

H = 32
OFF_WIN, OFF_BIN, LAYER, OFF_L0 = 0, 128, 3200, 160
L_U, L_V, L_C, L_W, L_B = 0, 1024, 1088, 1120, 3168
OFF_WO = OFF_L0 + 3 * LAYER
OFF_BO = OFF_WO + 32
NPARAM = OFF_BO + 1


@pytest.fixture(scope="module")
def hier(port):
    ia, ja, val = P.aniso2d_p1(22, 0.05, 0.5)
    prm = oracle.AMGParams(smoother=10, presmooth_iter=2, postsmooth_iter=2, coarse_dof=50)
    assert port.setup(ia, ja, val, prm) == 0
    assert port.num_levels() >= 3
    return ia, ja, val


def test_loss_gradient_finite_differences(port, hier):
    ia, ja, val = hier
    n = len(ia) - 1
    E = port.learn_errors(2, 7)
    om = np.float32(1.0 + 0.4 * np.random.default_rng(1).uniform(-1, 1, n))
    L, d = port.learn_loss_grad(om, E)
    assert 0 < L < 1
    for i in (0, n // 3, n // 2, n - 1):
        op, omn = om.copy(), om.copy()
        op[i] += np.float32(2e-3)
        omn[i] -= np.float32(2e-3)
        h = (float(op[i]) - float(omn[i])) / 2
        fd = (port.learn_loss_grad(op, E)[0] - port.learn_loss_grad(omn, E)[0]) / (2 * h)
        assert abs(fd - d[i]) <= 1e-4 * abs(d[i]) + 1e-10, (i, fd, d[i])


@pytest.mark.parametrize("ncyc", [1, 4])
def test_k_cycle_loss_gradient_finite_differences(port, hier, ncyc):
    ia, ja, val = hier
    n = len(ia) - 1
    E = port.learn_errors(2, 9, None, 0)          # independent of omega
    om = np.float32(1.0 + 0.3 * np.random.default_rng(2).uniform(-1, 1, n))
    L, d = port.learn_loss_grad(om, E, ncyc)
    for i in (1, n // 2, n - 2):
        op, omn = om.copy(), om.copy()
        op[i] += np.float32(2e-3)
        omn[i] -= np.float32(2e-3)
        h = (float(op[i]) - float(omn[i])) / 2
        fd = (port.learn_loss_grad(op, E, ncyc)[0] - port.learn_loss_grad(omn, E, ncyc)[0]) / (2 * h)
        assert abs(fd - d[i]) <= 1e-4 * abs(d[i]) + 1e-10, (i, fd, d[i])


def _objective(port, om, E):
    """The training objective log(||E^4 z||^2 / ||E^2 z||^2) and its gradient."""
    l4, d4 = port.learn_loss_grad(om, E, 4)
    l2, d2 = port.learn_loss_grad(om, E, 2)
    return np.log(l4 / l2), d4 / l4 - d2 / l2


@pytest.mark.parametrize("name", ["aniso", "lognormal3d"])
def test_training_objective_points_to_the_better_weight(port, name):
    """The objective's gradient matches finite differences along a uniform
    change of omega, and at omega = 1 it points where the measured two-cycle
    contraction of each cycle's own errors improves: smaller omega for a
    strongly anisotropic 2D operator, larger for 3D log-normal diffusion."""
    if name == "aniso":
        ia, ja, val = P.aniso2d_p1(40, 1e-3, 0.3)
    else:
        ia, ja, val = P.kuhn3d_p1(13, P.lognormal_field(13, 1.0, 4.0, 3))
    prm = oracle.AMGParams(smoother=10, presmooth_iter=2, postsmooth_iter=2, coarse_dof=100)
    assert port.setup(ia, ja, val, prm) == 0
    n = len(ia) - 1
    E = port.learn_errors(4, 5, None, 0)
    om = np.ones(n, np.float32)
    f, g = _objective(port, om, E)
    h = 1e-3
    fd = (_objective(port, om + np.float32(h), E)[0] - _objective(port, om - np.float32(h), E)[0]) / (2 * h)
    assert abs(fd - g.sum()) <= 1e-4 * abs(g.sum())
    # the measured contraction of each cycle's own errors, at omega = 1 -+ 0.3
    step = -0.3 if name == "aniso" else 0.3
    assert (g.sum() > 0) == (name == "aniso")
    def rho(w):
        o = np.full(n, w, np.float32)
        Eo = port.learn_errors(4, 5, o, 2)
        return port.learn_loss_grad(o, Eo, 2)[0] ** 0.25
    assert rho(1.0 + step) < rho(1.0)
    port.free()


def random_params(seed):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-0.3, 0.3, NPARAM).astype(np.float32)
    return p


def torch_network(ia, ja, val, p):
    torch = pytest.importorskip("torch")
    n = len(ia) - 1
    prm = torch.tensor(p.astype(np.float64), requires_grad=True)
    rows = np.repeat(np.arange(n), np.diff(ia))
    diag = np.zeros(n)
    l1 = np.zeros(n)
    off = np.zeros(n)
    mx = np.zeros(n)
    for i in range(n):
        sl = slice(ia[i], ia[i + 1])
        c, v = ja[sl], val[sl]
        diag[i] = v[c == i][0]
        l1[i] = np.abs(v).sum()
        off[i] = v[c != i].sum()
        mx[i] = np.abs(v[c != i]).max()
    x = torch.tensor(np.stack([diag / l1, off / l1, mx / l1, np.ones(n)], 1))
    m = ja != rows
    ri, cj, av = rows[m], ja[m], val[m]
    e0 = av / np.sqrt(np.abs(diag[ri] * diag[cj]))
    e1 = np.clip(0.5 * np.log(np.abs(diag[cj] / diag[ri])), -4, 4)
    e = torch.tensor(np.stack([e0, e1], 1))
    deg = torch.tensor(np.bincount(ri, minlength=n).astype(np.float64))
    W_in = prm[OFF_WIN:OFF_WIN + 128].view(32, 4)
    h = torch.relu(x @ W_in.T + prm[OFF_BIN:OFF_BIN + 32])
    ri_t, cj_t = torch.tensor(ri), torch.tensor(cj)
    for l in range(3):
        b0 = OFF_L0 + l * LAYER
        U = prm[b0 + L_U:b0 + L_U + 1024].view(32, 32)
        V = prm[b0 + L_V:b0 + L_V + 64].view(32, 2)
        c = prm[b0 + L_C:b0 + L_C + 32]
        W = prm[b0 + L_W:b0 + L_W + 2048].view(32, 64)
        b = prm[b0 + L_B:b0 + L_B + 32]
        Pm = h @ U.T
        msg = torch.relu(Pm[cj_t] + e @ V.T + c)
        M = torch.zeros(n, 32, dtype=torch.float64).index_add(0, ri_t, msg) / deg[:, None]
        y = torch.cat([h, M], 1) @ W.T + b
        h = torch.relu(y) + h
    z = h @ prm[OFF_WO:OFF_WO + 32] + prm[OFF_BO]
    return prm, 2 * torch.sigmoid(z)


def test_gnn_backward_matches_autograd(port):
    torch = pytest.importorskip("torch")
    ia, ja, val = P.aniso2d_p1(9, 0.1, 0.9)
    p = random_params(3)
    om = port.gnn_forward(ia, ja, val, p, rounding=False)
    prm, om_t = torch_network(ia, ja, val, p)
    np.testing.assert_allclose(om, om_t.detach().numpy(), rtol=1e-4, atol=1e-5)
    dom = np.random.default_rng(4).uniform(-1, 1, len(om)).astype(np.float32)
    g = port.gnn_backward(p, dom)
    (om_t * torch.tensor(dom.astype(np.float64))).sum().backward()
    gt = prm.grad.numpy()
    for name, sl in [("W_in", slice(0, 160)), ("layers", slice(160, OFF_WO)),
                     ("out", slice(OFF_WO, NPARAM))]:
        err = np.linalg.norm(g[sl] - gt[sl]) / np.linalg.norm(gt[sl])
        assert err < 1e-4, (name, err)
