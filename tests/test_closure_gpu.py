"""The learned closure on a B200: the tensor-core CNN against the CPU oracle
(oracle/closure_oracle.py), the box filter, training, and the coupling into the solver.

The oracle rounds to BF16 where the GPU does (inputs, weights, hidden activations, dZ before
the input-gradient product) and sums in float64; the GPU sums in FP32 and evaluates GELU with
tanhf. A hidden activation that lands next to a BF16 rounding boundary can round the other
way, so the bars are relative: the output within 1e-2 of its largest magnitude, every
gradient within 3e-2 in the relative L2 norm, the loss within 1e-3.
"""
import numpy as np
import pytest

from conftest import load_oracle_module

pytestmark = pytest.mark.gpu

co = load_oracle_module("closure_oracle")
SCALES = ((2.0, 1.5, 1.2, 0.3), 0.3)


def _sample(Ny, Nx, seed):
    rng = np.random.default_rng(seed)
    y = np.linspace(-1, 1, Ny)[:, None]
    x = np.arange(Nx)[None, :] * 2 * np.pi / Nx
    w = 3 * y + 0.5 * np.sin(3 * x + 2 * y) + 0.1 * rng.standard_normal((Ny, Nx))
    psi = 1.5 * y - 0.5 * y ** 3 + 0.05 * np.cos(2 * x) * (1 - y ** 2)
    u = 1.5 * (1 - y ** 2) + 0.1 * rng.standard_normal((Ny, Nx))
    v = 0.1 * np.sin(2 * x) * (1 - y ** 2) + 0.01 * rng.standard_normal((Ny, Nx))
    tau = 0.2 * np.sin(x + 3 * y) * (1 - y ** 2) + 0.02 * rng.standard_normal((Ny, Nx))
    return [np.ascontiguousarray(a * np.ones((Ny, Nx))) for a in (w, psi, u, v, tau)]


def _net(nse, Nx, Ny, H, seed, max_batch=1):
    y = np.linspace(-1, 1, Ny)
    net = nse.Cnn(Nx, Ny, y, H, max_batch)
    net.init_params(seed, last_gain=0.5)
    net.set_scales(*SCALES)
    return net, y


def _dev(torch, a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("Nx,Ny,H", [(32, 17, 32), (64, 33, 16), (256, 129, 32)])
def test_forward_matches_oracle(nse, cuda, Nx, Ny, H):
    torch = cuda
    net, y = _net(nse, Nx, Ny, H, 3)
    w, psi, u, v, _ = _sample(Ny, Nx, 3)
    out = torch.zeros((Ny, Nx), dtype=torch.float64, device="cuda")
    net.forward(_dev(torch, w), _dev(torch, psi), _dev(torch, u), _dev(torch, v), out)
    got = out.cpu().numpy()
    ref = co.predict(net.params(), w, psi, u, v, y, SCALES, bf=True)
    assert np.abs(got - ref).max() <= 1e-2 * np.abs(ref).max()
    assert np.all(got[0] == 0) and np.all(got[-1] == 0)


@pytest.mark.parametrize("Nx,Ny,H,idx", [(32, 17, 32, (0,)), (64, 33, 32, (2, 0, 3))])
def test_gradients_match_oracle(nse, cuda, Nx, Ny, H, idx):
    torch = cuda
    net, y = _net(nse, Nx, Ny, H, 5, max_batch=len(idx))
    S = [_sample(Ny, Nx, 10 + s) for s in range(4)]
    stack = [_dev(torch, np.stack([smp[f] for smp in S])) for f in range(5)]
    loss = net.gradients(*stack, idx=idx)
    ref_loss, ref_grads = co.loss_and_grads(net.params(), [S[i] for i in idx], y, SCALES, bf=True)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss, (loss, ref_loss)
    for layer in range(4):
        gw, gb = net.get_grads(layer)
        assert _rel(gw, ref_grads[layer][0]) < 3e-2, (layer, _rel(gw, ref_grads[layer][0]))
        assert _rel(gb, ref_grads[layer][1]) < 3e-2, (layer, _rel(gb, ref_grads[layer][1]))


def test_training_reduces_loss(nse, cuda):
    torch = cuda
    Nx, Ny = 64, 33
    teacher, y = _net(nse, Nx, Ny, 16, 11)
    net, _ = _net(nse, Nx, Ny, 16, 12, max_batch=2)
    S = [_sample(Ny, Nx, 20 + s) for s in range(2)]
    fields = [_dev(torch, np.stack([smp[f] for smp in S])) for f in range(4)]
    target = torch.zeros((2, Ny, Nx), dtype=torch.float64, device="cuda")
    for s in range(2):
        teacher.forward(*[f[s] for f in fields], target[s])
    first = net.gradients(*fields, target, idx=(0, 1))
    for _ in range(300):
        net.train_step(*fields, target, lr=3e-3, idx=(0, 1), want_loss=False)
    last = net.gradients(*fields, target, idx=(0, 1))
    assert np.isfinite(last) and last < 0.1 * first, (first, last)


def test_box_filter_matches_oracle(nse, cuda):
    torch = cuda
    rng = np.random.default_rng(4)
    f = rng.standard_normal((65, 128))
    coarse = torch.zeros((9, 16), dtype=torch.float64, device="cuda")
    nse.box_filter(_dev(torch, f), 128, 65, coarse, 16, 9)
    assert np.allclose(coarse.cpu().numpy(), co.box_filter(f, 16, 9), rtol=1e-13, atol=1e-14)


def test_zero_model_leaves_the_solver_unchanged(nse, cuda):
    cfg = dict(Nx=256, Ny=129, Lx=2 * np.pi, stretch=1, beta=2.0, Ub=1.0, Reb=5000.0, F0=0.05, nforce=8,
               lin_drag=1e-3, adapt=1, cfl=0.5)
    a, b = nse.Solver(**cfg), nse.Solver(**cfg)
    w0 = _sample(129, 256, 8)[0]
    a.set_omega(w0)
    b.set_omega(w0)
    net = nse.Cnn(256, 129, b.metric(0), 32, 1)
    for layer in range(4):
        ci, co_ = net.shape(layer)
        net.set_params(layer, np.zeros((co_, 9, ci), np.float32), np.zeros(co_, np.float32))
    net.set_scales(*SCALES)
    b.set_closure(net)
    a.step(20, use_graph=True)
    b.step(20, use_graph=True)
    assert np.array_equal(a.fields()[0], b.fields()[0])
    # a nonzero model changes the interior and keeps the run finite
    net.init_params(1)
    net.set_scales((5.0, 2.0, 1.5, 0.3), 0.05)
    b.set_closure(net)
    a.step(20, use_graph=True)
    b.step(20, use_graph=True)
    wa, wb = a.fields()[0], b.fields()[0]
    assert np.all(np.isfinite(wb)) and not np.array_equal(wa, wb)
