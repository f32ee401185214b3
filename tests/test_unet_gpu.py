"""The learned U-Net preconditioner's tcgen05 kernels against the oracle's
numpy restatement (oracle/unet.py): every layer of the forward pass, the
parameter gradients of the backward pass, the Adam step, and that training
on residual -> error pairs lowers the loss.

Tolerances: activations are stored in bfloat16, so a layer recomputed by the
oracle from the GPU's own input may differ by an ulp of bfloat16 where the
FP32 (GPU) and FP64 (oracle) sums round differently (2^-7 of the layer's
largest value); gradients flow through bfloat16 tensors, so they are
compared in relative L2 (5e-2) and direction (cosine >= 0.998)."""
import numpy as np
import pytest

from oracle import unet as ou

pytestmark = pytest.mark.gpu

GRIDS = [(128, 16, 8), (256, 8, 8)]


def Net(shape, seed=0):
    from aeolus_b200.unet import UNet
    return UNet(shape, seed=seed)


def problem(shape, seed):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    mask = (rng.random((nz, ny, nx)) > 0.1).astype(np.float32)
    r = rng.standard_normal((nz, ny, nx)) * mask
    e = rng.standard_normal((nz, ny, nx)) * mask
    return r, e, mask


def params_dict(net):
    from aeolus_b200.unet import split_params
    return split_params(net.params())


@pytest.mark.parametrize("shape", GRIDS)
def test_forward_layers_match_the_oracle(shape):
    net = Net(shape, seed=3)
    r, e, mask = problem(shape, 1)
    net.set_mask(mask)
    net.set_out_scale(2.5)
    z = net.apply(r)
    P = params_dict(net)
    A = {k: net.activation(k).astype(np.float64) for k in ("x", "e1a", "e1", "p1", "e2a", "e2", "p2", "e3a", "e3",
                                                           "u2", "d2", "u1", "d1")}
    assert np.array_equal(ou.bf16(A["x"]), A["x"])
    np.testing.assert_allclose(A["x"], ou.inputs(r, mask), rtol=0, atol=2 ** -7 * np.abs(A["x"]).max())

    def close(got, want, name):
        tol = 2 ** -7 * max(np.abs(want).max(), 1e-30)
        bad = np.abs(got - want) > tol
        assert bad.mean() < 1e-3 and np.abs(got - want).max() <= 4 * tol, (name, np.abs(got - want).max(), tol)

    def layer(name, inp, relu=True):
        W, b = P[name]
        y = ou.conv(inp, ou.bf16(W), b)
        return np.maximum(y, 0) if relu else y

    close(A["e1a"], ou.bf16(layer("e1a", A["x"])), "e1a")
    close(A["e1"], ou.bf16(layer("e1", A["e1a"])), "e1")
    close(A["p1"], ou.bf16(ou.pool(A["e1"])), "p1")
    close(A["e2a"], ou.bf16(layer("e2a", A["p1"])), "e2a")
    close(A["e2"], ou.bf16(layer("e2", A["e2a"])), "e2")
    close(A["p2"], ou.bf16(ou.pool(A["e2"])), "p2")
    close(A["e3a"], ou.bf16(layer("e3a", A["p2"])), "e3a")
    close(A["e3"], ou.bf16(layer("e3", A["e3a"])), "e3")
    close(A["u2"], ou.bf16(ou.up(A["e3"]) + A["e2"]), "u2")
    close(A["d2"], ou.bf16(layer("d2", A["u2"])), "d2")
    close(A["u1"], ou.bf16(ou.up(A["d2"]) + A["e1"]), "u1")
    close(A["d1"], ou.bf16(layer("d1", A["u1"])), "d1")
    s = ou.input_scale(r, mask)
    out = layer("out", A["d1"], relu=False)[..., 0] * (2.5 / s) * mask
    np.testing.assert_allclose(z, out, rtol=1e-4, atol=1e-5 * np.abs(out).max())


@pytest.mark.parametrize("shape", GRIDS)
def test_gradients_match_the_oracle(shape):
    net = Net(shape, seed=5)
    r, e, mask = problem(shape, 2)
    net.set_mask(mask)
    net.set_out_scale(3.0)
    loss = net.gradients(r, e)
    from aeolus_b200.unet import split_params
    G = split_params(net.grads())
    P = params_dict(net)
    x = ou.inputs(r, mask)
    A = ou.forward(P, x)
    s = ou.input_scale(r, mask)
    L, gout = ou.loss_and_grad_out(A["out"], e, mask)
    assert abs(loss - L) <= 2e-2 * L
    Gr = ou.backward(P, A, gout)
    for name, _, _ in ou.LAYERS:
        wscale = np.linalg.norm(Gr[name][0])
        for q, what in ((0, "W"), (1, "b")):
            got, want = G[name][q].astype(np.float64).ravel(), Gr[name][q].ravel()
            nw = np.linalg.norm(want)
            if nw <= 1e-3 * wscale:
                # a gradient that vanishes by construction (the output bias:
                # the loss ignores constant shifts of the output)
                assert np.linalg.norm(got) <= 1e-2 * wscale, (name, what, np.linalg.norm(got), wscale)
                continue
            relerr = np.linalg.norm(got - want) / nw
            cos = got @ want / (np.linalg.norm(got) * nw)
            assert relerr < 5e-2 and cos > 0.998, (name, what, relerr, cos)


def test_adam_step_matches_the_oracle():
    shape = (128, 16, 8)
    net = Net(shape, seed=7)
    r, e, mask = problem(shape, 3)
    net.set_mask(mask)
    net.set_out_scale(1.0)
    from aeolus_b200.unet import split_params
    p0 = net.params()
    net.gradients(r, e)
    g = net.grads()
    net.train_step(r, e, lr=1e-3)
    p1 = net.params()
    P0, G = split_params(p0), split_params(g)
    Mo = {n: [np.zeros_like(P0[n][0], dtype=np.float64), np.zeros_like(P0[n][1], dtype=np.float64)] for n, _, _ in ou.LAYERS}
    Vo = {n: [np.zeros_like(P0[n][0], dtype=np.float64), np.zeros_like(P0[n][1], dtype=np.float64)] for n, _, _ in ou.LAYERS}
    Pn = ou.adam(P0, {n: (G[n][0].astype(np.float64), G[n][1].astype(np.float64)) for n, _, _ in ou.LAYERS}, Mo, Vo, 1,
                 lr=1e-3)
    from aeolus_b200.unet import join_params
    ref = join_params(Pn)
    big = np.abs(g) > 1e-6 * np.abs(g).max()
    assert np.abs(p1 - ref)[big].max() < 2e-5          # step of lr with the gradient's sign
    assert np.abs(p1 - p0)[~big].max() <= 1.01e-3


def test_training_lowers_the_loss_on_poisson_pairs():
    from aeolus_b200.multigrid import MGPreconditionedCG
    shape = (128, 16, 8)
    nx, ny, nz = shape
    mg = MGPreconditionedCG(shape, (1.0, 1.0, 1.0), bc=("periodic", "periodic", "neumann"), tol=1e-10)
    rng = np.random.default_rng(11)
    pairs = []
    for _ in range(8):
        r = rng.standard_normal((nz, ny, nx))
        r -= r.mean()
        e, st = mg.solve(r)
        assert st["status"] == "converged"
        pairs.append((r, e))
    from aeolus_b200.unet import UNet, error_scale
    net = UNet(shape, seed=1)
    net.set_mask(np.ones((nz, ny, nx), dtype=np.float32))
    net.set_out_scale(error_scale(pairs))
    first = np.mean([net.gradients(r, e) for r, e in pairs])
    # the learning rate decays geometrically as in train_streaming: per-pair
    # Adam steps at a constant rate leave the last epoch's loss wandering, and
    # the weight-gradient sums are FP32 atomics (not bit-reproducible)
    nstep = 12 * len(pairs)
    for q in range(nstep):
        r, e = pairs[q % len(pairs)]
        net.train_step(r, e, lr=2e-3 * (0.05 ** (q / (nstep - 1))))
    last = np.mean([net.gradients(r, e) for r, e in pairs])
    assert last < 0.7 * first, (first, last)
