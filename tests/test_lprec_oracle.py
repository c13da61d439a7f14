"""The oracle's restatement of the learned pressure preconditioner, pinned
against PyTorch autograd (an independent implementation of the same dilated
3^3 convolutions, run here in FP64 on the CPU): forward output, the A-norm
training loss of M(r) = N(r) + D^-1 r and the weight gradient.  The network
has no reference counterpart, so torch is its pin."""
import numpy as np
import pytest

from oracle import oracle as O


def _torch_net(T, typ, r, ev, w, dil):
    import torch
    nw = w.size
    offs = [0, 27 * 3 * 16, 27 * 3 * 16 + 27 * 256, 27 * 3 * 16 + 2 * 27 * 256, nw]
    cin, cout = [3, 16, 16, 16], [16, 16, 16, 1]
    W = torch.tensor(w, dtype=torch.float64, requires_grad=True)

    def tw(l):  # [tap = kz,ky,kx][ci][co] -> torch [co][ci][kz][ky][kx]
        return W[offs[l]:offs[l + 1]].reshape(3, 3, 3, cin[l], cout[l]).permute(4, 3, 0, 1, 2)

    t = torch.tensor(typ.astype(np.int64))
    fl, so = (t == 1).double(), (t == 2).double()
    rt = torch.tensor(r, dtype=torch.float64) * fl
    s = torch.sqrt(torch.sum(rt ** 2) / fl.sum())
    def f(x):
        h = torch.stack([x, fl, so])[None]
        for l in range(4):
            h = torch.nn.functional.conv3d(h, tw(l), padding=dil[l], dilation=dil[l])
            if l < 3:
                h = torch.relu(h)
        return h[0, 0]

    z = (f(rt / s) - f(torch.zeros_like(rt))) * s * fl
    k = torch.zeros(1, 1, 3, 3, 3, dtype=torch.float64)
    for (a, b, c) in ((0, 1, 1), (2, 1, 1), (1, 0, 1), (1, 2, 1), (1, 1, 0), (1, 1, 2)):
        k[0, 0, a, b, c] = 1.0
    d = torch.nn.functional.conv3d((t != 2).double()[None, None], k, padding=1)[0, 0]
    dinv = torch.where(fl > 0, 1.0 / d.clamp(min=1.0), torch.zeros_like(d))
    m = (z + dinv * rt) * fl
    Am = (d * m - torch.nn.functional.conv3d(m[None, None], k, padding=1)[0, 0]) * fl
    et = torch.tensor(ev, dtype=torch.float64) * fl
    loss = (torch.sum(m * Am) - 2.0 * torch.sum(m * rt)) / torch.sum(et * rt) + 1.0
    loss.backward()
    return z.detach().numpy().ravel(), float(loss.detach()), W.grad.numpy()


@pytest.mark.parametrize("shape,dil", [((16, 24, 8), (1, 2, 4, 1)), ((8, 8, 16), (1, 1, 1, 1))])
def test_lp_oracle_vs_torch_autograd(shape, dil):
    torch = pytest.importorskip("torch")
    nx, ny, nz = shape
    rng = np.random.default_rng(3)
    typ = rng.choice([0, 1, 1, 1, 2], size=(nz, ny, nx)).astype(np.uint8)
    r = rng.standard_normal((nz, ny, nx)).astype(np.float32)
    ev = (r + 0.5 * rng.standard_normal((nz, ny, nx))).astype(np.float32)  # any e with e.r > 0 normalises
    w = (rng.standard_normal(O.lib().orc_lp_num_weights()) * 0.2).astype(np.float32)
    loss, z, g = O.lp_loss_grad(typ, r, ev, w, shape, dil=dil, round_bf16=False)
    zt, lt, gt = _torch_net(torch, typ, r, ev, w, dil)
    # the oracle keeps FP32 inputs and activations, torch FP64: 1e-6 bounds that
    assert np.max(np.abs(z - zt)) <= 1e-6 * np.max(np.abs(zt))
    assert abs(loss - lt) <= 1e-6 * abs(lt)
    assert np.linalg.norm(g - gt) <= 1e-6 * np.linalg.norm(gt)


def test_lp_forward_is_zero_off_fluid_and_scale_free():
    rng = np.random.default_rng(5)
    shape = (8, 16, 8)
    typ = rng.choice([0, 1, 2], size=shape[::-1]).astype(np.uint8)
    r = rng.standard_normal(shape[::-1]).astype(np.float32)
    w = (rng.standard_normal(O.lib().orc_lp_num_weights()) * 0.2).astype(np.float32)
    z, inv_s = O.lp_forward(typ, r, w, shape)
    assert np.all(z[typ.ravel() != 1] == 0.0)
    fl = typ.ravel() == 1
    assert abs(inv_s - 1.0 / np.sqrt(np.mean(r.ravel()[fl].astype(np.float64) ** 2))) < 1e-6 * inv_s
    # N is applied to r / rms(r) and scaled back: z(4 r) = 4 z(r) (a power of two keeps every rounding)
    z4, _ = O.lp_forward(typ, 4.0 * r, w, shape)
    assert np.array_equal(z4, 4.0 * z)


def centre_chain_weights(a):
    """Weights whose only path is the centre tap, channel 0 -> 0 -> 0 -> 0 -> 0,
    with gain a in layer 0 and 1 elsewhere: z = bf16(a) r on fluid cells."""
    nw = O.lib().orc_lp_num_weights()
    offs = [0, 27 * 3 * 16, 27 * 3 * 16 + 27 * 256, 27 * 3 * 16 + 2 * 27 * 256]
    w = np.zeros(nw, np.float32)
    w[offs[0] + 13 * 3 * 16] = a
    w[offs[1] + 13 * 16 * 16] = 1.0
    w[offs[2] + 13 * 16 * 16] = 1.0
    w[offs[3] + 13 * 16] = 1.0
    return w


@pytest.mark.parametrize("a,expect", [(1 + 2.0 ** -9, 1.0), (1 + 3 * 2.0 ** -9, 1 + 2.0 ** -7),
                                      (1 + 2.0 ** -8, 1.0), (1 + 3 * 2.0 ** -8, 1 + 2.0 ** -6)])
def test_bf16_rounding_is_nearest_even(a, expect):
    # below half, above half, and the two ties (to the even significand)
    shape = (8, 8, 8)
    typ = np.ones(shape, np.uint8)
    r = np.ones(shape, np.float32)
    z, inv_s = O.lp_forward(typ, r, centre_chain_weights(a), shape, round_bf16=True)
    assert inv_s == 1.0
    assert np.all(z == np.float32(expect))
    z, _ = O.lp_forward(typ, r, centre_chain_weights(a), shape, round_bf16=False)
    assert np.all(z == np.float32(a))
