"""The learned prior's tcgen05 convolutions (csrc/conv.cu) against the FP64
oracle (oracle.conv3x3*), through the C ABI.

The kernels multiply BF16 operands exactly and accumulate in FP32, so with the
oracle fed the same BF16-rounded operands: FP32 outputs agree to relative L2
<= 1e-5; BF16 outputs agree with the oracle's result rounded to BF16 except
where the two sides of a rounding boundary differ (<= 1e-3 relative L2, about
one BF16 ulp on a few elements); the full network's output, whose hidden
activations are BF16, agrees to 1e-4; its gradients, which pass
through BF16 activations and BF16 output gradients, agree to 2e-2."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _bf(rng, *shape, scale=1.0):
    from oracle import oracle as O
    return O.bf16_round((rng.standard_normal(shape) * scale).astype(np.float32))


def _kern():
    from reconnet_b200.learned_prior import ConvKernels
    return ConvKernels("cuda")


@pytest.mark.parametrize("cin,cout", [(32, 32), (8, 32), (32, 1)])
# widths of 8k, 2k and odd pixels: 8, 2 and 1 pixels per TMA box row
@pytest.mark.parametrize("hw", [(5, 200), (3, 128), (4, 131), (3, 150)])
def test_conv_forward_fp32_matches_oracle(cin, cout, hw, rng):
    import torch
    from oracle import oracle as O
    from reconnet_b200.learned_prior import pack_weights, to_blocked
    H, W = hw
    x = _bf(rng, 2, cin, H, W)
    w = _bf(rng, cout, 3, 3, cin, scale=0.2)
    b = rng.standard_normal(cout).astype(np.float32)
    k = _kern()
    xb = to_blocked(torch.from_numpy(x).float().cuda())
    got = k.conv(xb, pack_weights(torch.from_numpy(w).float().cuda()), torch.from_numpy(b).cuda(), cin, cout, 3)
    k.check()
    assert rel_l2(got.cpu().numpy(), O.conv3x3(x, w, b)) <= 1e-5


def test_conv_relu_bf16_and_residual_modes(rng):
    import torch
    from oracle import oracle as O
    from reconnet_b200.learned_prior import from_blocked, pack_weights, to_blocked
    k = _kern()
    x = _bf(rng, 2, 32, 4, 160)
    w = _bf(rng, 32, 3, 3, 32, scale=0.1)
    b = (rng.standard_normal(32) * 0.1).astype(np.float32)
    got = from_blocked(k.conv(to_blocked(torch.from_numpy(x).float().cuda()), pack_weights(torch.from_numpy(w).float().cuda()),
                              torch.from_numpy(b).cuda(), 32, 32, 0)).cpu().numpy()
    ref = O.bf16_round(np.maximum(O.conv3x3(x, w, b), 0).astype(np.float32))
    assert rel_l2(got, ref) <= 1e-3
    # one output channel plus the FP32 residual
    w1 = _bf(rng, 1, 3, 3, 32, scale=0.1)
    res = rng.random((2, 4, 160)).astype(np.float32)
    got = k.conv(to_blocked(torch.from_numpy(x).float().cuda()), pack_weights(torch.from_numpy(w1).float().cuda()),
                 torch.tensor([0.25], device="cuda"), 32, 1, 1, aux=torch.from_numpy(res).cuda()).cpu().numpy()
    assert rel_l2(got, O.conv3x3(x, w1, [0.25])[:, 0] + res) <= 1e-5
    k.check()


def test_conv_input_gradient_with_relu_mask(rng):
    import torch
    from oracle import oracle as O
    from reconnet_b200.learned_prior import from_blocked, pack_dgrad_weights, to_blocked
    k = _kern()
    dy = _bf(rng, 2, 32, 4, 140)
    w = _bf(rng, 32, 3, 3, 32, scale=0.1)
    act = O.bf16_round(np.maximum(rng.standard_normal((2, 32, 4, 140)), 0).astype(np.float32))
    got = from_blocked(k.conv(to_blocked(torch.from_numpy(dy).float().cuda()),
                              pack_dgrad_weights(torch.from_numpy(w).float().cuda()), None, 32, 32, 2,
                              aux=to_blocked(torch.from_numpy(act).float().cuda()))).cpu().numpy()
    ref = O.bf16_round((O.conv3x3_dgrad(dy, w) * (act > 0)).astype(np.float32))
    assert rel_l2(got, ref) <= 1e-3
    # the same through an 8-channel input (the last layer's gradient)
    w5 = _bf(rng, 1, 3, 3, 32, scale=0.1)
    dy5 = np.zeros((2, 8, 4, 140))
    dy5[:, 0] = _bf(rng, 2, 4, 140)
    got = from_blocked(k.conv(to_blocked(torch.from_numpy(dy5).float().cuda()),
                              pack_dgrad_weights(torch.from_numpy(w5).float().cuda()), None, 8, 32, 2,
                              aux=to_blocked(torch.from_numpy(act).float().cuda()))).cpu().numpy()
    ref = O.bf16_round((O.conv3x3_dgrad(dy5[:, :1], w5) * (act > 0)).astype(np.float32))
    assert rel_l2(got, ref) <= 1e-3
    k.check()


@pytest.mark.parametrize("cin,cout", [(32, 32), (8, 32), (32, 8)])
def test_conv_weight_gradient_matches_oracle(cin, cout, rng):
    import torch
    from oracle import oracle as O
    from reconnet_b200.learned_prior import to_blocked, unpack_wgrad
    k = _kern()
    x = _bf(rng, 3, cin, 7, 300)
    dy = _bf(rng, 3, cout, 7, 300)
    g = k.wgrad(to_blocked(torch.from_numpy(x).float().cuda()), to_blocked(torch.from_numpy(dy).float().cuda()), cin, cout)
    k.check()
    dw, db = unpack_wgrad(g, cin, cout)
    rdw, rdb = O.conv3x3_wgrad(x, dy)
    assert rel_l2(dw.cpu().numpy(), rdw) <= 1e-5
    assert rel_l2(db.cpu().numpy(), rdb) <= 1e-5


def test_network_gradients_match_oracle_chain(rng):
    """PriorCNN.backward against the same network in FP64 with BF16 rounding
    at the points where the kernels store BF16 (activations, output gradient)."""
    import torch
    from oracle import oracle as O
    from reconnet_b200.learned_prior import PriorCNN
    net = PriorCNN("cuda", seed=3)
    u = rng.random((2, 6, 150)).astype(np.float32)
    t = rng.random((2, 6, 150)).astype(np.float32)
    out, acts = net.forward(torch.from_numpy(u).cuda(), keep=True)
    d_out = (2.0 / u.size) * (out - torch.from_numpy(t).cuda())
    dws, dbs = net.backward(acts, d_out.contiguous())
    W = [O.bf16_round(w.cpu().numpy()) for w in net.w]
    B = [b.cpu().numpy().astype(np.float64) for b in net.b]
    a = [O.bf16_round(u)[:, None]]
    for li in range(4):
        a.append(O.bf16_round(np.maximum(O.conv3x3(a[-1], W[li], B[li]), 0).astype(np.float32)))
    ref_out = O.conv3x3(a[4], W[4], B[4])[:, 0] + u
    # the hidden activations are rounded to BF16 between layers, so an FP32
    # accumulation that lands on the other side of a rounding boundary from
    # the FP64 sum moves that activation by one BF16 ulp: 1e-4, not 1e-5
    assert rel_l2(out.cpu().numpy(), ref_out) <= 1e-4
    d = O.bf16_round(((2.0 / u.size) * (ref_out - t)).astype(np.float32))[:, None]
    for li in (4, 3, 2, 1, 0):
        rdw, rdb = O.conv3x3_wgrad(a[li], d)
        assert rel_l2(dws[li].cpu().numpy(), rdw) <= 2e-2, li
        assert rel_l2(dbs[li].cpu().numpy(), rdb) <= 2e-2, li
        if li:
            d = O.bf16_round((O.conv3x3_dgrad(d, W[li]) * (a[li] > 0)).astype(np.float32))


def test_prior_training_reduces_loss_and_beats_identity(rng):
    """A few hundred Adam steps on noisy -> clean pairs of random-ellipse
    images: the loss falls and the trained network is closer to the clean
    images than its input is (what the prior gains over no prior)."""
    import torch
    from reconnet_b200.learned_prior import PriorCNN
    from reconnet_b200.phantom import ellipse_phantom
    g = np.random.default_rng(11)
    clean = np.stack([ellipse_phantom(64, 64, 4.0, 4.0, g) for _ in range(24)]).astype(np.float32)
    noisy = clean + g.normal(0, 0.004, clean.shape).astype(np.float32)
    ct, nt = torch.from_numpy(clean).cuda(), torch.from_numpy(noisy).cuda()
    net = PriorCNN("cuda", seed=1)
    losses = net.train(nt[:20], ct[:20], steps=300, batch=8, lr=2e-3, log_every=50)
    assert losses[-1] < 0.5 * losses[0]
    held_in, held_clean = nt[20:], ct[20:]
    den = net.denoise(held_in)
    err_net = float(((den - held_clean) ** 2).mean())
    err_id = float(((held_in - held_clean) ** 2).mean())
    assert err_net < 0.7 * err_id
