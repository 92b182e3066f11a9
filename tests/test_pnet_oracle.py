"""CPU: pin the network oracle (oracle/pnet_reference.py).  Its 3x3x3 layer, written with
torch's conv3d and our weight layout, must equal a plain loop convolution; its gradient
must equal central finite differences in float64."""
import numpy as np
import torch

from oracle import pnet_reference as R


def test_conv3_layout_matches_direct_loop():
    rng = np.random.default_rng(3)
    shape = (6, 5, 4)
    N = int(np.prod(shape))
    cin, cout = 3, 4
    x = rng.standard_normal((N, cin))
    w = rng.standard_normal(27 * cin * cout)
    b = rng.standard_normal(cout)
    tw = R._torch_weight("conv3", torch.tensor(w), cin, cout)
    tx = torch.tensor(x).reshape(shape[2], shape[1], shape[0], cin).permute(3, 0, 1, 2).unsqueeze(0)
    got = torch.nn.functional.conv3d(tx, tw, torch.tensor(b), padding=1)[0].permute(1, 2, 3, 0).reshape(N, cout)
    assert np.allclose(got.numpy(), R.direct_conv3(x, w, b, shape), atol=1e-12)


def test_param_count():
    offs, total = R.offsets()
    assert len(offs) == 12 and 1.0e5 < total < 2.0e5
    assert all(w % 8 == 0 for w, _ in offs)


def test_oracle_gradient_finite_differences():
    """The oracle's autograd gradient (without BF16 rounding) against central differences."""
    rng = np.random.default_rng(5)
    shape = (5, 6, 4)
    N = int(np.prod(shape))
    _, total = R.offsets()
    p = rng.standard_normal(total) * 0.2
    x = rng.standard_normal((N, 2))
    t = rng.standard_normal(N) * 0.1
    orig = R._bf16
    R._bf16 = lambda a: a
    try:
        def loss(pp):
            pp = pp if torch.is_tensor(pp) else torch.tensor(pp, dtype=torch.float64)
            y = R.forward(pp, torch.tensor(x, dtype=torch.float64), shape)
            m = torch.zeros(shape[2], shape[1], shape[0], dtype=torch.bool)
            m[1:-1, 1:-1, 1:-1] = True
            d = (y - torch.tensor(t))[m.reshape(-1)]
            return (d * d).mean()
        pt = torch.tensor(p, dtype=torch.float64, requires_grad=True)
        loss(pt).backward()
        g = pt.grad.numpy()
        offs, _ = R.offsets()
        for (wo, bo) in (offs[0], offs[5], offs[9], offs[11]):
            for idx in (wo, wo + 7, bo):
                e = np.zeros(total)
                e[idx] = 1e-6
                fd = (float(loss(p + e)) - float(loss(p - e))) / 2e-6
                assert abs(fd - g[idx]) <= 1e-6 + 1e-5 * abs(fd)
    finally:
        R._bf16 = orig
