"""Plain PyTorch (CPU, FP64) restatement of StereoNet's quarter-resolution
front: FeatureNet (stereonet.py:1022-1070), CostVolume (740-842),
CostFilter (1071-1109) and SoftArgmin (843-900).  With ``bf16=True`` the
operands of the six convolutions the BF16 path runs on the tensor cores
(FeatureNet c1..c4, CostFilter c1 and c2, the cost volume included) are
rounded to BF16 first and every layer output to FP32, as the GPU kernels
store them; CostFilter c3 and the soft-argmin stay unrounded.  Test
infrastructure: the numerics reference for the tensor-core convolutions.
"""

import numpy as np
import torch
import torch.nn.functional as F


def unpack(w):
    """StereoNetWeights -> dict of torch FP64 tensors (all_params order)."""
    a = w.arch
    C, Cm = a.feat_C, a.cost_C
    it = iter(w.blocks)
    t = {}
    for i, ic in enumerate((1, C, C, C)):
        t["fw%d" % i] = torch.from_numpy(next(it)).reshape(C, ic, 3, 3)
        t["fb%d" % i] = torch.from_numpy(next(it))
    for i, (ic, oc) in enumerate(((C, Cm), (Cm, Cm), (Cm, 1))):
        t["cw%d" % i] = torch.from_numpy(next(it)).reshape(oc, ic, 3, 3, 3)
        t["cb%d" % i] = torch.from_numpy(next(it))
    return t


def _leaky(x):
    return torch.where(x > 0, x, x * 0.2)


def front(w, left, right, H, W, bf16=False):
    """Images as float arrays in [0, 1] (H x W) -> d0 [h][w] (quarter res)."""
    t = unpack(w)
    D = w.arch.D
    if bf16:
        rnd = lambda x: x.to(torch.bfloat16).to(torch.float64)          # noqa: E731
        f32 = lambda x: x.to(torch.float32).to(torch.float64)           # noqa: E731
    else:
        rnd = f32 = lambda x: x                                           # noqa: E731
    x = torch.stack([torch.as_tensor(np.asarray(left, np.float64).reshape(H, W)),
                     torch.as_tensor(np.asarray(right, np.float64).reshape(H, W))])[:, None]
    x = f32(x)
    for i in range(4):
        x = F.conv2d(rnd(x), rnd(t["fw%d" % i]), t["fb%d" % i], stride=2 if i < 2 else 1,
                     padding=1)
        x = f32(_leaky(x) if i < 3 else x)
    fl, fr = x[0], x[1]                                    # [C][h][w]
    C, h, wq = fl.shape
    vol = torch.full((C, D, h, wq), 2.0, dtype=torch.float64)
    for d in range(D):
        if d < wq:
            vol[:, d, :, d:] = (fl[:, :, d:] - fr[:, :, :wq - d]).abs()
    vol = f32(vol)
    v = vol[None]
    for i in range(2):
        v = f32(_leaky(F.conv3d(rnd(v), rnd(t["cw%d" % i]), t["cb%d" % i], padding=1)))
    cost = F.conv3d(v, t["cw2"], t["cb2"], padding=1)[0, 0]          # [D][h][w]
    dd = torch.arange(D, dtype=torch.float64)[:, None, None]
    xx = torch.arange(wq, dtype=torch.float64)[None, None, :]
    cost = cost + torch.where((dd >= 1) & (xx < dd), 8.0, 0.0)
    neg = -cost
    e = torch.exp(neg - neg.max(dim=0, keepdim=True).values)
    return ((dd * e).sum(0) / e.sum(0)).numpy()
