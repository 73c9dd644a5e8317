"""CPU oracle of the learned-guess network — TEST INFRASTRUCTURE ONLY.

The network has no counterpart in the reference: the reference seeds each
Poisson solve with the previous potential (RootGrid::solvePoissonPSOR keeps
phi between calls, src/Grid/RootGrid/RootGridField.cpp:65-103). This module
restates the network that libfopis_gpu.so trains (3-level 3D U-Net,
16/32/64 channels, 3x3x3 convolutions, 1x1 head) in float64 with torch on the
CPU, rounding to BF16 wherever the GPU stores BF16 (activations, features,
convolution weights; biases and head stay FP32), so that the GPU's forward
activations and its parameter gradients can be checked against it. Gradients
come from autograd with straight-through rounding: the GPU also rounds its
gradient tensors to BF16, which the comparison's tolerance absorbs.

Grids are the multigrid levels of the solver: unknowns per axis n (glue
indices 1..n on a periodic axis, 2..nx-1 otherwise), coarsened to n/2 while a
periodic axis stays even and >= 4 and a non-periodic one >= 3; coarse point I
sits at fine 2I (periodic) or 2I+1.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as Fn

LAYERS = [(16, 16, 0), (16, 32, 1), (32, 64, 2), (64, 64, 2), (64, 32, 1), (32, 16, 0)]
HEAD = 16


def param_layout():
    """Offsets of W[27][cout][cin], b[cout] per convolution, then head w[16], b."""
    off, out = 0, []
    for cin, cout, _ in LAYERS:
        w = off
        off += 27 * cin * cout
        b = off
        off += cout
        out.append((w, b, cin, cout))
    return out, off, off + HEAD + 1


def levels(nxyz, per):
    lv = [tuple(n if p else n - 2 for n, p in zip(nxyz, per))]
    while len(lv) < 3:
        f = lv[-1]
        ok = all((n % 2 == 0 and n >= 4) if p else n >= 3 for n, p in zip(f, per))
        if not ok:
            raise ValueError("grid too small for three levels")
        lv.append(tuple(n // 2 for n in f))
    return lv


def bf16(x: torch.Tensor) -> torch.Tensor:
    return x.to(torch.bfloat16).to(x.dtype)


def st(x: torch.Tensor) -> torch.Tensor:
    """Round to BF16 in the forward pass, identity in the backward pass."""
    return x + (bf16(x) - x).detach()


def up_matrix(nf: int, nc: int, per: bool) -> np.ndarray:
    """Trilinear prolongation along one axis (the solver's)."""
    P = np.zeros((nf, nc))
    for f in range(nf):
        if per:
            if f % 2 == 0:
                P[f, f // 2] = 1.0
            else:
                P[f, f // 2] += 0.5
                P[f, (f // 2 + 1) % nc] += 0.5
        else:
            if f % 2 == 1:
                if (f - 1) // 2 < nc:
                    P[f, (f - 1) // 2] = 1.0
            else:
                hi, lo = f // 2, f // 2 - 1
                if lo >= 0:
                    P[f, lo] += 0.5
                if hi < nc:
                    P[f, hi] += 0.5
    return P


def fine_index(nc: int, per: bool) -> np.ndarray:
    return np.arange(nc) * 2 + (0 if per else 1)


def features(params, rho0, phi1, phi2):
    """Input channels on the level-0 unknowns: r1/sigma_r, (f - mean)/sigma_f,
    (phi1 - phi2)/sigma_d, phi1/sigma_phi; returns (x0 [16, n0, n1, n2],
    sigma_d, periodic axes, unknown index)."""
    nxyz = (params.nx, params.ny, params.nz)
    b = bytes(params.boundary).split(b"\0")[0].decode()
    per = [b[2 * a] == "P" for a in range(3)]
    shape = tuple(n + 2 for n in nxyz)
    rho0, phi1, phi2 = (np.asarray(a, np.float64).reshape(shape) for a in (rho0, phi1, phi2))
    idx, im, ip = [], [], []
    for a in range(3):
        o, n, nref = (1, nxyz[a], nxyz[a]) if per[a] else (2, nxyz[a] - 2, nxyz[a])
        g = np.arange(n) + o

        def wrap(v):
            if per[a]:
                v = np.where(v == 0, nref, v)
                v = np.where(v == nref + 1, 1, v)
            return v
        idx.append(g)
        im.append(wrap(g - 1))
        ip.append(wrap(g + 1))
    I = np.ix_(*idx)
    f = rho0[I] / params.eps0
    M = f.size
    allper = all(per)
    fm = f.sum() / M if allper else 0.0
    sf = np.sqrt(max(np.sum(f * f) / M - fm * fm, 0.0)) or 1.0
    d = phi1[I] - phi2[I]
    sd = np.sqrt(max(np.sum(d * d) / M, 0.0))
    sp = np.sqrt(max(np.sum(phi1[I] ** 2) / M, 0.0)) or 1.0
    p0 = phi1[I]
    nb = (phi1[np.ix_(im[0], idx[1], idx[2])] + phi1[np.ix_(ip[0], idx[1], idx[2])] +
          phi1[np.ix_(idx[0], im[1], idx[2])] + phi1[np.ix_(idx[0], ip[1], idx[2])] +
          phi1[np.ix_(idx[0], idx[1], im[2])] + phi1[np.ix_(idx[0], idx[1], ip[2])])
    fc = f - fm
    r1 = fc - (6.0 * p0 - nb)
    sr = np.sqrt(np.mean(r1 * r1)) or 1.0
    x0 = np.zeros((16,) + f.shape)
    x0[0] = r1 / sr
    x0[1] = fc / sf
    x0[2] = d / sd if sd > 0 else 0.0
    x0[3] = p0 / sp
    x0 = x0.astype(np.float32).astype(np.float64)
    return x0, sd, per, I


class Net:
    """The network on float64 tensors; prm is the flat FP32 parameter vector."""

    def __init__(self, prm: np.ndarray, lv, per):
        self.layout, _, self.n = param_layout()
        self.prm = torch.tensor(np.asarray(prm, np.float64), requires_grad=True)
        self.lv, self.per = lv, per
        self.P = [[torch.tensor(up_matrix(lv[l][a], lv[l + 1][a], per[a])) for a in range(3)] for l in range(2)]
        self.fi = [[torch.tensor(fine_index(lv[l + 1][a], per[a])) for a in range(3)] for l in range(2)]

    def conv(self, l, x):
        w, b, cin, cout = self.layout[l]
        W = self.prm[w:w + 27 * cin * cout].reshape(3, 3, 3, cout, cin).permute(3, 4, 0, 1, 2)
        W = st(W)
        return Fn.conv3d(x[None], W, self.prm[b:b + cout], padding=1)[0]

    def down(self, l, x):
        i, j, k = self.fi[l]
        return x[:, i][:, :, j][:, :, :, k]

    def up(self, l, x):
        Pa, Pb, Pc = self.P[l]
        return torch.einsum("ai,bj,ck,xijk->xabc", Pa, Pb, Pc, x)

    def forward(self, x0):
        act = {}
        x0 = torch.tensor(x0)
        act["x0"] = x0
        act["e0"] = e0 = st(torch.relu(self.conv(0, x0)))
        act["d1"] = d1 = self.down(0, e0)
        act["e1"] = e1 = st(torch.relu(self.conv(1, d1)))
        act["d2"] = d2 = self.down(1, e1)
        act["e2"] = e2 = st(torch.relu(self.conv(2, d2)))
        act["e3"] = e3 = st(torch.relu(self.conv(3, e2)))
        act["u1"] = u1 = st(self.up(1, e3))
        act["a4"] = a4 = st(torch.relu(self.conv(4, u1)))
        act["u0"] = u0 = st(self.up(0, a4 + e1))
        act["a5"] = a5 = st(torch.relu(self.conv(5, u0)))
        h = self.prm[self.n - HEAD - 1:self.n - 1]
        out = torch.einsum("c,cxyz->xyz", h, a5 + e0) + self.prm[self.n - 1]
        act["out"] = out
        return out, act


def evaluate(params, prm, rho0, phi1, phi2, phi_target=None):
    """Prediction (on the unknowns, physical units), activations, loss and the
    gradient of the loss for every parameter."""
    x0, sd, per, I = features(params, rho0, phi1, phi2)
    lv = levels((params.nx, params.ny, params.nz), per)
    net = Net(prm, lv, per)
    out, act = net.forward(x0)
    res = {"act": {k: v.detach().numpy() for k, v in act.items()}, "sigma_d": sd,
           "pred": sd * out.detach().numpy()}
    if phi_target is not None:
        shape = tuple(n + 2 for n in (params.nx, params.ny, params.nz))
        scale = 1.0 / sd if sd > 0 else 0.0
        t = (np.asarray(phi_target).reshape(shape)[I] - np.asarray(phi1).reshape(shape)[I]) * scale
        loss = torch.mean((out - torch.tensor(t)) ** 2)
        loss.backward()
        res["loss"] = float(loss.detach())
        res["grad"] = net.prm.grad.numpy().copy()
    return res
