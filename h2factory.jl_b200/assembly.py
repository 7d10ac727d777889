"""Device-side assembly of near-field blocks for large maps (construction time, not the product path).

A method supplies the near blocks (H2Factory's near interactions, src/nearinteractions/nearmul.jl:
54-111). For the Laplace/Helmholtz kernels on hundreds of millions of entries this is done on the
GPU with torch, batch by batch, straight into the column-major block layout the core takes
(`H2Core.set_near_device`), so the blocks never cross PCIe.
"""

from __future__ import annotations

import math

import numpy as np


def near_blocks_device(core, kernel: str = "laplace", wavenumber: float = 0.0,
                       device: str = "cuda:0", batch_entries: int = 1 << 26):
    """Assemble every near block of `core` on `device` and attach them to the core."""
    import torch

    test, trial = core.test, core.trial
    near = core.plans.near
    nvt = np.diff(test.value_ptr).astype(np.int64)
    nvs = np.diff(trial.value_ptr).astype(np.int64)
    nr = nvt[near[:, 0]]
    nc = nvs[near[:, 1]]
    sizes = nr * nc
    offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    total = int(sizes.sum())
    cplx = core.field == "complex"
    dt = torch.complex128 if cplx else torch.float64
    out = torch.empty(max(total, 1), dtype=dt, device=device)
    m = int(max(nvt.max(initial=1), nvs.max(initial=1)))
    # padded per-leaf point tables
    def table(tree, nv):
        leaves = np.nonzero(nv > 0)[0]
        tab = np.zeros((tree.nnodes, m, 3))
        for n in leaves:
            v = tree.values(int(n))
            tab[n, :v.size, :tree.dim] = tree.points[v]
        return torch.from_numpy(tab).to(device)

    pt = table(test, nvt)
    ps = pt if trial is test else table(trial, nvs)
    per = max(1, batch_entries // (m * m))
    i_idx = torch.arange(m, device=device)
    for s in range(0, near.shape[0], per):
        e = min(near.shape[0], s + per)
        a = torch.from_numpy(near[s:e, 0].astype(np.int64)).to(device)
        b = torch.from_numpy(near[s:e, 1].astype(np.int64)).to(device)
        xa = pt[a]                      # (P, m, 3)
        yb = ps[b]
        d = xa[:, :, None, :] - yb[:, None, :, :]
        r = torch.sqrt((d * d).sum(-1))  # (P, m, m) rows i, cols j
        safe = torch.where(r > 0, r, torch.ones_like(r))
        if kernel == "laplace":
            k = torch.where(r > 0, 1.0 / (4.0 * math.pi * safe), torch.zeros_like(r))
        elif kernel == "helmholtz":
            k = torch.where(r > 0, torch.exp(1j * wavenumber * safe) / (4.0 * math.pi * safe),
                            torch.zeros_like(r, dtype=torch.complex128))
        else:
            raise ValueError(kernel)
        k = k.to(dt)
        nrb = torch.from_numpy(nr[s:e]).to(device)
        ncb = torch.from_numpy(nc[s:e]).to(device)
        ob = torch.from_numpy(offsets[s:e]).to(device)
        valid = (i_idx[None, :, None] < nrb[:, None, None]) & (i_idx[None, None, :] < ncb[:, None, None])
        dest = ob[:, None, None] + i_idx[None, :, None] + i_idx[None, None, :] * nrb[:, None, None]
        out[dest[valid]] = k[valid]
    core.set_near_device(out, offsets)
    return out, offsets
