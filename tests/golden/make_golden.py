"""Generate the closed-form golden fixtures of tests/golden/*.npz.

The reference (Julia) cannot run here, so its known-answer tests are restated: each fixture holds
inputs and the outputs that the reference's tests derive in closed form, computed here with
plain numpy from those formulas -- never from the oracle or the CUDA library.

* worked_example.npz   docs/src/implementing/example.md:28-257
    32 points on [0, 1], K(s,t) = 1 + 2s + 3t + (4+i)st, x_j = sin(j) + i cos(2j);
    y = F x, transpose(F) x, F' x, and the scaled products (2-i) op(F) x + (3+2i) * (2+i).
* clusters_b4.npz      test/farinteractions/test_farmul.jl:17-97
    8 points, far matrix F[1:4,5:8] = F[5:8,1:4] = c = 2 - i; x ~ N(0,1) complex (seeded);
    far products in all orientations and the (alpha, beta) accumulation case.
* clusters_6x20.npz    test/farinteractions/test_component_harness.jl:88-118
    6 clusters x 20 points, F[i,j] = c iff clusters differ, complex c = 2 - i and real c = 2.
* toeplitz_smoke.npz   test/H2Toeplitz/test_smoke.jl:27-78
    wrap-around multilevel Toeplitz matrices for shapes (3,), (3,2), (2,2,2), (3,2,2), (3,3,3),
    (3,2,4), built densely from the kernel (no FFT), and T x, T' x for seeded complex x.

Run:  python tests/golden/make_golden.py
"""

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def worked_example():
    n = 32
    s = np.linspace(0.0, 1.0, n)
    F = 1 + 2 * s[:, None] + 3 * s[None, :] + (4 + 1j) * s[:, None] * s[None, :]
    j = np.arange(1, n + 1)
    x = np.sin(j) + 1j * np.cos(2 * j)
    out0 = np.full(n, 2.0 + 1j)
    a, b = 2 - 1j, 3 + 2j
    np.savez(os.path.join(HERE, "worked_example.npz"), coords=s, F=F, x=x,
             y_fwd=F @ x, y_t=F.T @ x, y_h=F.conj().T @ x,
             out0=out0, alpha=a, beta=b,
             ys_fwd=a * (F @ x) + b * out0, ys_t=a * (F.T @ x) + b * out0,
             ys_h=a * (F.conj().T @ x) + b * out0)


def clusters_b4():
    pts = np.array([0.0, 0.1, 5.0, 5.1, 40.0, 40.1, 45.0, 45.1])
    c = 2.0 - 1.0j
    F = np.zeros((8, 8), np.complex128)
    F[:4, 4:] = c
    F[4:, :4] = c
    rng = np.random.default_rng(20240101)
    x = (rng.standard_normal(8) + 1j * rng.standard_normal(8)) / np.sqrt(2)
    y0 = (rng.standard_normal(8) + 1j * rng.standard_normal(8)) / np.sqrt(2)
    a, b = 0.7 + 0.3j, -0.4 + 0.2j
    np.savez(os.path.join(HERE, "clusters_b4.npz"), points=pts, c=c, F=F, x=x,
             y_fwd=F @ x, y_t=F.T @ x, y_h=F.conj().T @ x, y0=y0, alpha=a, beta=b,
             y_acc=a * (F @ x) + b * y0)


def clusters_6x20():
    k, n = 6, 20
    pts = np.array([c * 100.0 + 0.1 * j / (n - 1) for c in range(k) for j in range(n)])
    cid = np.repeat(np.arange(k), n)
    rng = np.random.default_rng(20240102)
    out = {"points": pts, "cid": cid}
    for tag, c in (("c", 2.0 - 1.0j), ("r", 2.0)):
        F = np.where(cid[:, None] != cid[None, :], c, 0)
        if tag == "r":
            x = rng.standard_normal(k * n)
            F = F.astype(np.float64)
        else:
            x = (rng.standard_normal(k * n) + 1j * rng.standard_normal(k * n)) / np.sqrt(2)
        out.update({f"{tag}_c": c, f"{tag}_x": x, f"{tag}_fwd": F @ x, f"{tag}_t": F.T @ x,
                    f"{tag}_h": F.conj().T @ x})
    np.savez(os.path.join(HERE, "clusters_6x20.npz"), **out)


def dense_multilevel_toeplitz(kernel, s):
    """T[lin(i), lin(j)] = kernel[mod(i - j, ts)] per axis (column-major linear indices)."""
    ts = kernel.shape
    nd = len(s)
    idx = np.stack(np.meshgrid(*[np.arange(v) for v in s], indexing="ij"), -1)
    idx = idx.reshape(-1, nd, order="F")
    key = (idx[:, None, :] - idx[None, :, :]) % np.array(ts)
    return kernel[tuple(key[..., d] for d in range(nd))]


def toeplitz_smoke():
    rng = np.random.default_rng(7)
    out = {}
    for q, s in enumerate(((3,), (3, 2), (2, 2, 2), (3, 2, 2), (3, 3, 3), (3, 2, 4))):
        ts = tuple(2 * v - 1 for v in s)
        kernel = rng.standard_normal(ts) + 1j * rng.standard_normal(ts)
        T = dense_multilevel_toeplitz(kernel, s)
        n = int(np.prod(s))
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        out[f"s{q}"] = np.array(s)
        out[f"kernel{q}"] = kernel
        out[f"x{q}"] = x
        out[f"Tx{q}"] = T @ x
        out[f"THx{q}"] = T.conj().T @ x
    np.savez(os.path.join(HERE, "toeplitz_smoke.npz"), **out)


if __name__ == "__main__":
    worked_example()
    clusters_b4()
    clusters_6x20()
    toeplitz_smoke()
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))
