"""Many maps of uneven size multiplied as one batch, with the pass sequence captured in a graph.

A product of a small map is launch-bound: its ~10 kernels run for a few microseconds each. The
batch gives every map its own workspace and CUDA stream (so maps overlap on the device) and
captures the whole batch -- every map's near pass, upward pass, I2O and downward pass -- once in a
CUDA graph; a replay then costs one launch from the host for all maps. Inputs and outputs live in
fixed device buffers that the graph reads and writes (`set_inputs`, `outputs`).
"""

from __future__ import annotations

import numpy as np

from .core import H2Workspace, OrientedMap, mul_


class BatchedMaps:
    """y_k = op_k(A_k) x_k for a list of cores, one right-hand-side block per map."""

    def __init__(self, cores, nrhs, device: int = 0, modes=None):
        import torch

        self.torch = torch
        self.dev = f"cuda:{device}"
        self.nrhs = [int(r) for r in nrhs]
        self.modes = list(modes) if modes is not None else [0] * len(cores)
        self.ws = [H2Workspace(c, max_nrhs=r, device=device) for c, r in zip(cores, self.nrhs)]
        self.streams = [torch.cuda.Stream(self.dev) for _ in cores]
        self.inputs, self.outputs = [], []
        for k, (c, r) in enumerate(zip(cores, self.nrhs)):
            nin = c.trial.npoints if self.modes[k] == 0 else c.test.npoints
            nout = c.test.npoints if self.modes[k] == 0 else c.trial.npoints
            self.inputs.append(torch.zeros((r, nin), dtype=self.dtype(k), device=self.dev).t())
            self.outputs.append(torch.zeros((r, nout), dtype=self.dtype(k), device=self.dev).t())
        self.graph = None

    def dtype(self, k: int):
        return self.torch.complex128 if self.ws[k].core.field == "complex" else self.torch.float64

    def set_inputs(self, xs) -> None:
        for dst, x in zip(self.inputs, xs):
            dst.copy_(x)

    def _issue(self, base) -> None:
        """Every map's product on its own stream, forked from and joined back to `base`."""
        torch = self.torch
        for k, ws in enumerate(self.ws):
            s = self.streams[k]
            s.wait_stream(base)
            op = ws if self.modes[k] == 0 else OrientedMap(ws, self.modes[k])
            with torch.cuda.stream(s):
                mul_(self.outputs[k], op, self.inputs[k], stream=s.cuda_stream)
            base.wait_stream(s)

    def run_eager(self) -> None:
        self._issue(self.torch.cuda.current_stream(self.dev))

    def capture(self) -> None:
        """Record the batch once (after one eager run has set every kernel's attributes)."""
        torch = self.torch
        self.run_eager()
        torch.cuda.synchronize(self.dev)
        s0 = torch.cuda.Stream(self.dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s0):
            self._issue(s0)
        self.graph = g

    def replay(self) -> None:
        self.graph.replay()

    def rhs_total(self) -> int:
        return int(np.sum(self.nrhs))

    def close(self) -> None:
        self.graph = None
        for ws in self.ws:
            ws.close()
