"""Batched uneven images under a captured CUDA graph (no reference counterpart).

A :class:`BatchPlan` fixes the batch structure (emitters per image), the
detector geometry and the precision.  It owns static device buffers for the
emitters, amplitudes and output, autotunes the forward kernel shape on the
first batch, and captures the whole forward (workspace reset, record prep,
persistent direct-sum kernel) in one CUDA graph, so each later batch is a
host->device copy plus one graph replay.
"""

from __future__ import annotations

from typing import Optional, Sequence

import numpy as np
import torch

from .. import _native as nat
from . import _core


class BatchPlan:
    def __init__(
        self,
        counts: Sequence[int],
        geom: nat.Geom,
        precision: int = nat.SPLIT,
        out_kind: int = nat.OUT_I64,
        amplitudes: Optional[str] = None,
        device=None,
        autotune: bool = True,
        graph: bool = True,
        config=None,
    ):
        """counts: emitters per image; amplitudes: None, "float32" or "float64"."""
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.counts = np.asarray(counts, dtype=np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)
        self.geom = geom
        self.precision = precision
        self.out_kind = out_kind
        n = int(self.offsets[-1])
        self.atoms = torch.zeros((n, 4), dtype=torch.float64, device=self.device)
        self.amplitudes = None
        if amplitudes is not None:
            dt = torch.float32 if amplitudes in ("float32", torch.float32) else torch.float64
            self.amplitudes = torch.ones(n, dtype=dt, device=self.device)
        self.out = torch.empty((len(self.counts), geom.nx, geom.ny), dtype=_core._OUT_DTYPES[out_kind],
                               device=self.device)
        self.config = config
        self._autotune = autotune and config is None
        self._use_graph = graph
        self._graph = None
        self._role = f"plan{id(self)}"

    def _launch(self):
        return _core.forward(self.atoms, self.offsets, self.geom, self.precision, self.out_kind,
                             amplitudes=self.amplitudes, out=self.out, config=self.config, role=self._role)

    def _prepare(self):
        if self._autotune:
            # tune on up to 8 images spread over the sorted emitter counts
            order = np.argsort(self.counts)
            pick = np.unique(order[np.linspace(0, len(order) - 1, min(8, len(order))).astype(int)])
            rows = [self.atoms[self.offsets[i]:self.offsets[i + 1]] for i in pick]
            sub = torch.cat(rows).contiguous()
            sub_off = np.concatenate([[0], np.cumsum(self.counts[pick])]).astype(np.int64)
            sub_amp = None
            if self.amplitudes is not None:
                sub_amp = torch.cat([self.amplitudes[self.offsets[i]:self.offsets[i + 1]] for i in pick]).contiguous()
            self.config = _core.tune(sub, sub_off, self.geom, self.precision, self.out_kind, amplitudes=sub_amp,
                                     role=self._role)
            self._autotune = False
        if self._use_graph and self._graph is None:
            s = torch.cuda.Stream(self.device)
            s.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.stream(s):
                self._launch()  # warm-up on the capture stream: allocates the workspace
            torch.cuda.current_stream(self.device).wait_stream(s)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=s):
                self._launch()
            self._graph = g

    def load(self, atoms=None, amplitudes=None):
        """Copy a new batch into the static buffers (stream-ordered)."""
        if atoms is not None:
            self.atoms.copy_(torch.as_tensor(atoms, dtype=torch.float64), non_blocking=True)
        if amplitudes is not None:
            if self.amplitudes is None:
                raise ValueError("plan was built without amplitudes")
            self.amplitudes.copy_(torch.as_tensor(amplitudes), non_blocking=True)

    def run(self, atoms=None, amplitudes=None) -> torch.Tensor:
        """Forward of the loaded (or given) batch; returns the static output tensor."""
        self.load(atoms, amplitudes)
        self._prepare()
        if self._graph is not None:
            self._graph.replay()
        else:
            self._launch()
        return self.out

    def cta_times(self) -> np.ndarray:
        """Per-CTA busy time (ns) of the last launch (synchronises)."""
        return _core.cta_times(self.device, role=self._role)

    def check(self):
        _core.workspace_error(self.device, role=self._role)

    def close(self):
        self._graph = None
        _core.WORKSPACES.drop(self.device, self._role)
