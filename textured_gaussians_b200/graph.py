"""Forward + backward of the renderer captured in one CUDA graph.

The path has two data-dependent sizes, both read back to the host in eager
mode exactly where the reference reads them: the packed entry count (nnz,
fully_fused_projection_packed_2dgs_fwd.cu:274-275) and the intersection count
(isect_tiles.cu:200-201).  A CUDA graph cannot contain those reads, so under
a :class:`SizePlan` in "capture" mode every such op sizes its buffers by a
capacity instead:

* an eager "record" pass first notes each size, in call order;
* the capture gives call k the capacity ``max(ceil(size_k * slack), size_k + floor)``;
* the kernels read the true count from device memory; the unused tail is
  inert (packed entries with radius 0, intersection keys padded to sort after
  every real key and never reached by the compositor);
* each op zeroes, inside the graph, a device overflow flag that its kernels
  raise if a replay needs more than the capacity.

:class:`GraphedStep` records, captures and replays a user step function
(forward, loss and ``backward()`` of this package's renderer); after a replay
``overflowed()`` reads the flags (one synchronisation) and ``recapture()``
re-plans the sizes.  Gradients land in the leaves' ``.grad`` tensors, which
the capture allocates and every replay overwrites.
"""
from __future__ import annotations

import gc
import math
import threading
from typing import Callable, List, Optional

import torch

_local = threading.local()


class SizePlan:
    """Context that switches the data-dependent ops to "record" or "capture" mode."""

    def __init__(self, mode: str, capacities: Optional[List[int]] = None):
        assert mode in ("record", "capture")
        self.mode = mode
        self.sizes: List[int] = []
        self.capacities = list(capacities or [])
        self.k = 0
        self.flags: List[torch.Tensor] = []

    def __enter__(self):
        self._prev = getattr(_local, "plan", None)
        _local.plan = self
        return self

    def __exit__(self, *exc):
        _local.plan = self._prev

    def next_capacity(self) -> int:
        if self.k >= len(self.capacities):
            raise RuntimeError("the captured step makes more size-dependent calls than the recorded one")
        cap = self.capacities[self.k]
        self.k += 1
        return cap

    def new_flag(self, device) -> torch.Tensor:
        f = torch.zeros((1,), dtype=torch.int32, device=device)
        self.flags.append(f)
        return f


def active_plan() -> Optional[SizePlan]:
    return getattr(_local, "plan", None)


def _detach(x):
    if isinstance(x, torch.Tensor):
        return x.detach()
    if isinstance(x, (tuple, list)):
        return type(x)(_detach(v) for v in x)
    if isinstance(x, dict):
        return {k: _detach(v) for k, v in x.items()}
    return x


class GraphedStep:
    """One CUDA graph holding ``fn()``: forward, loss and backward.

    ``fn`` takes no arguments and reads its inputs from tensors whose storage
    stays put (update them in place between replays); it should set the
    leaves' ``.grad`` to None before its forward.  What it returns is kept,
    detached, as ``self.out`` and refreshed by every replay; the leaves'
    ``.grad`` are the tensors the capture allocated (running ``fn`` eagerly
    afterwards rebinds them).  No autograd graph that reaches the leaves may
    be alive when capturing (the capture's gradient accumulation must run on
    the capturing stream).
    """

    def __init__(self, fn: Callable[[], object], slack: float = 1.25, floor: int = 4096, warmup: int = 2):
        self.fn, self.slack, self.floor, self.warmup = fn, slack, floor, warmup
        self.graph: Optional[torch.cuda.CUDAGraph] = None
        self.out = None
        self.capture()

    def capture(self):
        self.graph, self.out, self.flags = None, None, []
        gc.collect()
        with SizePlan("record") as rec:
            _detach(self.fn())
        torch.cuda.synchronize()
        self.sizes = rec.sizes
        self.capacities = [max(int(math.ceil(n * self.slack)), n + self.floor) for n in self.sizes]
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            for _ in range(self.warmup):
                with SizePlan("capture", self.capacities):
                    _detach(self.fn())
        torch.cuda.current_stream().wait_stream(side)
        gc.collect()
        self.graph = torch.cuda.CUDAGraph()
        with SizePlan("capture", self.capacities) as plan:
            with torch.cuda.graph(self.graph):
                self.out = _detach(self.fn())
        self.flags = plan.flags

    recapture = capture

    def replay(self):
        self.graph.replay()
        return self.out

    def overflowed(self) -> bool:
        """True if the last replay needed more than a captured capacity (synchronises)."""
        if not self.flags:
            return False
        return bool(torch.stack([f.reshape(()) for f in self.flags]).any().item())
