"""A forward projection captured as a CUDA graph (extension; not in the
reference): fixed device buffers of rays and image, replayed with one
graph launch per step (vt_graph_create / vt_graph_launch / vt_graph_finish).

    g = ProjectionGraph(pc, starts, ends)     # CUDA tensors (R, 3), float64
    g.launch()                                # enqueue on the current stream
    img = g.out                               # valid once the stream has run it
    stats = g.finish()                        # wait, counters; raises on failure

Refill ``g.starts`` / ``g.ends`` in place between launches to project other
rays of the same count.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L
from .vortrace import ProjectionCloud


class ProjectionGraph:
    def __init__(self, pc: ProjectionCloud, starts: torch.Tensor, ends: torch.Tensor, *,
                 reduction: str = "integrate", kernel: str = "auto"):
        mode = pc._validate_reduction(reduction)
        if not (starts.is_cuda and ends.is_cuda):
            raise ValueError("starts / ends must be CUDA tensors")
        self.starts = starts.to(torch.float64).contiguous()
        self.ends = ends.to(torch.float64).contiguous()
        if self.starts.shape != self.ends.shape or self.starts.shape[-1] != 3:
            raise ValueError("starts / ends must have identical shapes (R, 3)")
        n = self.starts.shape[0]
        self.out = torch.empty((n, pc._nout(mode)), dtype=torch.float64,
                               device=self.starts.device)
        self._pc = pc
        self._lib = pc._cloud._lib
        h = C.c_void_p()
        L.check(self._lib.vt_graph_create(pc._cloud._h, self.starts.data_ptr(),
                                          self.ends.data_ptr(), n, mode, L.KERNELS[kernel],
                                          self.out.data_ptr(), C.byref(h)))
        self._h = h

    def _stream(self, stream):
        s = stream if stream is not None else torch.cuda.current_stream(self.out.device)
        return s.cuda_stream

    def launch(self, stream=None):
        L.check(self._lib.vt_graph_launch(self._h, self._stream(stream)))
        return self.out

    def finish(self, stream=None) -> dict:
        st = L.Stats()
        L.check(self._lib.vt_graph_finish(self._h, self._stream(stream), C.byref(st)))
        return st.as_dict()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.vt_graph_destroy(h)
            self._h = None
