"""Optional NVTX ranges around the host-side phases (assembly, linear solve,
Newton iteration, time step, serving round) for a timeline profiler.  Off
unless the environment sets FEA_B200_NVTX=1; then every range is pushed and
popped on the calling thread through torch.cuda.nvtx."""
from __future__ import annotations

import contextlib
import os

ENABLED = os.environ.get("FEA_B200_NVTX", "0") not in ("", "0")


@contextlib.contextmanager
def nvtx(name: str):
    if not ENABLED:
        yield
        return
    import torch
    torch.cuda.nvtx.range_push(name)
    try:
        yield
    finally:
        torch.cuda.nvtx.range_pop()
