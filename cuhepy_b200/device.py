"""Device resolution with the reference's signature (src/cuhepy/device.py:26-61).

This build has no CPU implementation: ``"cpu"`` is rejected, and ``"auto"``
and ``"gpu"`` both load and probe the B200 backend and raise if it is absent,
instead of silently falling back to a CPU path.
"""

from __future__ import annotations

from collections.abc import Callable
from typing import Any, Literal

DeviceMode = Literal["auto", "cpu", "gpu"]


def resolve_device(requested: DeviceMode, gpu_loader: Callable[[], type[Any]]) -> tuple[str, type[Any]]:
    if requested not in ("auto", "cpu", "gpu"):
        raise ValueError("device must be 'auto', 'cpu', or 'gpu'")
    if requested == "cpu":
        raise NotImplementedError("cuhepy_b200 computes on the B200 only; use device='gpu' or 'auto'")
    gpu_cls = gpu_loader()
    gpu_cls(skip_key_gen=True)
    return "gpu", gpu_cls
