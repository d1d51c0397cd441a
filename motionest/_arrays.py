"""Array interop: the reference's API takes NumPy or CuPy arrays; motionest accepts NumPy
arrays, torch tensors and any CUDA array exposing __dlpack__ (CuPy included), computes on the
GPU, and returns results of the caller's kind (NumPy in -> NumPy out, device in -> torch CUDA
tensor out)."""
import numpy as np
import torch


def is_numpy(a):
    return isinstance(a, (np.ndarray, np.generic))


def to_device(a, dtype=None, device=None):
    """Return a contiguous CUDA tensor view/copy of `a` (no copy if already suitable)."""
    dev = device or torch.device("cuda", torch.cuda.current_device())
    if isinstance(a, torch.Tensor):
        t = a
    elif is_numpy(a):
        t = torch.from_numpy(np.ascontiguousarray(a))
    elif hasattr(a, "__dlpack__"):
        t = torch.from_dlpack(a)
    else:
        t = torch.as_tensor(np.asarray(a))
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    if t.device != dev:
        t = t.to(dev, non_blocking=False)
    return t.contiguous()


def like_input(result, ref):
    """Return `result` (CUDA tensor) as the caller's array kind."""
    if is_numpy(ref):
        return result.cpu().numpy()
    return result


def as_float64_host(a):
    if isinstance(a, torch.Tensor):
        return a.detach().to("cpu", torch.float64).numpy()
    if hasattr(a, "get"):  # CuPy
        return np.asarray(a.get(), dtype=np.float64)
    return np.asarray(a, dtype=np.float64)
