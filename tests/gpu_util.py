"""Helpers for the GPU parity tests: device buffers (torch) handed to the C ABI."""
import numpy as np
import torch


def dev(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


def host(t: torch.Tensor) -> np.ndarray:
    torch.cuda.synchronize()
    return t.cpu().numpy()


def stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def bits_equal(a: np.ndarray, b: np.ndarray) -> bool:
    return a.dtype == b.dtype and np.array_equal(a.view(np.uint8), b.view(np.uint8))
