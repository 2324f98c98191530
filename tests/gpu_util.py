"""Device buffers for the GPU tests: torch holds the memory, the library's
C ABI does the work (pointers and the current stream are passed through)."""
import numpy as np


def torch():
    import torch as t

    return t


def dev(array):
    t = torch()
    return t.from_numpy(np.ascontiguousarray(array)).cuda()


def empty(shape, dtype):
    t = torch()
    return t.empty(shape, dtype=dtype, device="cuda")


def ptr(tensor):
    return tensor.data_ptr()


def stream():
    return torch().cuda.current_stream().cuda_stream


def host(tensor):
    torch().cuda.synchronize()
    return tensor.cpu().numpy()


def same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype == np.float32:
        return bool((a.view(np.uint32) == b.astype(np.float32).view(np.uint32)).all())
    return bool((a == b).all())
