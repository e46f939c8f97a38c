"""GPU-side helpers for the -m gpu tests (torch is only device plumbing)."""
import ctypes
import os

import numpy as np

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_ref_gpu = None


def dev(a, torch):
    """numpy (col-major [col,row] layout) -> CUDA tensor with the same memory order."""
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a).cuda()


def host(t):
    return t.detach().cpu().numpy().astype(np.float64)


def spectra(Kx, Ky, M, torch):
    return dev(O.kernel_freq(Kx, M), torch), dev(O.kernel_freq(Ky, M), torch)


def ref_gpu():
    """The reference's own srkTrainingForward / srkCudnnForward /
    MeasureCD_Batched built from its sources (oracle/_ref), or None."""
    global _ref_gpu
    if _ref_gpu is None:
        path = os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so")
        if not os.path.exists(path):
            return None
        L = ctypes.CDLL(path)
        P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.ref_train_ws_create.argtypes = [I, I, P]
        L.ref_train_ws_create.restype = P
        L.ref_train_ws_destroy.argtypes = [P, P]
        L.ref_train_forward.argtypes = [P, P, P, P, I, I, I, F, I, P, P, P]
        L.ref_train_forward.restype = I
        fp = ctypes.POINTER(ctypes.c_float)
        L.ref_measure_cd.argtypes = [P, I, I, I, I, P, fp, fp, fp]
        L.ref_measure_cd.restype = I
        L.ref_cudnn_ws_create.argtypes = [I, I, I, I, P]
        L.ref_cudnn_ws_create.restype = P
        L.ref_cudnn_ws_destroy.argtypes = [P, P]
        L.ref_cudnn_forward.argtypes = [P, P, P, P, I, I, I, F, I, P, P, P]
        L.ref_cudnn_forward.restype = I
        _ref_gpu = L
    return _ref_gpu
