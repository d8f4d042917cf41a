"""Python front end of libfinflo_nn.so: the BF16 tensor-core kernels of the
learned warm start (include/finflo_nn.h).

torch tensors provide the device memory and the stream; every computation
goes through the library's kernels.  The wrappers check shapes, dtypes and
strides and raise NNError on a non-zero status.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfinflo_nn.so")
_SRC = os.path.join(_HERE, "csrc", "ff_nn.cu")
_HDR = os.path.join(_HERE, "..", "include", "finflo_nn.h")
NVCC_FLAGS = ["-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-shared", "-std=c++17"]

SYMBOLS = ["ffnn_gemm", "ffnn_silu_bwd", "ffnn_colsum", "ffnn_transpose", "ffnn_to_bf16", "ffnn_mse",
           "ffnn_adam", "ffnn_error"]


class NNError(RuntimeError):
    pass


def build(force: bool = False) -> str:
    newest = max(os.path.getmtime(_SRC), os.path.getmtime(_HDR))
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < newest:
        subprocess.check_call(["nvcc"] + NVCC_FLAGS + ["-o", LIB_PATH, _SRC], cwd=os.path.dirname(_SRC))
    return LIB_PATH


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise NNError(f"{LIB_PATH} is missing: run __graft_entry__.build() first")
        L = ctypes.CDLL(LIB_PATH)
        vp, ci, cl, cf = ctypes.c_void_p, ctypes.c_int, ctypes.c_long, ctypes.c_float
        L.ffnn_gemm.argtypes = [vp, ci, vp, ci, ci, ci, ci, vp, ci, vp, ci, ci, vp, ci, ci, vp]
        L.ffnn_silu_bwd.argtypes = [vp, vp, cl, vp, vp, vp]
        L.ffnn_colsum.argtypes = [vp, ci, ci, ci, vp, vp]
        L.ffnn_transpose.argtypes = [vp, ci, ci, ci, vp, ci, ci, vp]
        L.ffnn_to_bf16.argtypes = [vp, cl, vp, vp]
        L.ffnn_mse.argtypes = [vp, ci, vp, ci, ci, vp, vp, vp, vp]
        L.ffnn_adam.argtypes = [vp, vp, vp, vp, cl, cf, cf, cf, cf, ci, cf, vp, vp, ci, vp]
        L.ffnn_error.argtypes = [ci]
        _LIB = L
    return _LIB


def _check(rc, what):
    if rc != 0:
        raise NNError(f"{what} failed with status {rc}")


def _ptr(t):
    return None if t is None else t.data_ptr()


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


def _rowmajor(t, name):
    if t.dim() != 2 or t.stride(1) != 1:
        raise NNError(f"{name}: expected a row-major 2-D tensor")
    return t.stride(0)


def gemm(A, B, *, bias=None, act=0, zf=None, yb=None, atomic=False, ksplit=0):
    """zf / yb <- A[M,K] @ B[N,K]^T (+ bias), BF16 operands, FP32 sums."""
    import torch
    if A.dtype != torch.bfloat16 or B.dtype != torch.bfloat16:
        raise NNError("gemm: operands must be bfloat16")
    M, K = A.shape
    N = B.shape[0]
    if B.shape[1] != K:
        raise NNError(f"gemm: K mismatch {A.shape} x {B.shape}")
    lda, ldb = _rowmajor(A, "A"), _rowmajor(B, "B")
    ldz = _rowmajor(zf, "zf") if zf is not None else 0
    ldy = _rowmajor(yb, "yb") if yb is not None else 0
    for t, n in ((zf, "zf"), (yb, "yb")):
        if t is not None and (t.shape[0] < M or t.shape[1] < N):
            raise NNError(f"gemm: {n} too small")
    if bias is not None and (bias.dtype != torch.float32 or bias.numel() < N):
        raise NNError("gemm: bias must be float32 [N]")
    _check(lib().ffnn_gemm(A.data_ptr(), lda, B.data_ptr(), ldb, M, N, K, _ptr(bias), act, _ptr(zf), ldz,
                           int(atomic), _ptr(yb), ldy, ksplit, _stream()), "ffnn_gemm")


def silu_bwd(dy, z, dzb=None, dzf=None):
    _check(lib().ffnn_silu_bwd(dy.data_ptr(), z.data_ptr(), z.numel(), _ptr(dzb), _ptr(dzf), _stream()),
           "ffnn_silu_bwd")


def colsum(x, out):
    rows, cols = x.shape
    _check(lib().ffnn_colsum(x.data_ptr(), rows, cols, _rowmajor(x, "x"), out.data_ptr(), _stream()),
           "ffnn_colsum")


def transpose(x, out, rows_pad=None):
    rows, cols = x.shape
    rows_pad = rows if rows_pad is None else rows_pad
    _check(lib().ffnn_transpose(x.data_ptr(), rows, cols, _rowmajor(x, "x"), out.data_ptr(), _rowmajor(out, "out"),
                                rows_pad, _stream()), "ffnn_transpose")


def to_bf16(x, out):
    _check(lib().ffnn_to_bf16(x.data_ptr(), x.numel(), out.data_ptr(), _stream()), "ffnn_to_bf16")


def mse(pred, tgt, grad, loss, gradf=None):
    rows, ld = pred.shape
    cols = tgt.shape[1]
    _check(lib().ffnn_mse(pred.data_ptr(), ld, tgt.data_ptr(), rows, cols, grad.data_ptr(), _ptr(gradf),
                          loss.data_ptr(), _stream()), "ffnn_mse")


def adam(w, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0, w16=None, w16t=None, rows=0):
    _check(lib().ffnn_adam(w.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), w.numel(), lr, b1, b2, eps, step,
                           wd, _ptr(w16), _ptr(w16t), rows, _stream()), "ffnn_adam")


def error(reset=True):
    rc = lib().ffnn_error(int(reset))
    if rc:
        raise NNError(f"a tensor-core kernel reported status {rc}")
