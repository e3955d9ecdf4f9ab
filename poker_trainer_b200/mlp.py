"""The leaf-value network over libdcfr's dcfr_mlp_* entry points.

The network is trained and evaluated by the library's own BF16 tcgen05 GEMM
kernels (FP32 accumulation, FP32 master weights, Adam). torch tensors are
used here only to hold device memory; every computation runs in libdcfr.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .solver import check, lib


def _dev(t):
    """Device pointer of a contiguous CUDA float32 torch tensor."""
    import torch
    assert t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
    return C.c_void_p(t.data_ptr())


def _bind():
    L = lib()
    if getattr(L, "_mlp_bound", False):
        return L
    P = C.c_void_p
    L.dcfr_mlp_create.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.POINTER(P)]
    L.dcfr_mlp_destroy.argtypes = [P]
    L.dcfr_mlp_destroy.restype = None
    L.dcfr_mlp_num_params.argtypes = [P, C.POINTER(C.c_uint64)]
    L.dcfr_mlp_get_params.argtypes = [P, P]
    L.dcfr_mlp_set_params.argtypes = [P, P]
    L.dcfr_mlp_forward.argtypes = [P, P, C.c_int32, P]
    L.dcfr_mlp_gradients.argtypes = [P, P, P, P, C.c_int32, C.POINTER(C.c_float), P]
    L.dcfr_mlp_train_step.argtypes = [P, P, P, P, C.c_int32, C.c_float, C.POINTER(C.c_float)]
    L.dcfr_mlp_backward.argtypes = [P, P, P, P, C.c_int32, C.POINTER(C.c_float)]
    L.dcfr_mlp_gradients_device.argtypes = [P, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]
    L.dcfr_mlp_adam_step.argtypes = [P, C.c_float, C.c_float]
    L.dcfr_gemm_bf16.argtypes = [P, P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P, P, C.c_int32, P]
    L.dcfr_gemm_bf16_timed.argtypes = [P, P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P, P, C.c_int32,
                                       C.c_int32, P, C.POINTER(C.c_float)]
    L._mlp_bound = True
    return L


def pad128(x: int) -> int:
    return (x + 127) // 128 * 128


class LeafNet:
    """MLP in_dim -> layers x hidden (GELU) -> out_dim."""

    def __init__(self, in_dim: int, hidden: int = 1024, layers: int = 4, out_dim: int = 2652, max_batch: int = 1024,
                 seed: int = 0):
        L = _bind()
        h = C.c_void_p()
        check(L.dcfr_mlp_create(in_dim, hidden, layers, out_dim, max_batch, seed, C.byref(h)))
        self._h = h
        self.in_dim, self.hidden, self.layers, self.out_dim, self.max_batch = in_dim, hidden, layers, out_dim, max_batch
        n = C.c_uint64()
        check(L.dcfr_mlp_num_params(h, C.byref(n)))
        self.num_params = n.value
        self.kin = [pad128(in_dim)] + [hidden] * layers
        self.nout = [hidden] * layers + [pad128(out_dim)]

    def close(self):
        if getattr(self, "_h", None):
            lib().dcfr_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def params(self) -> np.ndarray:
        out = np.zeros(self.num_params, np.float32)
        check(lib().dcfr_mlp_get_params(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def set_params(self, flat: np.ndarray):
        flat = np.ascontiguousarray(flat, np.float32)
        assert flat.size == self.num_params
        check(lib().dcfr_mlp_set_params(self._h, flat.ctypes.data_as(C.c_void_p)))

    def split(self, flat: np.ndarray):
        """Views of a flat parameter (or gradient) vector: [(W_t, b)] per layer,
        W_t padded [nout][kin]."""
        out, off = [], 0
        ws = []
        for k, n in zip(self.kin, self.nout):
            ws.append(flat[off:off + n * k].reshape(n, k))
            off += n * k
        for i, n in enumerate(self.nout):
            out.append((ws[i], flat[off:off + n]))
            off += n
        return out

    def forward(self, x):
        import torch
        torch.cuda.synchronize()
        y = torch.empty((x.shape[0], self.out_dim), dtype=torch.float32, device=x.device)
        check(lib().dcfr_mlp_forward(self._h, _dev(x), x.shape[0], _dev(y)))
        return y

    def gradients(self, x, target, mask=None):
        import torch
        torch.cuda.synchronize()
        loss = C.c_float()
        g = np.zeros(self.num_params, np.float32)
        check(lib().dcfr_mlp_gradients(self._h, _dev(x), _dev(target), _dev(mask) if mask is not None else None,
                                       x.shape[0], C.byref(loss), g.ctypes.data_as(C.c_void_p)))
        return loss.value, g

    def backward(self, x, target, mask=None) -> float:
        """Loss of this batch; its gradients stay on the device
        (grad_tensor), for a data-parallel sum before adam_step."""
        import torch
        torch.cuda.synchronize()
        loss = C.c_float()
        check(lib().dcfr_mlp_backward(self._h, _dev(x), _dev(target), _dev(mask) if mask is not None else None,
                                      x.shape[0], C.byref(loss)))
        return loss.value

    def grad_tensor(self):
        """The library's flat gradient buffer as a CUDA float32 torch tensor
        (a view, no copy; valid while the network lives)."""
        import torch
        ptr = C.c_void_p()
        n = C.c_uint64()
        check(lib().dcfr_mlp_gradients_device(self._h, C.byref(ptr), C.byref(n)))
        return torch.as_tensor(_DeviceArray(ptr.value, n.value), device="cuda")

    def adam_step(self, lr: float = 1e-3, grad_scale: float = 1.0):
        """One Adam step on the device gradients times grad_scale."""
        import torch
        torch.cuda.synchronize()
        check(lib().dcfr_mlp_adam_step(self._h, lr, grad_scale))

    def train_step(self, x, target, mask=None, lr: float = 1e-3) -> float:
        import torch
        torch.cuda.synchronize()
        loss = C.c_float()
        check(lib().dcfr_mlp_train_step(self._h, _dev(x), _dev(target), _dev(mask) if mask is not None else None,
                                        x.shape[0], lr, C.byref(loss)))
        return loss.value


class _DeviceArray:
    """A device buffer owned by the library, exposed to torch without a copy
    (the CUDA array interface)."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f4", "data": (ptr, False), "version": 3,
                                         "strides": None, "stream": None}


def gemm_bf16(a, b, epi: int = 0, bias=None, z=None):
    """c = epi(a @ b^T) with the library's tensor-core kernel; a [m][k] and
    b [n][k] are CUDA bfloat16 tensors."""
    import torch
    L = _bind()
    m, k = a.shape
    n = b.shape[0]
    out_dtype = torch.float32 if epi in (0, 1) else torch.bfloat16
    c = torch.empty((m, n), dtype=out_dtype, device=a.device)
    if epi == 2 and z is None:
        z = torch.empty((m, n), dtype=torch.bfloat16, device=a.device)
    torch.cuda.synchronize()
    check(L.dcfr_gemm_bf16(C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), C.c_void_p(c.data_ptr()), m, n, k, epi,
                           C.c_void_p(bias.data_ptr()) if bias is not None else None,
                           C.c_void_p(z.data_ptr()) if z is not None else None, n, None))
    return c, z


def gemm_time(m: int, n: int, k: int, reps: int = 50, epi: int = 0, seed: int = 0) -> float:
    """Milliseconds per launch of the library's GEMM on an [m][k] x [n][k]^T
    product with epilogue `epi` (dcfr_gemm_bf16_timed: CUDA events around
    `reps` back-to-back launches on the current stream, after 3 warm-up
    launches)."""
    import torch
    L = _bind()
    g = torch.Generator(device="cuda").manual_seed(seed)
    a = torch.randn(m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    bias = torch.randn(n, device="cuda", generator=g)
    c = torch.empty((m, n), dtype=torch.float32 if epi in (0, 1) else torch.bfloat16, device="cuda")
    z = torch.randn(m, n, device="cuda", generator=g).to(torch.bfloat16) if epi in (2, 3) else None
    stream = torch.cuda.current_stream()
    args = (C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), C.c_void_p(c.data_ptr()), m, n, k, epi,
            C.c_void_p(bias.data_ptr()) if epi in (1, 2) else None, C.c_void_p(z.data_ptr()) if z is not None else None,
            n)
    ms = C.c_float()
    torch.cuda.synchronize()
    check(L.dcfr_gemm_bf16_timed(*args, 3, C.c_void_p(stream.cuda_stream), C.byref(ms)))
    check(L.dcfr_gemm_bf16_timed(*args, reps, C.c_void_p(stream.cuda_stream), C.byref(ms)))
    return ms.value


def main():
    import argparse
    import json
    ap = argparse.ArgumentParser(description="Times the library's BF16 tcgen05 GEMM (dcfr_gemm_bf16).")
    ap.add_argument("m", type=int)
    ap.add_argument("n", type=int)
    ap.add_argument("k", type=int)
    ap.add_argument("--reps", type=int, default=50)
    ap.add_argument("--epi", type=int, default=0, help="0 plain, 1 +bias, 2 +bias GELU, 3 x GELU'(z)")
    args = ap.parse_args()
    ms = gemm_time(args.m, args.n, args.k, args.reps, args.epi)
    print(json.dumps({"m": args.m, "n": args.n, "k": args.k, "epi": args.epi, "ms": ms,
                      "tflops": 2.0 * args.m * args.n * args.k / (ms * 1e-3) / 1e12}))


if __name__ == "__main__":
    main()
