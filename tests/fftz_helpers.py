"""Helpers shared by the tests: run one problem through the GPU library's C ABI
(device or host buffers) or through the reference library, and build the
numpy views needed to compare them with the oracle."""
import ctypes as C

import numpy as np

import aoclfftz_b200
from aoclfftz_b200 import abi


def real_dtype(dtype):
    return np.float32 if dtype == "f32" else np.float64


def cplx_dtype(dtype):
    return np.complex64 if dtype == "f32" else np.complex128


def span(dims, vecs, side, n0=None):
    """Scalar elements spanned by one side ('in'/'out') of a descriptor, in the
    side's element units (complex or real)."""
    s = 1
    for i, (n, is_, os_) in enumerate(dims):
        if i == 0 and n0 is not None:
            n = n0
        s += (n - 1) * (is_ if side == "in" else os_)
    for (n, is_, os_) in vecs:
        if n > 0:
            s += (n - 1) * (is_ if side == "in" else os_)
    return s


def run_gpu(dtype, dims, vecs, x_in, out_scalars, fft_type=0, direction=0, placement=1, host=False, ilp64=False,
            repeat=1, lib=None, pinned=False):
    """Executes one problem on the GPU through aoclfftz_setup_* / execute.

    x_in: raw input buffer (numpy; viewed as the real scalar type).
    out_scalars: real scalars of the output buffer. Returns (out_raw, plan_text).
    With host=True the library receives host pointers and stages them itself.
    """
    import torch
    lib = lib or aoclfftz_b200.load()
    real = real_dtype(dtype)
    xin = np.ascontiguousarray(x_in).view(real).ravel()
    tdt = torch.float32 if dtype == "f32" else torch.float64
    outs = []
    if host and pinned:
        # page-locked host memory: the library pipelines copy-in / passes / copy-out
        if placement == 0:
            t = torch.zeros(max(xin.size, out_scalars), dtype=tdt).pin_memory()
            buf = t.numpy()
            buf[: xin.size] = xin
            pin = pout = buf.ctypes.data
            hold = [buf, t]
        else:
            ti = torch.from_numpy(xin.copy()).pin_memory()
            to = torch.zeros(out_scalars, dtype=tdt).pin_memory()
            hin, hout = ti.numpy(), to.numpy()
            pin, pout = hin.ctypes.data, hout.ctypes.data
            hold = [hin, hout, ti, to]
    elif host:
        if placement == 0:
            buf = np.zeros(max(xin.size, out_scalars), dtype=real)
            buf[: xin.size] = xin
            pin = pout = buf.ctypes.data
            hold = [buf]
        else:
            hin = xin.copy()
            hout = np.zeros(out_scalars, dtype=real)
            pin, pout = hin.ctypes.data, hout.ctypes.data
            hold = [hin, hout]
    else:
        if placement == 0:
            d = torch.zeros(max(xin.size, out_scalars), dtype=tdt, device="cuda")
            d[: xin.size] = torch.from_numpy(xin).to("cuda")
            pin = pout = d.data_ptr()
            hold = [d]
        else:
            din = torch.from_numpy(xin.copy()).to("cuda")
            dout = torch.zeros(out_scalars, dtype=tdt, device="cuda")
            pin, pout = din.data_ptr(), dout.data_ptr()
            hold = [din, dout]
    desc, keep = abi.make_desc(pin, pout, dims, vecs, fft_type, direction, placement, ilp64=ilp64)
    h = abi.setup(lib, desc, dtype, ilp64=ilp64)
    if not h:
        raise RuntimeError("GPU setup failed: %s" % lib.aoclfftz_gpu_last_error().decode())
    try:
        txt = C.create_string_buffer(2048)
        lib.aoclfftz_gpu_describe(h, txt, 2048)
        for _ in range(repeat):
            if placement == 0 and not host and repeat > 1:
                hold[0][: xin.size] = torch.from_numpy(xin).to("cuda")
            elif placement == 0 and host and repeat > 1:
                hold[0][: xin.size] = xin
            rc = lib.aoclfftz_execute(h)
            if rc != 0:
                raise RuntimeError("GPU execute failed (%d): %s" % (rc, lib.aoclfftz_gpu_last_error().decode()))
            assert lib.aoclfftz_gpu_synchronize(h) == 0
            if host:
                o = (hold[0] if placement == 0 else hold[1])[:out_scalars].copy()
            else:
                o = (hold[0] if placement == 0 else hold[1])[:out_scalars].cpu().numpy().copy()
            outs.append(o)
    finally:
        lib.aoclfftz_destroy(h)
    return (outs[0] if repeat == 1 else outs), txt.value.decode()


def gather(raw, dims_side, vecs_side, dtype, complex_side=True, n0=None):
    """Collects the logical array [vec..., dim_{r-1}, ..., dim_0] from a raw
    strided buffer. dims_side/vecs_side: lists of (n, stride)."""
    arr = raw.view(cplx_dtype(dtype)) if complex_side else raw
    shape, strides = [], []
    for (n, s) in reversed(vecs_side):
        shape.append(n)
        strides.append(s)
    for i, (n, s) in reversed(list(enumerate(dims_side))):
        shape.append(n0 if (i == 0 and n0 is not None) else n)
        strides.append(s)
    idx = np.zeros(shape, dtype=np.int64)
    for ax, (n, s) in enumerate(zip(shape, strides)):
        sh = [1] * len(shape)
        sh[ax] = n
        idx = idx + (np.arange(n, dtype=np.int64) * s).reshape(sh)
    return arr[idx]


def scatter(values, dims_side, vecs_side, total, dtype, complex_side=True, n0=None):
    """Inverse of gather: places a logical array into a raw buffer of `total`
    scalars (zeros elsewhere)."""
    if complex_side:
        buf = np.zeros(total // 2, dtype=cplx_dtype(dtype))
    else:
        buf = np.zeros(total, dtype=real_dtype(dtype))
    shape, strides = [], []
    for (n, s) in reversed(vecs_side):
        shape.append(n)
        strides.append(s)
    for i, (n, s) in reversed(list(enumerate(dims_side))):
        shape.append(n0 if (i == 0 and n0 is not None) else n)
        strides.append(s)
    idx = np.zeros(shape, dtype=np.int64)
    for ax, (n, s) in enumerate(zip(shape, strides)):
        sh = [1] * len(shape)
        sh[ax] = n
        idx = idx + (np.arange(n, dtype=np.int64) * s).reshape(sh)
    buf[idx] = values
    return buf.view(real_dtype(dtype))
