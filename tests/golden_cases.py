"""Case table of the golden fixtures (tests/golden/reference_outputs.npz) and
the helpers that rebuild each case's input and read its output.

A case is a full aoclfftz descriptor: dtype, transform type (0 c2c, 1 real),
direction, placement, dims and vecs as (n, in_stride, out_stride), dims[0]
innermost, plus the seed of its synthetic input.
"""
import numpy as np

from aoclfftz_b200 import synthetic
from fftz_helpers import cplx_dtype, gather, real_dtype, scatter, span


def _c2c(name, dtype, dims, vecs, d=0, pl=1, seed=11):
    return dict(name=name, dtype=dtype, type=0, dir=d, placement=pl, dims=dims, vecs=vecs, seed=seed)


def _real(name, dtype, shape, batch, d, inplace=False, seed=13):
    rdims = list(reversed(shape))
    n0 = rdims[0]
    h0 = n0 // 2 + 1
    rrow = 2 * h0 if inplace else n0
    r_str, c_str = [1], [1]
    for i in range(1, len(rdims)):
        r_str.append(r_str[-1] * (rrow if i == 1 else rdims[i - 1]))
        c_str.append(c_str[-1] * (h0 if i == 1 else rdims[i - 1]))
    rtot = r_str[-1] * (rrow if len(rdims) == 1 else rdims[-1])
    ctot = c_str[-1] * (h0 if len(rdims) == 1 else rdims[-1])
    if d == 0:
        dims = [(rdims[i], r_str[i], c_str[i]) for i in range(len(rdims))]
        vecs = [(batch, rtot, ctot)]
    else:
        dims = [(rdims[i], c_str[i], r_str[i]) for i in range(len(rdims))]
        vecs = [(batch, ctot, rtot)]
    return dict(name=name, dtype=dtype, type=1, dir=d, placement=0 if inplace else 1, dims=dims, vecs=vecs,
                seed=seed)


CASES = []
for dt in ("f32", "f64"):
    for n in (8, 64, 512, 1024, 4096):  # pow2 iterative / four-step in the reference
        CASES.append(_c2c("pow2_%d_%s" % (n, dt), dt, [(n, 1, 1)], [(2, n, n)], 0))
        CASES.append(_c2c("pow2_%d_%s_bwd" % (n, dt), dt, [(n, 1, 1)], [(2, n, n)], 1))
    for n in (6, 15, 60, 210, 1000, 2310):  # Cooley-Tukey over radices 2..13
        CASES.append(_c2c("ct_%d_%s" % (n, dt), dt, [(n, 1, 1)], [(3, n, n)], 0))
    for n in (17, 97, 251, 1009):  # Bluestein primes
        CASES.append(_c2c("blue_%d_%s" % (n, dt), dt, [(n, 1, 1)], [(1, n, n)], 0))
        CASES.append(_c2c("blue_%d_%s_bwd" % (n, dt), dt, [(n, 1, 1)], [(1, n, n)], 1))
    CASES.append(_c2c("colmajor_64x8_%s" % dt, dt, [(64, 8, 8)], [(8, 1, 1)], 0))
    CASES.append(_c2c("strided_100_%s" % dt, dt, [(100, 2, 3)], [(5, 300, 400)], 0))
    CASES.append(_c2c("inplace_128_%s" % dt, dt, [(128, 1, 1)], [(4, 130, 130)], 1, pl=0))
    CASES.append(_c2c("nd_16x8_%s" % dt, dt, [(16, 1, 1), (8, 16, 16)], [(2, 128, 128)], 0))
    CASES.append(_c2c("nd_5x6x7_%s" % dt, dt, [(5, 1, 1), (6, 5, 5), (7, 30, 30)], [(1, 210, 210)], 0))
    for n in (16, 50, 1024):
        CASES.append(_real("r2c_%d_%s" % (n, dt), dt, [n], 2, 0))
        CASES.append(_real("c2r_%d_%s" % (n, dt), dt, [n], 2, 1))
    CASES.append(_real("r2c_inplace_50_%s" % dt, dt, [50], 4, 0, inplace=True))
    CASES.append(_real("r2c_3d_8x8x16_%s" % dt, dt, [8, 8, 16], 1, 0))
    CASES.append(_real("c2r_3d_8x8x16_%s" % dt, dt, [8, 8, 16], 1, 1))
    CASES.append(_real("r2c_3d_inplace_8x12x32_%s" % dt, dt, [8, 12, 32], 1, 0, inplace=True))


def in_is_complex(c):
    return c["type"] == 0 or c["dir"] == 1


def out_is_complex(c):
    return c["type"] == 0 or c["dir"] == 0


def half(c):
    return c["dims"][0][0] // 2 + 1


def lshape(c, n0=None):
    dims = [d[0] for d in c["dims"]]
    if n0 is not None:
        dims[0] = n0
    return [v[0] for v in reversed(c["vecs"])] + list(reversed(dims))


def logical_input(c):
    """The case's logical input array [vecs..., dims reversed...]."""
    dt = c["dtype"]
    if c["type"] == 0:
        shp = lshape(c)
        return synthetic.complex_uniform(c["seed"], int(np.prod(shp)), cplx_dtype(dt)).reshape(shp)
    rshape = lshape(c)
    x = synthetic.normal(c["seed"], int(np.prod(rshape))).reshape(rshape)
    if c["dir"] == 0:
        return x.astype(real_dtype(dt))
    # c2r input: the half spectrum of a real signal (Hermitian-consistent)
    import oracle
    rank = len(c["dims"])
    return oracle.rfftn(x, rank=rank).astype(cplx_dtype(dt))


def in_scalars(c):
    n0 = half(c) if (c["type"] == 1 and c["dir"] == 1) else None
    s = span(c["dims"], c["vecs"], "in", n0=n0)
    return 2 * s if in_is_complex(c) else s


def out_scalars(c):
    n0 = half(c) if (c["type"] == 1 and c["dir"] == 0) else None
    s = span(c["dims"], c["vecs"], "out", n0=n0)
    return 2 * s if out_is_complex(c) else s


def case_input(c):
    """Raw input buffer (real scalar view) of the case."""
    x = logical_input(c)
    n0 = half(c) if (c["type"] == 1 and c["dir"] == 1) else None
    total = in_scalars(c)
    if c["placement"] == 0:
        total = max(total, out_scalars(c))
    return scatter(x, [(d[0], d[1]) for d in c["dims"]], [(v[0], v[1]) for v in c["vecs"]], total, c["dtype"],
                   complex_side=in_is_complex(c), n0=n0)


def logical_output(c, raw):
    n0 = half(c) if (c["type"] == 1 and c["dir"] == 0) else None
    return gather(np.asarray(raw), [(d[0], d[2]) for d in c["dims"]], [(v[0], v[2]) for v in c["vecs"]], c["dtype"],
                  complex_side=out_is_complex(c), n0=n0)


def oracle_output(c):
    """FP64 oracle result of the case (restated algorithms)."""
    import oracle
    x = logical_input(c)
    rank = len(c["dims"])
    if c["type"] == 0:
        y = np.asarray(x, dtype=np.complex128)
        sign = -1 if c["dir"] == 0 else +1
        for k in range(rank):
            ax = y.ndim - 1 - k
            y = np.moveaxis(oracle.fft(np.moveaxis(y, ax, -1), sign=sign), -1, ax)
        return y
    if c["dir"] == 0:
        return oracle.rfftn(np.asarray(x, dtype=np.float64), rank=rank)
    return oracle.irfftn(np.asarray(x, dtype=np.complex128), c["dims"][0][0], rank=rank)


def tolerance(c):
    import oracle
    N = int(np.prod([d[0] for d in c["dims"]]))
    return oracle.tol(N, c["dtype"])
