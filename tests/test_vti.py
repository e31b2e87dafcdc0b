"""The VTI output (smac_vti_write) against the reference's own writer,
FileInOut::output_vti_binary_cellData, built from its source for the host
(oracle/_ref/libref_io.so) and run here: the files must be equal byte for
byte.  The appended block is packed by the numpy restatement in the oracle
(the GPU packing is tests/test_gpu_vti.py's)."""
import ctypes

import numpy as np
import pytest

from mydemcfd_b200 import _native as nat
from mydemcfd_b200 import build
from mydemcfd_b200 import workloads as W
from oracle import oracle as O
from oracle import ref as REF


@pytest.fixture(scope="module")
def lib():
    build.build()
    return nat.load()


def fields(N, seed):
    sh = W.shapes(N)
    r = lambda tag, key: W.uniform_pm1(W.substream(seed, tag), int(np.prod(sh[key]))).reshape(sh[key])  # noqa: E731
    return (r(1, "cell") * 1e3, np.abs(r(2, "cell")), r(3, "x"), r(4, "y"), r(5, "z"), np.abs(r(6, "cell")))


def write_ours(lib, N, h, origin, block, path):
    d = nat.GridDesc(*N, *h)
    buf = np.frombuffer(block, dtype=np.uint8).copy()
    o = (ctypes.c_double * 3)(*origin)
    nat.check(lib.smac_vti_write(ctypes.byref(d), o, ctypes.c_void_p(buf.ctypes.data), str(path).encode()))


@pytest.mark.skipif(not REF.io_available(), reason="reference writer oracle/_ref/libref_io.so not built")
@pytest.mark.parametrize("N,h,origin", [
    ((6, 5, 4), (0.1, 0.2, 0.3), (0.0, 0.0, 0.0)),
    ((17, 9, 12), (1.0 / 3.0, 0.125, 1e-3), (-0.5, 1.25, 3.0)),
])
def test_vti_file_equals_reference(lib, tmp_path, N, h, origin):
    p, a, vx, vy, vz, sf = fields(N, seed=3)
    ref = REF.write_vti(N, h, origin, p, a, vx, vy, vz, sf, tmp_path / "ref", 7)
    ours = tmp_path / "ours.vti"
    write_ours(lib, N, h, origin, O.vti_block(N, p, a, vx, vy, vz, sf), ours)
    assert open(ref, "rb").read() == open(ours, "rb").read()


def test_vti_block_bytes_and_refusals(lib):
    d = nat.GridDesc(4, 5, 6, 1.0, 1.0, 1.0)
    assert lib.smac_vti_block_bytes(ctypes.byref(d)) == 16 + 24 * 4 * 5 * 6
    bad = nat.GridDesc(0, 5, 6, 1.0, 1.0, 1.0)
    assert lib.smac_vti_block_bytes(ctypes.byref(bad)) == 0
    o = (ctypes.c_double * 3)(0.0, 0.0, 0.0)
    big = nat.GridDesc(1024, 1024, 1024, 1.0, 1.0, 1.0)  # velocity block over 2^32 bytes
    assert lib.smac_vti_write(ctypes.byref(big), o, ctypes.c_void_p(256), b"/nonexistent/x.vti") == nat.BAD_SHAPE
    assert lib.smac_vti_write(ctypes.byref(d), o, None, b"x.vti") == nat.BAD_ARG
