"""VTI output on the GPU: smac_vti_pack + one copy + smac_vti_write, and the
asynchronous VtiWriter, against the reference's own writer run on the host
(oracle/_ref/libref_io.so): the files must be equal byte for byte."""
import ctypes
import time

import numpy as np
import pytest
import torch

from mydemcfd_b200 import _native as nat
from mydemcfd_b200 import workloads as W
from mydemcfd_b200.vti import VtiWriter
from oracle import ref as REF

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not REF.io_available(), reason="reference writer oracle/_ref/libref_io.so not built")]


def fields(N, seed):
    sh = W.shapes(N)
    r = lambda tag, key: W.uniform_pm1(W.substream(seed, tag), int(np.prod(sh[key]))).reshape(sh[key])  # noqa: E731
    return (r(1, "cell") * 1e3, np.abs(r(2, "cell")), r(3, "x"), r(4, "y"), r(5, "z"), np.abs(r(6, "cell")))


def _cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("N,h,origin", [
    ((24, 24, 24), (1.0 / 24,) * 3, (0.0, 0.0, 0.0)),
    ((33, 17, 9), (0.1, 0.05, 0.2), (1.5, -2.0, 0.25)),
])
def test_vti_pack_and_write_equal_reference(tmp_path, N, h, origin):
    f = fields(N, seed=5)
    ref = REF.write_vti(N, h, origin, *f, tmp_path / "ref", 3)
    d = nat.GridDesc(*N, *h)
    lib = nat.load()
    block = torch.empty(lib.smac_vti_block_bytes(ctypes.byref(d)), dtype=torch.uint8, device="cuda")
    dev = [_cuda(a) for a in f]
    nat.check(lib.smac_vti_pack(ctypes.byref(d), *(ctypes.c_void_p(t.data_ptr()) for t in dev),
                                ctypes.c_void_p(block.data_ptr()),
                                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    host = block.cpu().numpy()
    path = tmp_path / "ours.vti"
    nat.check(lib.smac_vti_write(ctypes.byref(d), (ctypes.c_double * 3)(*origin), ctypes.c_void_p(host.ctypes.data),
                                 str(path).encode()))
    assert open(ref, "rb").read() == open(path, "rb").read()


def test_vti_writer_three_steps_equal_reference(tmp_path):
    """Three steps through the asynchronous writer (two host buffers, the
    third write reuses the first), the device fields overwritten right after
    each write() call."""
    N, h = (40, 32, 24), (0.025, 0.03125, 1.0 / 24)
    w = VtiWriter(N, h, tmp_path / "ours", origin=(0.1, 0.2, 0.3))
    dev = None
    paths = []
    for step in range(3):
        f = fields(N, seed=10 + step)
        if dev is None:
            dev = [_cuda(a) for a in f]
        else:
            for t, a in zip(dev, f):
                t.copy_(torch.from_numpy(a))
        paths.append((w.write(step, *dev), f))
    w.wait()
    for step, (path, f) in enumerate(paths):
        ref = REF.write_vti(N, h, (0.1, 0.2, 0.3), *f, tmp_path / "ref", step)
        assert open(ref, "rb").read() == open(path, "rb").read(), step


def test_vti_output_time_256(tmp_path):
    """The device side (pack + copy of 24 B per cell) and the whole call at
    256^3, beside the reference's host writer on the same fields (which in
    the reference follows a copy of every grid member to the host)."""
    N, h = (256, 256, 256), (1.0 / 256,) * 3
    f = fields(N, seed=2)
    t0 = time.perf_counter()
    REF.write_vti(N, h, (0.0, 0.0, 0.0), *f, tmp_path / "ref", 0)
    ref_s = time.perf_counter() - t0
    dev = [_cuda(a) for a in f]
    w = VtiWriter(N, h, tmp_path / "ours")
    w.write(0, *dev)
    w.wait()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    w.write(1, *dev)
    t_return = time.perf_counter() - t0
    w.wait()
    t_all = time.perf_counter() - t0
    print(f"VTI 256^3: write() returns after {t_return * 1e3:.1f} ms, file on disk after {t_all * 1e3:.1f} ms; "
          f"reference host writer {ref_s * 1e3:.1f} ms")
