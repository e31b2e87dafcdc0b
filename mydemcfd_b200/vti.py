"""VTK ImageData output of the cell fields over the C ABI: the reference's
FileInOut::output_vti_binary_cellData (CFD/FileInOut.cpp:144-262), the same
file byte for byte.

The appended block (pressure, alpha, cell-centred velocity and IBM solid
fraction as Float32) is packed on the GPU (smac_vti_pack), copied to a
pinned host buffer on a copy stream, and written (smac_vti_write) by a
host thread, so that a time-stepping loop continues while the file is
written.  Two host buffers alternate; a third write waits for the first.
"""
from __future__ import annotations

import ctypes
import os
import threading

import torch

from . import _native as nat


def _ptr(t):
    if t is None:
        return None
    assert t.is_cuda and t.is_contiguous(), "device tensors must be contiguous CUDA tensors"
    return ctypes.c_void_p(t.data_ptr())


class VtiWriter:
    """write(step, p, alpha, vx, vy, vz, ibm_sf) -> <outdir>/result_<step:06d>.vti
    (the reference's file name).  p, alpha, ibm_sf: cell tensors, vx, vy, vz:
    face tensors in the reference layout; alpha / ibm_sf may be None (0).
    The fields may be overwritten as soon as write() returns: the packing has
    been queued on the current stream before them."""

    def __init__(self, N, h, outdir, origin=(0.0, 0.0, 0.0), device=None):
        self.N, self.h, self.origin = tuple(N), tuple(h), tuple(float(x) for x in origin)
        self.outdir = str(outdir)
        os.makedirs(self.outdir, exist_ok=True)
        self.desc = nat.GridDesc(*self.N, *self.h)
        nbytes = nat.load().smac_vti_block_bytes(ctypes.byref(self.desc))
        if nbytes == 0:
            raise nat.SmacError(nat.BAD_SHAPE, f"bad grid {self.N}")
        dev = torch.device("cuda") if device is None else device
        self.block = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        self.host = [torch.empty(nbytes, dtype=torch.uint8).pin_memory() for _ in range(2)]
        self.copy_stream = torch.cuda.Stream(device=dev)
        self.packed = torch.cuda.Event()
        self.copied = [torch.cuda.Event(), torch.cuda.Event()]
        self.threads = [None, None]
        self.errors = []
        self.count = 0

    def _write_file(self, slot, path):
        try:
            self.copied[slot].synchronize()
            o = (ctypes.c_double * 3)(*self.origin)
            nat.check(nat.load().smac_vti_write(ctypes.byref(self.desc), o, ctypes.c_void_p(self.host[slot].data_ptr()),
                                                path.encode()))
        except Exception as e:  # noqa: BLE001  (reported by wait())
            self.errors.append(e)

    def write(self, step, p, alpha, vx, vy, vz, ibm_sf=None):
        slot = self.count % 2
        self.count += 1
        if self.threads[slot] is not None:  # the buffer's previous file is written
            self.threads[slot].join()
        stream = torch.cuda.current_stream()
        # the device block is reused: the previous copy out of it has finished
        stream.wait_stream(self.copy_stream)
        nat.check(nat.load().smac_vti_pack(ctypes.byref(self.desc), _ptr(p), _ptr(alpha), _ptr(vx), _ptr(vy), _ptr(vz),
                                           _ptr(ibm_sf), _ptr(self.block), ctypes.c_void_p(stream.cuda_stream)))
        self.packed.record(stream)
        with torch.cuda.stream(self.copy_stream):
            self.copy_stream.wait_event(self.packed)
            self.host[slot].copy_(self.block, non_blocking=True)
            self.copied[slot].record(self.copy_stream)
        path = os.path.join(self.outdir, f"result_{int(step):06d}.vti")
        self.threads[slot] = threading.Thread(target=self._write_file, args=(slot, path), daemon=True)
        self.threads[slot].start()
        return path

    def wait(self):
        """Block until every queued file is written; raise the first error."""
        for t in self.threads:
            if t is not None:
                t.join()
        if self.errors:
            raise self.errors[0]
