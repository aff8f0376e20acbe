"""The reference's kernel-call surface, served by libugks_b200.so.

pyUGKS launches every kernel as ``self.prg.<name>(queue, global_size,
local_size, *args)`` on a per-block ``cl.Program`` (``ugks_block.py:184``).
``KernelProgram`` keeps that surface: attribute names are the reference kernel
names, arguments come in the reference order, buffers are torch CUDA tensors
in the reference layout and scalars are Python ints / floats.  Each call
forwards to ``ugks_<name>(desc, g0, g1, *args, stream)``; the per-block
``ugks_block_desc`` takes the place of the generated OpenCL header.

``queue`` is a ``torch.cuda.Stream`` (or None for the current stream);
``local_size`` is accepted and ignored (the CUDA launch shape is fixed by the
library).
"""
from __future__ import annotations

import ctypes as C

from . import _lib


class KernelProgram:
    def __init__(self, desc: "_lib.BlockDesc"):
        self.desc = desc
        self._lib = _lib.lib()
        self._calls = {}

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        if name not in _lib.KERNEL_SIGNATURES:
            raise AttributeError("no kernel %r in the UGKS program" % name)
        call = self._calls.get(name)
        if call is None:
            call = self._make(name)
            self._calls[name] = call
        return call

    def _make(self, name):
        fn = getattr(self._lib, "ugks_" + name)
        sig = _lib.KERNEL_SIGNATURES[name]
        desc = C.byref(self.desc)

        def call(queue, global_size, local_size, *args):
            if len(args) != len(sig):
                raise TypeError("%s takes %d kernel arguments, got %d" % (name, len(sig), len(args)))
            conv = []
            for k, a in zip(sig, args):
                if k == "p":
                    if not a.is_cuda or not a.is_contiguous():
                        raise ValueError("%s: buffers must be contiguous CUDA tensors" % name)
                    conv.append(a.data_ptr())
                elif k == "i":
                    conv.append(int(a))
                else:
                    conv.append(float(a))
            g0 = int(global_size[0])
            g1 = int(global_size[1]) if len(global_size) > 1 else 1
            _lib.check(fn(desc, g0, g1, *conv, _stream_ptr(queue)), name)

        call.__name__ = name
        return call


def _stream_ptr(queue):
    import torch
    if queue is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(queue, int):
        return queue
    return queue.cuda_stream
