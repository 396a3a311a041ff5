"""The CUDA backend: device, state precision and the loaded C ABI.

Stands in for ``CUDABackend`` (frfs/backends/cuda/base.py:10-102) on the
path the DGFS system uses: it owns device memory (torch allocations made
once at set-up), the precision from ``[backend] precision``, and the
stream every kernel is launched on.  There is no CPU path: constructing it
without a CUDA device or without libbdgfs.so raises.
"""
import torch

from . import _lib


class CUDABackend:
    name = 'cuda'

    def __init__(self, cfg=None, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError('frfs_b200 needs a CUDA device (sm_100a)')
        prec = cfg.get('backend', 'precision', 'single') if cfg is not None else 'single'
        if prec not in ('single', 'double'):
            raise ValueError('Invalid floating point data type')
        self.fpdtype = torch.float32 if prec == 'single' else torch.float64
        self.device = torch.device(device if device is not None else 'cuda', )
        if self.device.index is None:
            self.device = torch.device('cuda', torch.cuda.current_device())
        _lib.lib()          # fail loudly now if the native library is absent
        self.stream = torch.cuda.current_stream(self.device)

    def zeros(self, *shape, dtype=None):
        return torch.zeros(*shape, dtype=dtype or self.fpdtype, device=self.device)

    def empty(self, *shape, dtype=None):
        return torch.empty(*shape, dtype=dtype or self.fpdtype, device=self.device)

    def const(self, array, dtype=None):
        return torch.as_tensor(array, dtype=dtype or self.fpdtype).to(self.device).contiguous()
