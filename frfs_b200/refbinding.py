"""ctypes binding of the collision entry points of libbdgfs, written for the
reference solver's side.

This file is the stub a maintainer of the reference would drop in as
``frfs/solvers/dgfs/bdgfs.py``: it depends on ``ctypes`` alone, like the
reference's own cuFFT binding (``frfs/solvers/dgfs/cufft.py:15-46``), and its
status-to-exception map follows ``cufft.py:91-120``.  The structures mirror
``include/bdgfs.h`` field for field; a test compiles the header with a C
compiler and compares every offset and size, and another checks that the
integration notes show this file verbatim.

Caller in the reference: ``DGFSSystem.collide`` (``solvers/dgfs/system.py:
199-218``) replaces its per-DOF ``self.sm.fs(...)`` loop with one
``vhs_collide`` over all DOFs; ``DGFSBiSystem.collide``
(``solvers/dgfsbi/system.py:241-252``) does the same with ``vss_collide``.
"""
import ctypes as C


class VhsGrid(C.Structure):             # bdgfs_vhs_grid
    _fields_ = [('Nv', C.c_int32), ('Nrho', C.c_int32), ('M', C.c_int32),
                ('fp64', C.c_int32), ('tile', C.c_int32), ('pad_', C.c_int32),
                ('prefac', C.c_double), ('cw', C.c_double),
                ('phase', C.c_void_p), ('gw', C.c_void_p), ('bb2', C.c_void_p),
                ('c0', C.c_void_p), ('ginv', C.c_void_p)]


class VhsBatch(C.Structure):            # bdgfs_vhs_batch
    _fields_ = [('grid', C.c_int32), ('pad_', C.c_int32), ('ndof', C.c_int64),
                ('f', C.c_void_p), ('Q', C.c_void_p), ('moments', C.c_void_p),
                ('index', C.c_void_p), ('count', C.c_void_p)]


class VssArgs(C.Structure):             # bdgfs_vss_args
    _fields_ = [('Nv', C.c_int32), ('nspcs', C.c_int32), ('Nrho', C.c_int32),
                ('M', C.c_int32), ('ndof', C.c_int64), ('fp64', C.c_int32),
                ('pad_', C.c_int32), ('f', C.c_void_p * 4), ('Q', C.c_void_p * 4),
                ('mfrac', C.c_void_p), ('prefac', C.c_void_p), ('rfac', C.c_void_p),
                ('rw', C.c_void_p), ('sz', C.c_void_p), ('b', C.c_void_p),
                ('c', C.c_void_p)]


# include/bdgfs.h status codes
STATUS = {-1: 'invalid argument', -2: 'CUDA error', -3: 'unsupported grid/precision',
          -4: 'bounded device wait timed out', -5: 'scratch buffer too small'}


class BdgfsError(RuntimeError):
    pass


def check(rc, what):
    """Raise for a non-zero status, as the reference's cuFFT binding does."""
    if rc != 0:
        raise BdgfsError(f'{what}: {STATUS.get(rc, "unknown status")} ({rc})')


# (restype, argtypes) of each entry point bound here, in header order
SIGNATURES = {
    'bdgfs_vhs_scratch_bytes': (C.c_size_t, [C.POINTER(VhsGrid), C.c_int32, C.c_int32]),
    'bdgfs_vhs_collide': (C.c_int32, [C.POINTER(VhsGrid), C.c_int32, C.POINTER(VhsBatch),
                                      C.c_int32, C.c_int32, C.c_void_p, C.c_size_t,
                                      C.c_void_p, C.c_void_p]),
    'bdgfs_vhs_collide_static': (C.c_int32, [C.POINTER(VhsGrid), C.c_int32,
                                             C.POINTER(VhsBatch), C.c_int32, C.c_int32,
                                             C.c_void_p]),
    'bdgfs_vss_scratch_bytes': (C.c_size_t, [C.c_int32, C.c_int32, C.c_int32]),
    'bdgfs_vss_collide': (C.c_int32, [C.POINTER(VssArgs), C.c_void_p, C.c_size_t,
                                      C.c_void_p]),
}


def load(path='libbdgfs.so'):
    """Open the library and declare the entry points above."""
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    return lib
