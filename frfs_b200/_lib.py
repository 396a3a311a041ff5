"""ctypes binding of ``libbdgfs.so`` (the C ABI declared in include/bdgfs.h).

The library is loaded from the package's ``_lib`` directory.  There is no
fallback: every product entry point raises if the library is missing or a
call returns a non-zero status.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, '_lib', 'libbdgfs.so')

BDGFS_OK = 0
_ERRORS = {-1: 'invalid argument', -2: 'CUDA error', -3: 'unsupported grid/precision',
           -4: 'bounded device wait timed out', -5: 'scratch buffer too small'}

# Every symbol include/bdgfs.h declares (tests check the export list).
EXPORTS = (
    'bdgfs_vhs_scratch_bytes', 'bdgfs_vhs_collide', 'bdgfs_vhs_tiles', 'bdgfs_fma_probe',
    'bdgfs_vhs_collide_static', 'bdgfs_wait_probe',
    'bdgfs_fr_disu', 'bdgfs_fr_invmass', 'bdgfs_fr_bc_update', 'bdgfs_fr_rhs', 'bdgfs_fr_rhs_gather',
    'bdgfs_fr_bc_update_gather', 'bdgfs_fr_rhs_tensor',
    'bdgfs_moments', 'bdgfs_residual', 'bdgfs_status_check',
    'bdgfs_gemm', 'bdgfs_colsum', 'bdgfs_adamw', 'bdgfs_relmse',
    'bdgfs_hybrid_classify', 'bdgfs_hybrid_project', 'bdgfs_hybrid_scatter',
    'bdgfs_hybrid_project_scatter', 'bdgfs_hybrid_heads', 'bdgfs_hybrid_shift',
    'bdgfs_hybrid_tfeatures', 'bdgfs_hybrid_heads_split',
    'bdgfs_bgk_moments', 'bdgfs_bgk_maxwellian', 'bdgfs_ars_stage',
    'bdgfs_esbgk_moments', 'bdgfs_esbgk_gaussian', 'bdgfs_shakov_moments', 'bdgfs_shakov_target',
    'bdgfs_bdf_step', 'bdgfs_vss_scratch_bytes', 'bdgfs_vss_collide', 'bdgfs_vss_project',
)


class BdgfsError(RuntimeError):
    pass


class VhsGrid(C.Structure):
    _fields_ = [('Nv', C.c_int32), ('Nrho', C.c_int32), ('M', C.c_int32),
                ('fp64', C.c_int32), ('tile', C.c_int32), ('pad_', C.c_int32),
                ('prefac', C.c_double), ('cw', C.c_double),
                ('phase', C.c_void_p), ('gw', C.c_void_p), ('bb2', C.c_void_p),
                ('c0', C.c_void_p), ('ginv', C.c_void_p)]


class VhsBatch(C.Structure):
    _fields_ = [('grid', C.c_int32), ('pad_', C.c_int32), ('ndof', C.c_int64),
                ('f', C.c_void_p), ('Q', C.c_void_p), ('moments', C.c_void_p),
                ('index', C.c_void_p), ('count', C.c_void_p)]


class FrEles(C.Structure):
    _fields_ = [('ndims', C.c_int32), ('nupts', C.c_int32), ('nfpts', C.c_int32),
                ('neles', C.c_int32), ('nv', C.c_int64), ('Nv', C.c_int32),
                ('fp64', C.c_int32),
                ('m0', C.c_void_p), ('dcorr', C.c_void_p), ('m3', C.c_void_p),
                ('smats', C.c_void_p), ('rcpdjac', C.c_void_p), ('pnorm', C.c_void_p),
                ('magn', C.c_void_p), ('nbr', C.c_void_p), ('c0', C.c_void_p),
                ('engine', C.c_int32), ('pad_', C.c_int32)]


class FrTensor(C.Structure):
    _fields_ = [('fsel', C.c_void_p), ('fdim', C.c_void_p), ('fsgn', C.c_void_p),
                ('m1line', C.c_void_p), ('p', C.c_int32), ('pad_', C.c_int32)]


class FrWall(C.Structure):
    _fields_ = [('nwall', C.c_int32), ('nbc', C.c_int32),
                ('fpt', C.c_void_p), ('bcid', C.c_void_p), ('uwall', C.c_void_p),
                ('fw', C.c_void_p), ('bcv', C.c_void_p), ('cw', C.c_double),
                ('kind', C.c_void_p), ('kinds_used', C.c_int32), ('pad_', C.c_int32)]


BC_DIFFUSE, BC_INLET, BC_OUTLET, BC_SPECULAR_X, BC_SPECULAR_Y, BC_SPECULAR_Z = range(6)


class GemmArgs(C.Structure):
    _fields_ = [('M', C.c_int64), ('N', C.c_int64), ('K', C.c_int64),
                ('A', C.c_void_p), ('sam', C.c_int64), ('sak', C.c_int64),
                ('B', C.c_void_p), ('sbn', C.c_int64), ('sbk', C.c_int64),
                ('a_bf16', C.c_int32), ('b_bf16', C.c_int32),
                ('alpha', C.c_float), ('beta', C.c_float),
                ('bias', C.c_void_p), ('act', C.c_int32), ('engine', C.c_int32),
                ('cf32', C.c_void_p), ('cbf16', C.c_void_p), ('ldc', C.c_int64),
                ('zout', C.c_void_p), ('zin', C.c_void_p), ('ldz', C.c_int64),
                ('status', C.c_void_p), ('pad_', C.c_int32),
                ('arow', C.c_void_p), ('crow', C.c_void_p), ('row_scale', C.c_void_p),
                ('mcount', C.c_void_p)]


class HybridArgs(C.Structure):
    _fields_ = [('ndof', C.c_int64), ('Nv', C.c_int32), ('fp64', C.c_int32),
                ('c0', C.c_void_p), ('ginv', C.c_void_p), ('cw', C.c_double),
                ('threshold', C.c_float), ('recheck', C.c_float), ('seed', C.c_uint64),
                ('counts', C.c_void_p), ('sur_idx', C.c_void_p), ('sur_inv_rho', C.c_void_p),
                ('sur_rho2', C.c_void_p), ('spec_idx', C.c_void_p), ('flag', C.c_void_p),
                ('eps', C.c_void_p), ('recheck_err', C.c_void_p), ('seed_dev', C.c_void_p),
                ('dev_rows', C.c_void_p), ('feat', C.c_void_p), ('feat_ld', C.c_int64),
                ('sur_s', C.c_void_p), ('fb_idx', C.c_void_p), ('sur_uT', C.c_void_p),
                ('center', C.c_int32), ('pad2_', C.c_int32)]


class ArsArgs(C.Structure):
    _fields_ = [('ndof', C.c_int64), ('Nv', C.c_int32), ('fp64', C.c_int32),
                ('c0', C.c_void_p), ('cw', C.c_double),
                ('prefac', C.c_double), ('omega', C.c_double), ('dt', C.c_double),
                ('stage', C.c_int32), ('flags', C.c_int32),
                ('ae', C.c_double * 4), ('ai', C.c_double * 4),
                ('f', C.c_void_p * 4), ('fout', C.c_void_p), ('L', C.c_void_p * 4),
                ('U', C.c_void_p * 5), ('LU', C.c_void_p * 4),
                ('model', C.c_int32), ('pad_', C.c_int32), ('Pr', C.c_double)]


class VssArgs(C.Structure):
    _fields_ = [('Nv', C.c_int32), ('nspcs', C.c_int32), ('Nrho', C.c_int32), ('M', C.c_int32),
                ('ndof', C.c_int64), ('fp64', C.c_int32), ('pad_', C.c_int32),
                ('f', C.c_void_p * 4), ('Q', C.c_void_p * 4), ('mfrac', C.c_void_p),
                ('prefac', C.c_void_p), ('rfac', C.c_void_p), ('rw', C.c_void_p),
                ('sz', C.c_void_p), ('b', C.c_void_p), ('c', C.c_void_p)]


class VssProjArgs(C.Structure):
    _fields_ = [('Nv', C.c_int32), ('nspcs', C.c_int32), ('ndof', C.c_int64),
                ('fp64', C.c_int32), ('pad_', C.c_int32), ('Q', C.c_void_p * 4),
                ('c0', C.c_void_p), ('mass', C.c_void_p), ('ginv', C.c_void_p)]


class BdfArgs(C.Structure):
    _fields_ = [('ndof', C.c_int64), ('Nv', C.c_int32), ('fp64', C.c_int32),
                ('c0', C.c_void_p), ('cw', C.c_double), ('prefac', C.c_double),
                ('omega', C.c_double), ('dt', C.c_double), ('q', C.c_int32),
                ('model', C.c_int32), ('Pr', C.c_double), ('a', C.c_double * 4),
                ('g', C.c_double * 3), ('b', C.c_double), ('f', C.c_void_p * 3),
                ('L', C.c_void_p * 3), ('U', C.c_void_p * 3), ('LU', C.c_void_p * 3),
                ('Unew', C.c_void_p), ('fout', C.c_void_p), ('flags', C.c_int32),
                ('pad_', C.c_int32)]


_lib = None


def lib():
    """Load libbdgfs.so once; raise if it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise BdgfsError(f'{LIBPATH} not built: run python -m frfs_b200.build')
        L = C.CDLL(LIBPATH)
        L.bdgfs_vhs_scratch_bytes.restype = C.c_size_t
        L.bdgfs_vss_scratch_bytes.restype = C.c_size_t
        L.bdgfs_vhs_scratch_bytes.argtypes = [C.POINTER(VhsGrid), C.c_int32, C.c_int32]
        L.bdgfs_vhs_collide.restype = C.c_int32
        L.bdgfs_vhs_collide.argtypes = [C.POINTER(VhsGrid), C.c_int32, C.POINTER(VhsBatch),
                                        C.c_int32, C.c_int32, C.c_void_p, C.c_size_t,
                                        C.c_void_p, C.c_void_p]
        L.bdgfs_vhs_collide_static.restype = C.c_int32
        L.bdgfs_vhs_collide_static.argtypes = [C.POINTER(VhsGrid), C.c_int32,
                                               C.POINTER(VhsBatch), C.c_int32, C.c_int32,
                                               C.c_void_p]
        L.bdgfs_vhs_tiles.restype = C.c_int32
        L.bdgfs_vhs_tiles.argtypes = [C.POINTER(VhsGrid), C.c_int32, C.c_void_p, C.c_int32]
        L.bdgfs_fma_probe.restype = C.c_int32
        L.bdgfs_fma_probe.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]
        vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        sig = {
            'bdgfs_fr_disu': [vp, vp, vp, vp],
            'bdgfs_fr_invmass': [vp, vp, vp, vp, vp],
            'bdgfs_fr_bc_update': [vp, vp, vp, vp],
            'bdgfs_fr_rhs': [vp, vp, vp, vp, vp, dbl, dbl, vp, dbl, vp, dbl, vp],
            'bdgfs_fr_rhs_gather': [vp, vp, vp, vp, vp, dbl, dbl, vp, dbl, vp, dbl, vp],
            'bdgfs_fr_bc_update_gather': [vp, vp, vp, vp, vp],
            'bdgfs_fr_rhs_tensor': [vp, vp, vp, vp, vp, vp, dbl, dbl, vp, dbl, vp, dbl, vp],
            'bdgfs_moments': [vp, i64, i32, i32, vp, dbl, vp, vp],
            'bdgfs_residual': [vp, vp, i64, i32, vp, vp],
            'bdgfs_status_check': [vp, i64, i32, vp, vp],
            'bdgfs_gemm': [C.c_void_p, vp],
            'bdgfs_relmse': [vp, vp, i64, i64, C.c_float, vp, vp, vp],
            'bdgfs_hybrid_classify': [vp, vp, vp],
            'bdgfs_hybrid_project': [vp, vp, vp],
            'bdgfs_hybrid_scatter': [vp, vp, vp, vp],
            'bdgfs_hybrid_project_scatter': [vp, vp, vp, vp],
            'bdgfs_hybrid_heads': [vp, vp, C.c_int64, C.c_int64, C.c_int32, vp, C.c_int64, vp],
            'bdgfs_hybrid_shift': [vp, vp, i32, vp, i32, C.c_float, vp],
            'bdgfs_hybrid_heads_split': [vp, vp, C.c_int64, C.c_int64, C.c_int32, vp, C.c_int64, vp],
            'bdgfs_hybrid_tfeatures': [vp, vp, i64, i64, i64, i64, i32, i64, vp],
            'bdgfs_bgk_moments': [vp, C.c_int64, C.c_int32, C.c_int32, vp, C.c_double, vp, vp],
            'bdgfs_bgk_maxwellian': [vp, C.c_int64, C.c_int32, C.c_int32, vp, vp, vp],
            'bdgfs_ars_stage': [vp, vp],
            'bdgfs_esbgk_moments': [vp, C.c_int64, C.c_int32, C.c_int32, vp, C.c_double, vp, vp],
            'bdgfs_esbgk_gaussian': [vp, C.c_int64, C.c_int32, C.c_int32, vp, C.c_double, vp, vp],
            'bdgfs_shakov_moments': [vp, C.c_int64, C.c_int32, C.c_int32, vp, C.c_double, vp, vp],
            'bdgfs_shakov_target': [vp, C.c_int64, C.c_int32, C.c_int32, vp, C.c_double, vp, vp],
            'bdgfs_bdf_step': [vp, vp],
            'bdgfs_vss_scratch_bytes': [C.c_int32, C.c_int32, C.c_int32],
            'bdgfs_vss_collide': [vp, vp, C.c_size_t, vp],
            'bdgfs_vss_project': [vp, vp],
            'bdgfs_colsum': [vp, i64, i64, vp, vp],
            'bdgfs_wait_probe': [C.c_uint32, i32, vp, vp],
            'bdgfs_adamw': [vp, vp, vp, vp, vp, i64, C.c_float, C.c_float, C.c_float,
                            C.c_float, C.c_float, i64, vp],
        }
        for name, at in sig.items():
            fn = getattr(L, name)
            fn.restype = C.c_int32
            fn.argtypes = at
        _lib = L
    return _lib


def check(rc, what):
    if rc != BDGFS_OK:
        raise BdgfsError(f'{what}: {_ERRORS.get(rc, rc)} (status {rc})')


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def ref(struct):
    return C.c_void_p(C.addressof(struct))
