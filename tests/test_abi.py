"""The C ABI library loads, exports every symbol include/bdgfs.h declares,
and the ctypes mirrors of its structs have the C layout (checked against
offsetof/sizeof from a C program compiled with the header)."""
import os
import re
import shutil
import subprocess

import pytest

from frfs_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, 'include', 'bdgfs.h')


def _declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r'\b(bdgfs_\w+)\s*\(', txt)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = _declared()
    assert len(names) >= 9
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.EXPORTS) | set(n for n in names if n not in _lib.EXPORTS) \
        and set(_lib.EXPORTS) <= set(names)


STRUCTS = {
    'bdgfs_vhs_grid': _lib.VhsGrid,
    'bdgfs_vhs_batch': _lib.VhsBatch,
    'bdgfs_fr_eles': _lib.FrEles,
    'bdgfs_fr_walls': _lib.FrWall,
    'bdgfs_fr_tensor': _lib.FrTensor,
    'bdgfs_gemm_args': _lib.GemmArgs,
    'bdgfs_hybrid_args': _lib.HybridArgs,
    'bdgfs_ars_args': _lib.ArsArgs,
    'bdgfs_bdf_args': _lib.BdfArgs,
    'bdgfs_vss_args': _lib.VssArgs,
    'bdgfs_vss_proj_args': _lib.VssProjArgs,
}


@pytest.mark.skipif(shutil.which('gcc') is None, reason='no C compiler')
def test_struct_layouts_match_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"',
             'int main(void) {']
    for cname, cls in STRUCTS.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ['return 0;', '}']
    src = tmp_path / 'off.c'
    src.write_text('\n'.join(lines))
    exe = tmp_path / 'off'
    subprocess.check_call(['gcc', str(src), '-o', str(exe)])
    out = subprocess.check_output([str(exe)], text=True)
    for line in out.splitlines():
        cname, field, val = line.split()
        cls = STRUCTS[cname]
        if field == 'sizeof':
            assert __import__('ctypes').sizeof(cls) == int(val), cname
        else:
            assert getattr(cls, field).offset == int(val), (cname, field)


def test_invalid_arguments_return_status_not_crash():
    L = _lib.lib()
    assert L.bdgfs_vhs_collide(None, 0, None, 0, 0, None, 0, None, None) == -1
    assert L.bdgfs_fr_disu(None, None, None, None) == -1
    assert L.bdgfs_fr_invmass(None, None, None, None, None) == -1
    assert L.bdgfs_residual(None, None, 0, 0, None, None) == -1
    assert L.bdgfs_vhs_scratch_bytes(None, 0, 1) == 0


def _header_params(name):
    """Number of parameters of `name` as include/bdgfs.h declares it."""
    txt = re.sub(r'/\*.*?\*/', '', open(HEADER).read(), flags=re.S)
    m = re.search(r'\b' + name + r'\s*\(([^)]*)\)\s*;', txt)
    assert m, name
    args = m.group(1).strip()
    return 0 if args in ('', 'void') else args.count(',') + 1


def test_reference_side_binding_matches_header_and_notes(tmp_path):
    """The stub INTEGRATION.md shows is frfs_b200/refbinding.py verbatim; its
    structures have the header's layout and each bound entry point the
    header's parameter count, and the library exports every one of them."""
    from frfs_b200 import refbinding as rb
    notes = open(os.path.join(ROOT, 'INTEGRATION.md')).read()
    m = re.search(r'<!-- refbinding\.py begin -->\n```python\n(.*?)```\n<!-- refbinding\.py end -->',
                  notes, flags=re.S)
    assert m, 'INTEGRATION.md lost the binding block'
    src = open(os.path.join(ROOT, 'frfs_b200', 'refbinding.py')).read()
    assert m.group(1) == src
    for name, (_, args) in rb.SIGNATURES.items():
        assert _header_params(name) == len(args), name
    L = rb.load(_lib.LIBPATH)
    for name in rb.SIGNATURES:
        assert hasattr(L, name)
    if shutil.which('gcc') is None:
        pytest.skip('no C compiler')
    mirror = {'bdgfs_vhs_grid': rb.VhsGrid, 'bdgfs_vhs_batch': rb.VhsBatch,
              'bdgfs_vss_args': rb.VssArgs}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"',
             'int main(void) {']
    for cname, cls in mirror.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ['return 0;', '}']
    (tmp_path / 'off.c').write_text('\n'.join(lines))
    subprocess.check_call(['gcc', str(tmp_path / 'off.c'), '-o', str(tmp_path / 'off')])
    import ctypes
    for line in subprocess.check_output([str(tmp_path / 'off')], text=True).splitlines():
        cname, field, val = line.split()
        cls = mirror[cname]
        got = ctypes.sizeof(cls) if field == 'sizeof' else getattr(cls, field).offset
        assert got == int(val), (cname, field)
