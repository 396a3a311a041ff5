"""Render the reference's BGK-family relaxation kernels and compile each
with the ARS harness into ``oracle/_ref/libref_ars_<model>.so`` (test
infrastructure; the outputs stay out of version control).

    python -m oracle.ref_adgfs.build <reference-root>

Models 'bgk' (bgk-direct-gll, 5 moments), 'esbgk' (esbgk-direct-gll, 11)
and 'shakov' (shakov-direct-gll, 14), each with omega = 0.81 and, for the
last two, Pr = 2/3, FP64: the template arguments of
frfs/solvers/adgfs/scattering.py:115-121.
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(ROOT, 'oracle', '_ref')
MODELS = {'bgk': dict(nalph=5, Pr=1.0), 'esbgk': dict(nalph=11, Pr=2.0 / 3.0),
          'shakov': dict(nalph=14, Pr=2.0 / 3.0)}
OMEGA = 0.81
NV = 16


def render_model(reference_root, model, vsize):
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from oracle.ref_vhs.render import render
    d = os.path.join(reference_root, 'frfs', 'solvers', 'adgfs', 'kernels', 'scattering')
    with open(os.path.join(d, f'{model}-direct-gll.mako')) as fh:
        src = fh.read()
    m = MODELS[model]
    return render(src, lookup_dir=d, soasz=32, vsize=vsize, nalph=m['nalph'], omega=OMEGA, Pr=m['Pr'],
                  dtype='double', nbdf=[1, 2, 3], nars=[1, 2, 3, 4])


def build(reference_root, nvcc='nvcc'):
    os.makedirs(OUT, exist_ok=True)
    built = []
    for model, m in MODELS.items():
        cu = os.path.join(OUT, f'ars_{model}.cu')
        with open(cu, 'w') as fh:
            fh.write(render_model(reference_root, model, NV**3))
        so = os.path.join(OUT, f'libref_ars_{model}.so')
        cmd = [nvcc, '-O3', '-std=c++17', '-gencode', 'arch=compute_100a,code=sm_100a', '-Xcompiler', '-fPIC',
               '-shared', f'-DREF_KERNELS="{cu}"', f'-DNALPH={m["nalph"]}']
        if model != 'bgk':
            cmd.append('-DHAS_MOMENT_NORM')
        subprocess.check_call(cmd + [os.path.join(HERE, 'harness.cu'), '-o', so])
        with open(os.path.join(OUT, f'ref_ars_{model}.json'), 'w') as fh:
            json.dump(dict(m, model=model, omega=OMEGA, Nv=NV), fh)
        built.append(so)
    return built


if __name__ == '__main__':
    if len(sys.argv) != 2 or not os.path.isdir(os.path.join(sys.argv[1], 'frfs')):
        sys.exit('usage: python -m oracle.ref_adgfs.build <reference-root>')
    print('\n'.join(build(os.path.abspath(sys.argv[1]))))
