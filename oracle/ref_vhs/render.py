"""Render the reference's vhs-gll Mako template (test infrastructure).

The template (frfs/solvers/dgfs/kernels/scattering/vhs-gll.mako) uses a
small part of Mako: a module block ``<%! ... %>``, one-line code blocks
``<% ... %>``, control lines ``% for ...:`` / ``% endfor`` (and the if
forms) and ``${expression}`` substitutions rendered with ``str``.  This
renderer translates exactly those into a Python function, as Mako itself
does, and runs it with the template arguments the reference passes
(frfs/solvers/dgfs/scattering.py:154-160).
"""
import re

_EXPR = re.compile(r'\$\{(.*?)\}')


def _compile(src):
    """Python source of a function render(ctx) -> str for the template."""
    out = ['def __render(__ctx):', '    globals().update(__ctx)', '    __buf = []']
    mod = []
    depth = 1
    i = 0
    lines = src.split('\n')
    while i < len(lines):
        line = lines[i]
        st = line.strip()
        if st.startswith('<%!'):                           # module-level block
            body = []
            rest = st[3:]
            while '%>' not in rest:
                body.append(rest)
                i += 1
                rest = lines[i]
            body.append(rest[:rest.index('%>')])
            mod.extend(b.strip() for b in body if b.strip())
            i += 1
            continue
        if st.startswith('%') and not st.startswith('%%'):  # control line
            stmt = st[1:].strip()
            key = stmt.split()[0].rstrip(':') if stmt else ''
            if key in ('endfor', 'endif', 'endwhile'):
                depth -= 1
            elif key in ('elif', 'else'):
                out.append('    ' * (depth - 1) + stmt)
            else:
                out.append('    ' * depth + stmt)
                depth += 1
            i += 1
            continue
        if st.startswith('<%') and st.endswith('%>') and not st.startswith('<%!'):
            out.append('    ' * depth + st[2:-2].strip())   # one-line code block
            i += 1
            continue
        if st.startswith('##'):                            # template comment
            i += 1
            continue
        parts, pos = [], 0
        for m in _EXPR.finditer(line):
            parts.append(repr(line[pos:m.start()]))
            parts.append('str(' + m.group(1) + ')')
            pos = m.end()
        parts.append(repr(line[pos:] + '\n'))
        out.append('    ' * depth + '__buf.append(' + ' + '.join(parts) + ')')
        i += 1
    out.append("    return ''.join(__buf)")
    return '\n'.join(mod + out)


def render(src, **args):
    ns = {}
    exec(compile(_compile(src), '<vhs-gll.mako>', 'exec'), ns)
    return ns['__render'](dict(args))


def render_vhs_gll(reference_root, Nrho, M, vsize, sw, prefac, qw, sz, gamma, L, qz, soasz=32):
    """The rendered CUDA source of the reference's vhs-gll kernels for one
    velocity grid, with the template arguments of scattering.py:154-160."""
    import os
    path = os.path.join(reference_root, 'frfs', 'solvers', 'dgfs', 'kernels', 'scattering',
                        'vhs-gll.mako')
    with open(path) as fh:
        src = fh.read()
    return render(src, Nrho=Nrho, M=M, vsize=vsize, sw=sw, prefac=prefac, soasz=soasz, qw=qw,
                  sz=sz, gamma=gamma, L=L, qz=qz)
