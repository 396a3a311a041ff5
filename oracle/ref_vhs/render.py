"""Render the reference's collision-kernel Mako templates (test infrastructure).

The templates (frfs/solvers/dgfs/kernels/scattering/vhs-gll.mako,
frfs/solvers/dgfsbi/kernels/scattering/vss-gll.mako) use a small part of
Mako: a module block ``<%! ... %>``, code blocks ``<% ... %>`` (one line or
several), control lines ``% for ...:`` / ``% endfor`` and the if forms, and
``${expression}`` substitutions rendered with ``str``.  This renderer
translates exactly those into a Python function, as Mako itself does, and
runs it with the template arguments the reference passes
(frfs/solvers/dgfs/scattering.py:154-160, frfs/solvers/dgfsbi/scattering.py:
153-163).
"""
import textwrap


def _subst(line):
    """Python expression joining the literal text of a line with its
    ${...} substitutions (braces inside an expression are matched)."""
    parts, pos = [], 0
    while True:
        i = line.find('${', pos)
        if i < 0:
            break
        depth, j = 1, i + 2
        while depth:
            depth += {'{': 1, '}': -1}.get(line[j], 0)
            j += 1
        parts.append(repr(line[pos:i]))
        parts.append('str(' + line[i + 2:j - 1] + ')')
        pos = j
    parts.append(repr(line[pos:] + '\n'))
    return ' + '.join(parts)


def _open_subst(text):
    """True when a ${ in text is not closed within it."""
    pos = 0
    while True:
        i = text.find('${', pos)
        if i < 0:
            return False
        depth, j = 1, i + 2
        while depth and j < len(text):
            depth += {'{': 1, '}': -1}.get(text[j], 0)
            j += 1
        if depth:
            return True
        pos = j


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
        if st.startswith('<%include') and st.endswith('/>'):
            name = st.split('file=', 1)[1].split('"')[1]
            out.append('    ' * depth + f'__buf.append(__include({name!r}, __ctx))')
            i += 1
            continue
        if st.startswith('<%') and '%>' not in st:
            # module block, or a code block over several lines
            module = st.startswith('<%!')
            body = [st[3:] if module else st[2:]]
            while True:
                i += 1
                if '%>' in lines[i]:
                    body.append(lines[i][:lines[i].index('%>')])
                    break
                body.append(lines[i])
            code = textwrap.dedent('\n'.join(body)).strip('\n')
            if module:
                mod.extend(c for c in code.split('\n') if c.strip())
            else:
                out.extend('    ' * depth + c for c in code.split('\n') if c.strip())
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
        if st.startswith('<%') and st.endswith('%>'):
            out.append('    ' * depth + st[2:-2].strip())   # one-line code block
            i += 1
            continue
        if st.startswith('##'):                            # template comment
            i += 1
            continue
        while _open_subst(line) and i + 1 < len(lines):     # ${...} over several lines
            i += 1
            line = line + '\n' + lines[i]
        out.append('    ' * depth + '__buf.append(' + _subst(line) + ')')
        i += 1
    out.append("    return ''.join(__buf)")
    return '\n'.join(mod + out)


def render(src, lookup_dir=None, **args):
    """Render template text with the given arguments; <%include file="x"/>
    renders lookup_dir/x.mako with the same arguments."""
    import os

    def include(name, ctx):
        with open(os.path.join(lookup_dir, name + '.mako')) as fh:
            return render(fh.read(), lookup_dir, **{k: v for k, v in ctx.items()
                                                    if not k.startswith('__')})
    ns = {'__include': include}
    exec(compile(_compile(src), '<template>', 'exec'), ns)
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
