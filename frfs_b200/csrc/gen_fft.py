"""Generate straight-line register DFT codelets (``fft_codelets.cuh``).

Build step of the package: ``python frfs_b200/csrc/gen_fft.py`` rewrites
``frfs_b200/csrc/fft_codelets.cuh``.  Each codelet is an in-place,
unnormalised DFT of length N on a register array ``cpx<T> x[N]`` with
natural input and output order:

    X[k] = sum_n x[n] * exp(sign * 2*pi*i * n*k / N),  sign = -1 (forward)
                                                        or +1 (inverse)

which are the sign/normalisation conventions of a Z2Z FFT (forward and
inverse both unnormalised).  Lengths with a coprime factor 3 (12 = 3*4,
24 = 3*8) use the Good-Thomas prime-factor split (Good 1958; Thomas 1963):
CRT index maps, no twiddle factors between the stages.  Otherwise the
factorisation is the textbook Cooley-Tukey mixed-radix split N = N1*N2
(input index n = N2*n1 + n2, output index k = k1 + N1*k2), applied
recursively with hand-written radix-2/3/4 butterflies; twiddles
exp(sign*2*pi*i*e/N) are evaluated in FP64 by numpy here and emitted as
literals, with the trivial ones (e = 0, N/4, N/2, 3N/4 and the odd
multiples of N/8) specialised.
"""
import os

import numpy as np

SIZES = (8, 12, 16, 24, 32)


class Emitter:
    def __init__(self):
        self.lines = []
        self.n = 0

    def tmp(self):
        self.n += 1
        return f't{self.n}'

    def emit(self, s):
        self.lines.append('    ' + s)

    def cdecl(self, re, im):
        v = self.tmp()
        self.emit(f'const T {v}r = {re}; const T {v}i = {im};')
        return v


def lit(v):
    return f'T({float(v)!r})'


def butterfly(em, xs, sign):
    """Small DFTs: xs are variable stems (with r/i parts)."""
    n = len(xs)
    if n == 1:
        return xs
    if n == 2:
        a, b = xs
        y0 = em.cdecl(f'{a}r + {b}r', f'{a}i + {b}i')
        y1 = em.cdecl(f'{a}r - {b}r', f'{a}i - {b}i')
        return [y0, y1]
    if n == 3:
        a, b, c = xs
        s = em.cdecl(f'{b}r + {c}r', f'{b}i + {c}i')
        d = em.cdecl(f'{b}r - {c}r', f'{b}i - {c}i')
        y0 = em.cdecl(f'{a}r + {s}r', f'{a}i + {s}i')
        t = em.cdecl(f'{a}r - T(0.5) * {s}r', f'{a}i - T(0.5) * {s}i')
        h = lit(np.sqrt(3.0) / 2.0)
        # w = exp(sign*2*pi*i/3) = -1/2 + sign*i*sqrt(3)/2
        # y1 = t + sign*i*h*d ; y2 = t - sign*i*h*d ; i*d = (-d.i, d.r)
        if sign < 0:
            y1 = em.cdecl(f'{t}r + {h} * {d}i', f'{t}i - {h} * {d}r')
            y2 = em.cdecl(f'{t}r - {h} * {d}i', f'{t}i + {h} * {d}r')
        else:
            y1 = em.cdecl(f'{t}r - {h} * {d}i', f'{t}i + {h} * {d}r')
            y2 = em.cdecl(f'{t}r + {h} * {d}i', f'{t}i - {h} * {d}r')
        return [y0, y1, y2]
    if n == 4:
        a, b, c, d = xs
        s0 = em.cdecl(f'{a}r + {c}r', f'{a}i + {c}i')
        d0 = em.cdecl(f'{a}r - {c}r', f'{a}i - {c}i')
        s1 = em.cdecl(f'{b}r + {d}r', f'{b}i + {d}i')
        d1 = em.cdecl(f'{b}r - {d}r', f'{b}i - {d}i')
        y0 = em.cdecl(f'{s0}r + {s1}r', f'{s0}i + {s1}i')
        y2 = em.cdecl(f'{s0}r - {s1}r', f'{s0}i - {s1}i')
        # w = sign*i ; y1 = d0 + w*d1 ; y3 = d0 - w*d1
        if sign < 0:     # w*d1 = -i*d1 = (d1.i, -d1.r)
            y1 = em.cdecl(f'{d0}r + {d1}i', f'{d0}i - {d1}r')
            y3 = em.cdecl(f'{d0}r - {d1}i', f'{d0}i + {d1}r')
        else:            # w*d1 = i*d1 = (-d1.i, d1.r)
            y1 = em.cdecl(f'{d0}r - {d1}i', f'{d0}i + {d1}r')
            y3 = em.cdecl(f'{d0}r + {d1}i', f'{d0}i - {d1}r')
        return [y0, y1, y2, y3]
    raise ValueError(n)


def twiddle(em, v, e, N, sign):
    e %= N
    if e == 0:
        return v
    if 4 * e == N:          # w = sign*i
        return (em.cdecl(f'{v}i', f'-{v}r') if sign < 0
                else em.cdecl(f'-{v}i', f'{v}r'))
    if 2 * e == N:
        return em.cdecl(f'-{v}r', f'-{v}i')
    if 4 * e == 3 * N:      # w = -sign*i
        return (em.cdecl(f'-{v}i', f'{v}r') if sign < 0
                else em.cdecl(f'{v}i', f'-{v}r'))
    ang = sign * 2.0 * np.pi * e / N
    c, s = np.cos(ang), np.sin(ang)
    if (8 * e) % N == 0:    # odd multiple of N/8: |c| = |s| = sqrt(2)/2
        h = lit(abs(c))
        sc, ss = ('+' if c > 0 else '-'), ('+' if s > 0 else '-')
        # (vr + i vi)(c + i s) = (c vr - s vi) + i (s vr + c vi)
        re = f'{h} * ({sc}{v}r {"-" if ss == "+" else "+"} {v}i)'
        im = f'{h} * ({ss}{v}r {sc} {v}i)'
        return em.cdecl(re, im)
    return em.cdecl(f'{v}r * {lit(c)} - {v}i * {lit(s)}',
                    f'{v}r * {lit(s)} + {v}i * {lit(c)}')


_ORDER = (4, 3, 2)


def radix_of(N):
    for r in _ORDER:
        if N % r == 0 and N != r:
            return r
    return N


def _opcount(N, order):
    global _ORDER
    saved, _ORDER = _ORDER, order
    try:
        em = Emitter()
        xs = [em.cdecl('x', 'y') for _ in range(N)]
        dft(em, xs, +1)
        body = '\n'.join(em.lines)
        return body.count(' + ') + body.count(' - ') + body.count('*')
    finally:
        _ORDER = saved


def best_order(N):
    """Radix preference (a permutation of 4, 3, 2) with the fewest operations."""
    import itertools
    return min(itertools.permutations((4, 3, 2)), key=lambda o: (_opcount(N, o), o))


def coprime_split(N):
    """(N1, N2) with N = N1*N2, gcd = 1, N1 the factor 3 (24 = 3*8,
    12 = 3*4), or None."""
    from math import gcd
    if N % 3 == 0 and N > 3 and gcd(3, N // 3) == 1:
        return 3, N // 3
    return None


def pfa(em, xs, sign, N1, N2):
    """Good-Thomas prime-factor split for coprime N1, N2 (no twiddles):
    n = (N2 n1 + N1 n2) mod N, k = (N2 t1 k1 + N1 t2 k2) mod N with
    t1 = N2^-1 mod N1, t2 = N1^-1 mod N2."""
    N = N1 * N2
    t1, t2 = pow(N2, -1, N1), pow(N1, -1, N2)
    A = [dft(em, [xs[(N2 * n1 + N1 * n2) % N] for n1 in range(N1)], sign) for n2 in range(N2)]
    X = [None] * N
    for k1 in range(N1):
        out = dft(em, [A[n2][k1] for n2 in range(N2)], sign)
        for k2 in range(N2):
            X[(N2 * t1 * k1 + N1 * t2 * k2) % N] = out[k2]
    return X


def dft(em, xs, sign):
    N = len(xs)
    if N <= 4:
        return butterfly(em, xs, sign)
    sp = coprime_split(N)
    if sp is not None:
        return pfa(em, xs, sign, *sp)
    N1 = radix_of(N)
    N2 = N // N1
    # step 1: N2 DFTs of size N1 over x[N2*n1 + n2]
    Y = [[None] * N1 for _ in range(N2)]
    for n2 in range(N2):
        out = butterfly(em, [xs[N2 * n1 + n2] for n1 in range(N1)], sign)
        for k1 in range(N1):
            Y[n2][k1] = twiddle(em, out[k1], n2 * k1, N, sign)
    # step 3: N1 DFTs of size N2 over n2
    X = [None] * N
    for k1 in range(N1):
        out = dft(em, [Y[n2][k1] for n2 in range(N2)], sign)
        for k2 in range(N2):
            X[k1 + N1 * k2] = out[k2]
    return X


def codelet(N, sign):
    global _ORDER
    _ORDER = best_order(N)
    em = Emitter()
    name = f'dft{N}_{"fwd" if sign < 0 else "inv"}'
    xs = []
    for n in range(N):
        v = em.tmp()
        em.emit(f'const T {v}r = x[{n}].x; const T {v}i = x[{n}].y;')
        xs.append(v)
    X = dft(em, xs, sign)
    for k in range(N):
        em.emit(f'x[{k}].x = {X[k]}r; x[{k}].y = {X[k]}i;')
    body = '\n'.join(em.lines)
    return (f'template <typename T>\n__device__ __forceinline__ void '
            f'{name}(cpx<T> (&x)[{N}])\n{{\n{body}\n}}\n')


def main():
    out = ['// Generated by gen_fft.py: unnormalised in-register DFT codelets.',
           '// Do not edit by hand.',
           '#pragma once', '#include "cpx.cuh"', '',
           'namespace bdgfs {', '']
    for N in SIZES:
        out.append(codelet(N, -1))
        out.append(codelet(N, +1))
    disp = ['template <int N, int SIGN, typename T>',
            '__device__ __forceinline__ void dft(cpx<T> (&x)[N])', '{']
    for N in SIZES:
        disp.append(f'    if constexpr (N == {N}) {{ if constexpr (SIGN < 0) '
                    f'dft{N}_fwd<T>(x); else dft{N}_inv<T>(x); }}')
    disp.append('}')
    out += disp + ['', '}  // namespace bdgfs', '']
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                        'fft_codelets.cuh')
    with open(path, 'w') as fh:
        fh.write('\n'.join(out))


def reference_check():
    """Self-check of the generated algebra by executing it in numpy."""
    import re
    for N in SIZES:
        for sign in (-1, 1):
            src = codelet(N, sign)
            rng = np.random.default_rng(N)
            x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
            env = {'x': x.copy(), 'T': float}
            body = src[src.index('{') + 1:src.rindex('}')]
            py = []
            for line in body.strip().splitlines():
                line = line.strip()
                for stmt in line.split(';'):
                    stmt = stmt.strip()
                    if not stmt:
                        continue
                    stmt = re.sub(r'^const T ', '', stmt)
                    stmt = re.sub(r'x\[(\d+)\]\.x', r'XR[\1]', stmt)
                    stmt = re.sub(r'x\[(\d+)\]\.y', r'XI[\1]', stmt)
                    py.append(stmt)
            XR, XI = x.real.copy(), x.imag.copy()
            env = {'XR': XR, 'XI': XI, 'T': float}
            exec('\n'.join(py), env)
            got = env['XR'] + 1j * env['XI']
            ref = (np.fft.fft(x) if sign < 0 else np.fft.ifft(x) * N)
            err = np.abs(got - ref).max() / np.abs(ref).max()
            assert err < 1e-13, (N, sign, err)


if __name__ == '__main__':
    reference_check()
    main()
