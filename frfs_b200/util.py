"""Registry helpers (the reference's frfs/util.py:subclass_where idiom) and
the expression evaluator of .ini options (frfs/nputil.py:npeval)."""
import re

import numpy as np

_NPEVAL_SYMS = {
    '__builtins__': {},
    'exp': np.exp, 'log': np.log, 'sin': np.sin, 'asin': np.arcsin, 'cos': np.cos,
    'acos': np.arccos, 'tan': np.tan, 'atan': np.arctan, 'atan2': np.arctan2,
    'abs': np.abs, 'fabs': np.abs, 'pow': np.power, 'sqrt': np.sqrt, 'tanh': np.tanh,
    'pi': np.pi}


def npeval(expr, variables):
    """Evaluate an .ini expression over numpy arrays: arithmetic, the
    functions above, comparisons (as in the C expressions the reference
    pastes into its kernels) and the names in ``variables``; no
    exponentiation operator (use pow), no attribute access."""
    if '^' in expr or '**' in expr:
        raise ValueError('Direct exponentiation is not supported; use pow')
    if not re.match(r'[A-Za-z0-9_ \t\n\r.,+\-*/%()<>=!]+$', expr):
        raise ValueError(f'Invalid characters in expression {expr!r}')
    if re.search(r'[A-Za-z_)]\s*\.\s*[A-Za-z_]', expr):
        raise ValueError(f'Invalid expression {expr!r}')
    return eval(expr, _NPEVAL_SYMS, dict(variables))


def all_subclasses(cls):
    out = []
    for c in cls.__subclasses__():
        out.append(c)
        out.extend(all_subclasses(c))
    return out


def subclass_where(cls, **kwargs):
    """The subclass of ``cls`` whose class attributes match ``kwargs``."""
    for s in all_subclasses(cls):
        if all(getattr(s, k, None) == v for k, v in kwargs.items()):
            return s
    attrs = ', '.join(f'{k} = {v}' for k, v in kwargs.items())
    raise KeyError(f'No subclasses of {cls.__name__} with {attrs}')
