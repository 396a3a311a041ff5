"""Registry helpers (the reference's frfs/util.py:subclass_where idiom)."""


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
