"""INI configuration with the reference's accessors.

Mirrors the interface of frfs/inifile.py:19-141 (``Inifile``): case is
preserved, ``;`` starts an inline comment, ``get*`` take an optional
default, ``getexpr`` substitutes ``[constants]`` names into an expression
(``items_as`` returns a section as typed values).
"""
import configparser
import io
import re

_sentinel = object()


class Inifile:
    def __init__(self, inistr=None):
        self._cp = cp = configparser.ConfigParser(inline_comment_prefixes=[';'],
                                                  interpolation=None)
        cp.optionxform = str
        if inistr:
            cp.read_string(inistr)

    @staticmethod
    def load(file):
        if isinstance(file, str):
            with open(file) as fh:
                return Inifile(fh.read())
        return Inifile(file.read())

    def set(self, section, option, value):
        value = str(value)
        try:
            self._cp.set(section, option, value)
        except configparser.NoSectionError:
            self._cp.add_section(section)
            self._cp.set(section, option, value)

    def hasopt(self, section, option):
        return self._cp.has_option(section, option)

    def hassect(self, section):
        return self._cp.has_section(section)

    def get(self, section, option, default=_sentinel, vars=None):
        try:
            return self._cp.get(section, option, vars=vars)
        except (configparser.NoSectionError, configparser.NoOptionError):
            if default is _sentinel:
                raise
            self.set(section, option, default)
            return self._cp.get(section, option, vars=vars)

    def getpath(self, section, option, default=_sentinel):
        import os
        return os.path.abspath(os.path.expanduser(self.get(section, option, default)))

    _bool_states = {'1': True, 'yes': True, 'true': True, 'on': True,
                    '0': False, 'no': False, 'false': False, 'off': False}

    def getbool(self, section, option, default=_sentinel):
        v = self.get(section, option, default)
        return self._bool_states[str(v).lower()]

    def getfloat(self, section, option, default=_sentinel):
        return float(self.get(section, option, default))

    def getint(self, section, option, default=_sentinel):
        return int(self.get(section, option, default))

    def getexpr(self, section, option, default=_sentinel, subs={}):
        expr = self.get(section, option, default)
        if subs:
            # substitute whole words, longest name first
            for k in sorted(subs, key=len, reverse=True):
                expr = re.sub(r'\b{0}\b'.format(re.escape(k)), str(subs[k]), expr)
        return '({0})'.format(expr)

    def items(self, section):
        return dict(self._cp.items(section)) if self._cp.has_section(section) else {}

    def items_as(self, section, type):
        iv = {}
        for k, v in self.items(section).items():
            try:
                iv[k] = type(v)
            except ValueError:
                pass
        return iv

    def tostr(self):
        buf = io.StringIO()
        self._cp.write(buf)
        return buf.getvalue()
