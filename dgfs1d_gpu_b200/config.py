"""INI configuration with the lookup interface the DGFS drivers use.

Same section/option names and lookup methods as the reference's
``Dictionary`` (dgfs1D/dictionary.py:18-137): ``[config] precision =
double|float`` selects the working dtype; ``-v section::key value`` style
overrides are passed as a nested ``defaults`` mapping.
"""
import configparser
import json
import os
import re

import numpy as np

_DTYPES = {'float': np.float32, 'double': np.float64}

# Names an initial- or boundary-condition expression may use: the function
# vocabulary of the reference's expression evaluator (nputil.py:12-20), so
# that its configuration files evaluate unchanged.
_EXPR_NAMES = {
    '__builtins__': None,
    'exp': np.exp, 'log': np.log, 'sin': np.sin, 'asin': np.arcsin,
    'cos': np.cos, 'acos': np.arccos, 'tan': np.tan, 'atan': np.arctan,
    'atan2': np.arctan2, 'abs': np.abs, 'pow': np.power, 'sqrt': np.sqrt,
    'tanh': np.tanh, 'pi': np.pi, 'linspace': np.linspace,
    'logspace': np.logspace}


def npeval(expr, variables):
    """Evaluate a configuration expression with NumPy (arrays broadcast).

    As in the reference: no ``**`` or ``^`` (use pow), only arithmetic,
    comparison and grouping characters, and no attribute access."""
    if '^' in expr or '**' in expr:
        raise ValueError('Direct exponentiation is not supported; use pow')
    if not re.match(r'[A-Za-z0-9 \t\n\r.,+\-*/%()<>=]+$', expr):
        raise ValueError('Invalid characters in expression')
    names = '|'.join(map(re.escape, list(_EXPR_NAMES) + list(variables)))
    if re.search(r'(%s|\))\s*\.' % names, expr):
        raise ValueError('Invalid expression')
    return eval(expr, dict(_EXPR_NAMES), dict(variables))


def _floatify(m):
    txt = m.group(0)
    return txt if ('.' in txt or 'e' in txt or 'E' in txt) else txt + '.0'


class Config:
    def __init__(self, inistr=None, defaults=None):
        cp = configparser.ConfigParser(inline_comment_prefixes=[';'],
                                       interpolation=None)
        cp.optionxform = str
        if inistr:
            cp.read_string(inistr)
        if defaults:
            cp.read_dict(defaults)
        self._cp = cp
        self._dtypename = self.lookupordefault('config', 'precision', 'double')
        if self._dtypename not in _DTYPES:
            raise ValueError(f'precision must be float or double, '
                             f'not {self._dtypename!r}')
        self._dtype = _DTYPES[self._dtypename]

    @staticmethod
    def load(path_or_file, defaults=None):
        if isinstance(path_or_file, str):
            with open(path_or_file) as fh:
                return Config(fh.read(), defaults)
        return Config(path_or_file.read(), defaults)

    @staticmethod
    def overrides(pairs):
        """Turn [('mesh::Ne', '4'), ...] into a read_dict mapping."""
        out = {}
        for key, value in pairs:
            sect, opt = key.split('::', 1)
            out.setdefault(sect, {})[opt] = str(value)
        return out

    def has_section(self, section):
        return self._cp.has_section(section)

    def lookup(self, section, option):
        return os.path.expandvars(self._cp.get(section, option))

    def lookupordefault(self, section, option, default):
        try:
            return type(default)(self._cp.get(section, option))
        except (configparser.Error, ValueError, TypeError):
            return default

    def lookupfloat(self, section, option):
        return self._dtype(self.lookup(section, option))

    def lookupfloats(self, section, options):
        return [self.lookupfloat(section, o) for o in options]

    def lookupint(self, section, option):
        return int(self.lookup(section, option))

    def lookupints(self, section, options):
        return [self.lookupint(section, o) for o in options]

    def lookupexpr(self, section, option, subs=None):
        expr = self.lookup(section, option)
        if not re.match(r'[A-Za-z0-9 \t\n\r.,+\-*/%()<>=\{\}\$]+$', expr):
            raise ValueError('Invalid characters in expression')
        for k, v in (subs or {}).items():
            expr = re.sub(r'\b%s\b' % re.escape(k), v, expr)
        # integer literals become floats (pow(2, -1) must not be integral)
        expr = re.sub(r'(?<![A-Za-z_0-9.])(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?',
                      _floatify, expr)
        return '(%s)' % expr

    def section_values(self, section, dtype):
        """{option: value} of the options of a section that convert to dtype
        (JSON lists to arrays); others are left out."""
        out = {}
        for k, v in self._cp.items(section):
            try:
                if '[' in v:
                    out[k] = self.lookup_list(section, k, dtype)
                else:
                    out[k] = dtype(v)
            except (ValueError, TypeError):
                pass
        return out

    def lookup_list(self, section, option, dtype):
        return np.array([dtype(v) for v in json.loads(self.lookup(section,
                                                                  option))])

    def lookupfloat_list(self, section, option):
        return self.lookup_list(section, option, self._dtype)

    def lookupint_list(self, section, option):
        return self.lookup_list(section, option, int)

    @property
    def dtypename(self):
        return self._dtypename

    @property
    def dtype(self):
        return self._dtype
