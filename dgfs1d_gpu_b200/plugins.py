"""Plugin lookup by class attribute, as the DGFS drivers select models.

``subclass_where(Base, scattering_model='vhs-gll')`` returns the first
(depth-first) subclass whose attribute equals the key, else KeyError -- the
semantics of dgfs1D/nputil.py:44-58.
"""


def subclasses(cls, just_leaf=False):
    sc = cls.__subclasses__()
    ssc = [g for s in sc for g in subclasses(s, just_leaf)]
    return [s for s in sc if not just_leaf or not s.__subclasses__()] + ssc


def subclass_where(cls, **kwargs):
    k, v = next(iter(kwargs.items()))
    for s in subclasses(cls):
        if getattr(s, k, None) == v:
            return s
    raise KeyError("No subclasses of {0} with cls.{1} == '{2}'"
                   .format(cls.__name__, k, v))
