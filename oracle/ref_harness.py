"""ORACLE HARNESS -- test infrastructure, not product code.

Imports the reference BLonD Python package from a read-only checkout with its
C++ backend pointed at the library that ``oracle/Makefile`` compiles from the
reference's own sources (``oracle/_ref/libblond_ref_{double,single}.so``).
It is used only by ``tests/golden/gen_golden.py`` in a container that holds
the reference checkout; the generated fixtures are what the tests read.

The reference imports matplotlib / h5py at module level
(``blond/llrf/cavity_feedback.py:23``, ``blond/input_parameters/ring_options.py``
via ``blond/plots``); neither is installed here, so a permissive stub module is
installed for them.  Nothing on the tracking path calls into the stubs.
"""
from __future__ import annotations

import importlib.abc
import importlib.machinery
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: BLOND_REFERENCE_ROOT, else a checkout named
# "reference" beside this repository
DEFAULT_REF = os.environ.get(
    "BLOND_REFERENCE_ROOT",
    os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))

_STUB_ROOTS = ("matplotlib", "pylab", "mpl_toolkits", "h5py")


class _Anything(types.ModuleType):
    """A module whose every attribute is another callable stub."""

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        sub = _Anything(f"{self.__name__}.{name}")
        setattr(self, name, sub)
        return sub

    def __call__(self, *args, **kwargs):
        return _Anything(self.__name__ + "()")


class _StubFinder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    def find_spec(self, fullname, path, target=None):
        if fullname.split(".")[0] in _STUB_ROOTS:
            return importlib.machinery.ModuleSpec(fullname, self, is_package=True)
        return None

    def create_module(self, spec):
        mod = _Anything(spec.name)
        mod.__path__ = []
        return mod

    def exec_module(self, module):
        return None


def import_reference(precision: str = "double", ref_root: str = DEFAULT_REF,
                     fast_math: bool = True):
    """Import ``blond`` from ``ref_root`` backed by the oracle/_ref library.

    Returns the imported ``blond`` package.  Must be called before anything
    else imports ``blond``.
    """
    tag = "" if fast_math else "nofm_"
    lib = os.path.join(HERE, "_ref", f"libblond_ref_{tag}{precision}.so")
    if not os.path.exists(lib):
        raise FileNotFoundError(
            f"{lib} missing: run `make -C oracle ref` with the reference present")
    if not any(isinstance(f, _StubFinder) for f in sys.meta_path):
        sys.meta_path.insert(0, _StubFinder())
    os.environ["LIBBLOND"] = lib
    if ref_root not in sys.path:
        sys.path.insert(0, ref_root)
    import blond  # noqa: F401
    from blond.utils import bmath as bm
    bm.use_cpp()
    if precision == "single":
        bm.use_precision("single")
        from blond.utils import butils_wrap_cpp as _cpp
        _cpp.load_libblond("single")  # honours LIBBLOND
    assert bm.device == "CPU_CPP", bm.device
    return blond
