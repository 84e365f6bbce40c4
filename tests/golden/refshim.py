"""Import shim for running the reference's pure-Python modules in this container.

Fixture generation only (tests/golden/make_golden.py): it is never imported by
the test suite, bench.py or the package, and it needs the reference checkout,
which exists only on the build machine.

The reference imports its C++ modules through ``cppimport`` (absent here) and a
``Timer`` from ``taskloaf`` (absent here), and uses the NumPy aliases ``np.int``
and ``np.float`` that NumPy 2 removed.  This shim:
  * serves ``cppimport.cppimport(name)`` from the modules that oracle/Makefile
    (target ``ref``) compiled from the reference sources into oracle/_ref/;
  * stubs ``taskloaf.Timer``;
  * restores the two NumPy aliases.
"""
import importlib.machinery
import importlib.util
import os
import sys
import types

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
# the reference checkout: TCT_REFERENCE, else a directory named "reference"
# beside this repository
REF = os.environ.get("TCT_REFERENCE") or os.path.join(os.path.dirname(REPO), "reference")
if not os.path.isdir(os.path.join(REF, "tectosaur")):
    raise ImportError("refshim: no reference checkout at %r (set TCT_REFERENCE)" % REF)
REF_BUILD = os.path.join(REPO, "oracle", "_ref")


def _load_ext(short):
    for suffix in importlib.machinery.EXTENSION_SUFFIXES:
        path = os.path.join(REF_BUILD, short + suffix)
        if os.path.exists(path):
            spec = importlib.util.spec_from_file_location(short, path)
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            return mod
    # modules this build does not compile (Mako-templated or unused) become
    # empty placeholders; touching them raises AttributeError.
    return types.ModuleType(short)


def install():
    if "cppimport" in sys.modules and getattr(sys.modules["cppimport"], "_tct_shim", False):
        return
    np.int = int
    np.float = float
    cpp = types.ModuleType("cppimport")
    cpp._tct_shim = True
    cpp.set_rtld_flags = lambda *a, **k: None
    cpp.cppimport = lambda name: _load_ext(name.split(".")[-1])
    cpp.setup_pybind11 = lambda cfg: None
    cpp.turn_off_strict_prototypes = lambda: None
    sys.modules["cppimport"] = cpp
    tl = types.ModuleType("taskloaf")

    class Timer:
        def __init__(self, *a, **k):
            pass

        def report(self, *a, **k):
            pass

    tl.Timer = Timer
    sys.modules["taskloaf"] = tl
    # The reference picks PyCUDA or PyOpenCL at import time; neither exists
    # here.  A placeholder backend lets the host-side modules import; any
    # attempt to reach a device raises.
    backend = types.ModuleType("tectosaur.util.cuda")

    def _no_device(*a, **k):
        raise RuntimeError("no PyCUDA/PyOpenCL device in this container")

    for name in ("compile", "empty_gpu", "zeros_gpu", "to_gpu", "threaded_get"):
        setattr(backend, name, _no_device)
    backend.cluda_preamble = ""
    sys.modules["tectosaur.util.cuda"] = backend
    if REF not in sys.path:
        sys.path.insert(0, REF)


install()
