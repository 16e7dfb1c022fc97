"""ORACLE -- test infrastructure only, and only in a container where the reference
source tree is present (it does not exist where the GPU tests run).

Imports the reference's own exmarg.search (the CPU path: numpy + numba) from the
reference source tree so that its outputs can pin the restatement and the golden
vectors.  Its top-level imports need healpy and lalsuite, which are absent, so
empty stand-in modules are registered for them first; the only lalsuite use on
the analysed path is the template profile (exmarg/profiles.py:26-47), which is
replaced by exmarg_b200.synth.profile (same return signature).  numba caches are
sent to a writable directory because the reference tree is read-only.

The source tree (the directory holding the `exmarg` package) is named by the
EXMARG_REFERENCE_SRC environment variable or passed as an argument.
"""

import os
import sys
import tempfile
import types

ENV = "EXMARG_REFERENCE_SRC"


def source_dir(src=None):
    """the reference source directory: the argument, else $EXMARG_REFERENCE_SRC (None if neither)"""
    return src or os.environ.get(ENV) or None


def available(src=None):
    src = source_dir(src)
    return bool(src) and os.path.isdir(os.path.join(src, "exmarg", "search"))


def import_reference(src=None):
    """the reference's exmarg.search module, with the TaylorF2 profile patched in"""
    src = source_dir(src)
    if not available(src):
        raise ImportError("reference source tree not found (pass its src directory or set %s); got %r" % (ENV, src))
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "exmarg_ref_numba"))
    for name in ("healpy", "lal", "lalsimulation"):
        if name not in sys.modules:
            sys.modules[name] = types.ModuleType(name)
    sys.modules["lalsimulation"].IMRPhenomXAS = 0
    if src not in sys.path:
        sys.path.insert(0, src)
    import exmarg.search as search
    import exmarg.search.bank as bank_mod
    import exmarg.profiles as prof_mod
    from exmarg_b200 import synth
    bank_mod.profile = synth.profile
    prof_mod.profile = synth.profile
    return search
