"""Import shim that lets the reference package run under Numba's CUDA simulator.

Used only by ``tests/golden/make_reference_fixtures.py`` when it generates
fixtures from the reference's own kernels on the CPU.  The image has Numba's
in-tree ``numba.cuda`` (with its simulator) but not the ``numba-cuda``
distribution the reference probes for, and lacks the CellML/CuPy packages
it imports at module level.  The shim:

1. registers an empty ``numba_cuda`` package so the backend probe passes;
2. provides stub modules for ``numba.cuda.core`` (caching classes),
   ``numba.cuda.serialize`` (``dumps``) and ``numba.cuda.utils``;
3. provides permissive stub modules for ``lxml``, ``rdflib``, ``pint``,
   ``cupy`` and ``cupyx`` (only the unused CellML/CuPy paths need them);
4. exposes ``numba.cuda.local/shared/const`` as proxies to the simulator's
   current kernel context, for device helpers whose ``cuda`` global the
   simulator does not swap.
"""

import builtins
import importlib.abc
import importlib.machinery
import os
import pickle
import sys
import types


def _package(name):
    mod = types.ModuleType(name)
    mod.__path__ = []
    mod.__spec__ = importlib.machinery.ModuleSpec(name, None, is_package=True)
    sys.modules[name] = mod
    return mod


_package("numba_cuda")


class _Anything:
    def __init__(self, *args, **kwargs):
        pass

    def __call__(self, *args, **kwargs):
        return _Anything()

    def __getattr__(self, name):
        return _Anything()

    def __mro_entries__(self, bases):
        return (object,)


class _StubModule(types.ModuleType):
    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return _Anything()


_STUB_TOPS = ("lxml", "rdflib", "pint", "cupy", "cupyx")
_NUMBA_STUBS = ("numba.cuda.core", "numba.cuda.serialize", "numba.cuda.utils")


class _StubFinder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    def find_spec(self, fullname, path, target=None):
        top = fullname.split(".")[0]
        if top in _STUB_TOPS or any(fullname == p or fullname.startswith(p + ".") for p in _NUMBA_STUBS):
            return importlib.machinery.ModuleSpec(fullname, self, is_package=True)
        return None

    def create_module(self, spec):
        mod = _StubModule(spec.name)
        mod.__path__ = []
        return mod

    def exec_module(self, module):
        if module.__name__ == "numba.cuda.core.caching":
            for cls in ("_CacheLocator", "CacheImpl", "IndexDataCacheFile"):
                setattr(module, cls, type(cls, (), {}))
        if module.__name__ == "numba.cuda.serialize":
            module.dumps = pickle.dumps


sys.meta_path.insert(0, _StubFinder())


def _patch_simulator():
    import numba.cuda as cuda_mod
    from numba.cuda.simulator import kernel as sim_kernel

    class _ContextProxy:
        def __init__(self, attr):
            self._attr = attr

        def __getattr__(self, name):
            return getattr(getattr(sim_kernel._get_kernel_context(), self._attr), name)

    for attr in ("local", "shared", "const"):
        if not hasattr(cuda_mod, attr):
            setattr(cuda_mod, attr, _ContextProxy(attr))


_patched = False
_original_import = builtins.__import__


def _import_hook(name, *args, **kwargs):
    global _patched
    module = _original_import(name, *args, **kwargs)
    if (not _patched and os.environ.get("NUMBA_ENABLE_CUDASIM") == "1"
            and "numba.cuda.simulator.kernel" in sys.modules):
        _patched = True
        _patch_simulator()
    return module


builtins.__import__ = _import_hook
