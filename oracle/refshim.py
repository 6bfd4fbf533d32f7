"""Loader for the reference's own CPU simulation code (test infrastructure only).

This module is part of the oracle: it is used by the parity tests and by the
fixture generator under ``tests/golden/`` to execute the reference's numba
kernels (``idi/simulation/cpu.py`` and ``idi/simulation/time.py``) unmodified,
on injected, seeded inputs.  Nothing in the product package imports it.

The reference package cannot be imported as ``import idi`` in this image:
``numexpr`` and ``h5py`` are not installed and ``idi/simulation/__init__.py``
probes for cupy.  So the loader

* registers a stand-in ``h5py`` module (only imported, never used on the path),
* registers a stand-in ``numexpr`` whose ``evaluate`` evaluates the handful of
  elementwise expressions the reference uses with numpy, in the caller's
  namespace (``time.py:94`` ``exp(-1j*(s*k-phases))[/d]``, and the
  ``idi/util/random.py`` expressions),
* builds a synthetic package whose ``__path__`` points at the reference tree,
  and imports ``util``, ``simulation.cpu``, ``simulation.time`` and
  ``simulation.simobj`` from it without running ``simulation/__init__.py``.

The reference tree location comes from ``IDI_REFERENCE``, else the read-only
checkout of the development container (``REF_ROOT``, the one place that names
it; the fixture generators, the Makefile's reference target and ``build()``
take it from here).  :func:`available` reports whether it is present.
"""

from __future__ import annotations

import importlib.util
import os
import sys
import types

import numpy as np

REF_ROOT = os.environ.get("IDI_REFERENCE", "/root/reference")
_PKG = "_idi_reference"


def available() -> bool:
    return os.path.isfile(os.path.join(REF_ROOT, "idi", "simulation", "cpu.py"))


_NE_FUNCS = {
    "exp": np.exp,
    "sqrt": np.sqrt,
    "sin": np.sin,
    "cos": np.cos,
    "log": np.log,
    "expm1": np.expm1,
    "log1p": np.log1p,
    "abs": np.abs,
    "real": np.real,
    "imag": np.imag,
    "sum": np.sum,  # numexpr's reduction sum(expr, axis=...)
}


def _ne_evaluate(expr, local_dict=None, global_dict=None, out=None, **_kw):
    frame = sys._getframe(1)
    ns = dict(frame.f_globals)
    ns.update(frame.f_locals)
    if global_dict:
        ns.update(global_dict)
    if local_dict:
        ns.update(local_dict)
    ns.update(_NE_FUNCS)
    res = eval(expr, {"__builtins__": {}}, ns)
    if out is not None:
        out[...] = res
        return out
    return np.asarray(res)


def _install_stubs():
    if "numexpr" not in sys.modules:
        ne = types.ModuleType("numexpr")
        ne.evaluate = _ne_evaluate
        ne.__stub__ = True
        sys.modules["numexpr"] = ne
    if "h5py" not in sys.modules:
        h5 = types.ModuleType("h5py")
        h5.__stub__ = True
        sys.modules["h5py"] = h5


def _load(modname: str, path: str, is_pkg: bool = False):
    full = f"{_PKG}.{modname}" if modname else _PKG
    if full in sys.modules:
        return sys.modules[full]
    if is_pkg:
        spec = importlib.util.spec_from_file_location(
            full, os.path.join(path, "__init__.py"), submodule_search_locations=[path]
        )
    else:
        spec = importlib.util.spec_from_file_location(full, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[full] = mod
    spec.loader.exec_module(mod)
    return mod


_cache = {}


def load():
    """Return a namespace with the reference modules ``cpu``, ``time``, ``simobj``, ``common``, ``util``."""
    if _cache:
        return types.SimpleNamespace(**_cache)
    if not available():
        raise RuntimeError(f"reference tree not found at {REF_ROOT}")
    _install_stubs()
    idi_dir = os.path.join(REF_ROOT, "idi")
    root = types.ModuleType(_PKG)
    root.__path__ = [idi_dir]
    sys.modules[_PKG] = root
    util = _load("util", os.path.join(idi_dir, "util"), is_pkg=True)
    sim = types.ModuleType(f"{_PKG}.simulation")
    sim.__path__ = [os.path.join(idi_dir, "simulation")]
    sys.modules[f"{_PKG}.simulation"] = sim
    cpu = _load("simulation.cpu", os.path.join(idi_dir, "simulation", "cpu.py"))
    tim = _load("simulation.time", os.path.join(idi_dir, "simulation", "time.py"))
    simobj = _load("simulation.simobj", os.path.join(idi_dir, "simulation", "simobj.py"))
    common = _load("simulation.common", os.path.join(idi_dir, "simulation", "common.py"))
    _cache.update(cpu=cpu, time=tim, simobj=simobj, util=util, common=common)
    return types.SimpleNamespace(**_cache)


def load_module(relname: str):
    """One more module of the reference package, e.g. ``reconstruction.cpusimple``
    (after :func:`load`; a subpackage is registered as an empty package, so its
    ``__init__`` with GPU imports does not run)."""
    load()
    idi_dir = os.path.join(REF_ROOT, "idi")
    parts = relname.split(".")
    for i in range(1, len(parts)):
        pkg = f"{_PKG}." + ".".join(parts[:i])
        if pkg not in sys.modules:
            m = types.ModuleType(pkg)
            m.__path__ = [os.path.join(idi_dir, *parts[:i])]
            sys.modules[pkg] = m
    return _load(relname, os.path.join(idi_dir, *parts[:-1], parts[-1] + ".py"))


class InjectedObject:
    """Duck-typed simobject (``.N``, ``.k``, ``.E``, ``.get()``, ``.get2()``) over fixed arrays.

    Mirrors the contract of ``idi/simulation/simobj.py:42-66``: ``get2()`` returns
    positions ``(N,3)`` and phases ``(N,1)``; ``get()`` their concatenation ``(N,4)``.
    Successive calls walk through a list of phase draws so that multi-image calls
    see independent, seeded phases.
    """

    def __init__(self, E, pos, phases):
        self.E = E
        self._pos = np.ascontiguousarray(pos, dtype=np.float64)
        ph = np.asarray(phases, dtype=np.float64)
        if ph.ndim == 1:
            ph = ph[None, :]
        self._phases = ph
        self._i = 0

    @property
    def N(self):
        return self._pos.shape[0]

    @property
    def k(self):
        return 2 * np.pi / (1.24 / self.E)

    def get2(self):
        ph = self._phases[self._i % len(self._phases)][:, None].copy()
        self._i += 1
        return self._pos.copy(), ph

    def get(self):
        p, ph = self.get2()
        return np.ascontiguousarray(np.concatenate([p, ph], -1))
