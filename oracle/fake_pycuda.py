"""Host stand-in for pycuda — TEST INFRASTRUCTURE ONLY.

Lets the reference's own Python engine (``simulation_toolkit.simulation_engine``
from the reference tree: ``DiffSim3d``, ``DwiSim3d``, ``SimGeometry3D``) run in a
container without a GPU or pycuda, so that its outputs can be recorded as
golden fixtures (tests/golden/make_golden.py).

* ``gpuarray.GPUArray`` wraps a numpy array (``.get()``, slicing, arithmetic).
* ``compiler.SourceModule(code)`` compiles the reference's template-substituted
  kernel source for the CPU (oracle/build.py) and ``get_function(name)``
  returns a launcher that emulates the grid on the host.
* Draws: ``set_normals(table)`` installs the injected normal table
  ``[N][nsteps][maxk]``; each walk launch is one time step, numbered from 0.
"""
from __future__ import annotations

import ctypes
import sys
import types

import numpy as np

from oracle.build import build_reference_kernel

_state = {"normals": None, "philox": None, "uniforms": None, "step": 0, "modules": [], "log": None}


class GPUArray:
    def __init__(self, arr):
        self.arr = np.ascontiguousarray(arr)

    # pycuda-like surface used by the reference engine and tests
    def get(self):
        return self.arr.copy()

    def copy(self):
        return GPUArray(self.arr.copy())

    @property
    def shape(self):
        return self.arr.shape

    @property
    def dtype(self):
        return self.arr.dtype

    @property
    def size(self):
        return self.arr.size

    def __getitem__(self, idx):
        return GPUArray(self.arr[idx])

    def _o(self, o):
        return o.arr if isinstance(o, GPUArray) else o

    def __sub__(self, o):
        return GPUArray(self.arr - self._o(o))

    def __add__(self, o):
        return GPUArray(self.arr + self._o(o))

    def __mul__(self, o):
        return GPUArray(self.arr * self._o(o))

    def __truediv__(self, o):
        return GPUArray(self.arr / self._o(o))

    def __pow__(self, p):
        return GPUArray(self.arr ** p)

    def ptr(self):
        return ctypes.c_void_p(self.arr.ctypes.data)


def _to_gpu(a):
    return GPUArray(np.array(a))


def _zeros(shape, dtype=np.float32):
    return GPUArray(np.zeros(shape, dtype=dtype))


def _ones(shape, dtype=np.float32):
    return GPUArray(np.ones(shape, dtype=dtype))


def _sum(a):
    return GPUArray(np.array(a.arr.sum()))


_SIGS = {
    "initstates": ("ref_run_initstates", False),
    "seedSpinsKernel": ("ref_run_seed", False),
    "randomWalk3d": ("ref_run_walk", True),
    "randomWalk3d_phase": ("ref_run_walk_phase", True),
    "randomWalk3d_phase_multidirr": ("ref_run_walk_multidir", True),
}


def _carg(a):
    if isinstance(a, GPUArray):
        return a.ptr()
    if isinstance(a, np.float32):
        return ctypes.c_float(float(a))
    if isinstance(a, np.uint32):
        return ctypes.c_uint(int(a))
    if isinstance(a, (np.int32, np.intc)):
        return ctypes.c_int(int(a))
    if isinstance(a, (int, np.integer)):
        return ctypes.c_int(int(a))
    raise TypeError(f"unsupported kernel argument {type(a)}")


class _Kernel:
    def __init__(self, lib, name):
        self.lib = lib
        self.name = name
        self.launcher, self.is_walk = _SIGS.get(name, (None, False))

    def __call__(self, *args, block=(1, 1, 1), grid=(1, 1)):
        if self.launcher is None:
            raise NotImplementedError(f"kernel {self.name} is not emulated on the host")
        fn = getattr(self.lib, self.launcher)
        fn.restype = None
        cargs = [ctypes.c_int(int(grid[0])), ctypes.c_int(int(block[0]))]
        if self.is_walk:
            cargs.append(ctypes.c_int(_state["step"]))
            _state["step"] += 1
            if _state["log"] is not None:
                _state["log"].append([float(a) for a in args if isinstance(a, np.float32)])
        cargs += [_carg(a) for a in args]
        fn(*cargs)


class SourceModule:
    def __init__(self, code, no_extern_c=False, **kw):
        self.path = build_reference_kernel(code)
        self.lib = ctypes.CDLL(str(self.path))
        self.lib.ref_set_normals.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        self.lib.ref_set_uniforms.argtypes = [ctypes.c_void_p, ctypes.c_int]
        self.lib.ref_set_philox.argtypes = [ctypes.c_uint, ctypes.c_uint, ctypes.c_uint]
        _state["modules"].append(self)
        self._apply()

    def _apply(self):
        n = _state["normals"]
        if n is not None:
            self.lib.ref_set_normals(n.ctypes.data, n.shape[1], n.shape[2])
        if _state["philox"] is not None:
            self.lib.ref_set_philox(*_state["philox"])
        u = _state["uniforms"]
        if u is not None:
            self.lib.ref_set_uniforms(u.ctypes.data, u.shape[1])
        else:
            self.lib.ref_set_uniforms(None, 0)

    def get_function(self, name):
        return _Kernel(self.lib, name)

    def exhausted(self) -> bool:
        return bool(self.lib.ref_exhausted())


def set_normals(table: np.ndarray):
    """Install normals[N][nsteps][maxk] (float32) and restart the step count."""
    table = np.ascontiguousarray(table, dtype=np.float32)
    _state["normals"] = table
    _state["philox"] = None
    _state["step"] = 0
    for m in _state["modules"]:
        m._apply()


def set_philox(key0: int, key1: int = 0, stream: int = 0):
    """Draw the reference's normals from the oracle's Philox stream at
    (walker, step, draw), component k % 3 of draw k // 3."""
    _state["normals"] = None
    _state["philox"] = (key0 & 0xFFFFFFFF, key1 & 0xFFFFFFFF, stream & 0xFFFFFFFF)
    _state["step"] = 0
    for m in _state["modules"]:
        m._apply()


def set_uniforms(table):
    _state["uniforms"] = None if table is None else np.ascontiguousarray(table, dtype=np.float32)
    for m in _state["modules"]:
        m._apply()


def record_scalars(log):
    """Append the float scalar arguments of every walk launch to `log`
    (None stops recording)."""
    _state["log"] = log


def reset_step(step: int = 0):
    _state["step"] = step


def install():
    """Register the stand-in modules under the pycuda names."""
    pkg = types.ModuleType("pycuda")
    autoinit = types.ModuleType("pycuda.autoinit")
    driver = types.ModuleType("pycuda.driver")
    driver.Context = types.SimpleNamespace(synchronize=lambda: None)
    gpuarray = types.ModuleType("pycuda.gpuarray")
    gpuarray.GPUArray = GPUArray
    gpuarray.to_gpu = _to_gpu
    gpuarray.zeros = _zeros
    gpuarray.ones = _ones
    gpuarray.sum = _sum
    compiler = types.ModuleType("pycuda.compiler")
    compiler.SourceModule = SourceModule
    curandom = types.ModuleType("pycuda.curandom")
    pkg.autoinit, pkg.driver, pkg.gpuarray, pkg.compiler, pkg.curandom = autoinit, driver, gpuarray, compiler, curandom
    for name, mod in [("pycuda", pkg), ("pycuda.autoinit", autoinit), ("pycuda.driver", driver),
                      ("pycuda.gpuarray", gpuarray), ("pycuda.compiler", compiler),
                      ("pycuda.curandom", curandom)]:
        sys.modules[name] = mod
