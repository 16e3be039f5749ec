"""CPU oracle (test infrastructure only): ctypes wrapper of liboracle.so, the Float64
restatement of the reference's TimeStep! in oracle/pi_oracle.cpp.

Only tests, __graft_entry__.smoke() and the CPU-baseline leg of bench.py use this module; the
product package never imports it.
"""
import ctypes as ct
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "planktonindividuals.jl_b200"))

from PlanktonIndividuals._native import CModel  # noqa: E402

LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build(force=False):
    srcs = [os.path.join(HERE, "pi_oracle.cpp"), os.path.join(ROOT, "include", "pi_numerics.h"),
            os.path.join(ROOT, "include", "pib200.h")]
    stale = not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in srcs)
    if force or stale:
        subprocess.run(["make", "-C", HERE], check=True, stdout=subprocess.DEVNULL)
    return LIB


def load():
    global _lib
    if _lib is None:
        build()
        _lib = ct.CDLL(LIB)
        dp = ct.POINTER(ct.c_double)
        _lib.orc_get_field.restype = ct.c_int
        _lib.orc_get_field.argtypes = [ct.c_void_p, ct.c_int32, dp]
        _lib.orc_get_rates.restype = ct.c_int
        _lib.orc_get_rates.argtypes = [ct.c_void_p, ct.c_int32, dp]
        _lib.orc_exp.restype = ct.c_double
        _lib.orc_exp.argtypes = [ct.c_double]
        _lib.orc_pow_int.restype = ct.c_double
        _lib.orc_pow_int.argtypes = [ct.c_double, ct.c_int]
        for name in ("orc_log", "orc_pow"):
            getattr(_lib, name).restype = ct.c_double
        _lib.orc_log.argtypes = [ct.c_double]
        _lib.orc_pow.argtypes = [ct.c_double, ct.c_double]
        _lib.orc_draw3.restype = None
        _lib.orc_draw3.argtypes = [ct.c_uint64, ct.c_uint32, ct.c_uint32, ct.c_uint32, ct.c_uint32, dp]
        _lib.orc_num_threads.restype = ct.c_int
    return _lib


FIELDS = {"par": 0, "Chl": 1, "pop": 2, "u1": 31, "v1": 32, "w1": 33, "u0": 34, "temp": 35}


class OracleModel(CModel):
    """Same methods as the product's native model, backed by the CPU oracle."""

    def __init__(self, grid, bgc_params, phyt_params, nsp, capacity, seed, mode="quota"):
        super().__init__(load(), "orc_", grid, bgc_params, phyt_params, nsp, capacity, seed, mode=mode)

    def get_field(self, name_or_idx):
        which = FIELDS.get(name_or_idx, name_or_idx)
        out = np.empty(self.G, dtype=np.float64)
        r = self.lib.orc_get_field(self.h, int(which), out.ctypes.data_as(ct.POINTER(ct.c_double)))
        if r:
            raise ValueError(f"bad field {name_or_idx}")
        return out.reshape(self.gshape, order="F")

    def get_plk(self, n):
        return self.get_field(3 + n)

    def get_rates(self, sp):
        out = np.empty(9 * self.capacity, dtype=np.float64)
        self.lib.orc_get_rates(self.h, int(sp), out.ctypes.data_as(ct.POINTER(ct.c_double)))
        names = ("PS", "VDOC", "VNH4", "VNO3", "VPO4", "rChl", "resp", "BS", "exu")
        return {k: out[q * self.capacity:(q + 1) * self.capacity] for q, k in enumerate(names)}


def from_workload(wl):
    m = OracleModel(wl.grid, wl.bgc, wl.phyt, wl.nsp, wl.capacity, wl.seed, mode=getattr(wl, "mode", "quota"))
    m.set_state(wl.individuals, wl.tracers)
    return m


def pi_exp(x):
    return load().orc_exp(float(x))


def pow_int(x, n):
    return load().orc_pow_int(float(x), int(n))


def pi_log(x):
    return load().orc_log(float(x))


def pi_pow(x, y):
    return load().orc_pow(float(x), float(y))


def draw3(seed, iteration, species, purpose, slot):
    r = (ct.c_double * 3)()
    load().orc_draw3(seed, iteration, species, purpose, slot, r)
    return tuple(r)


def num_threads():
    return load().orc_num_threads()
