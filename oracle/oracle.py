"""TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.

ctypes wrapper around the FP64 CPU oracle (oracle/astrosim_oracle.cpp), a
restatement of the reference program's algorithm (src/astrosim_fused.cu).  Only
tests/, the smoke check and bench.py's CPU-baseline leg use it, as the checker.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from astrosimgpu_cuda_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libastrosim_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "astrosim_fused_ref")
REF_BIN_F32 = os.path.join(HERE, "_ref", "astrosim_fused_ref_f32")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        u32p = C.POINTER(C.c_uint32)
        L.oracle_rng_bits.restype = C.c_uint64
        L.oracle_rng_bits.argtypes = [C.c_uint64] * 3
        L.oracle_rng_uniform.restype = C.c_double
        L.oracle_rng_uniform.argtypes = [C.c_uint64] * 3
        L.oracle_rng_normal.restype = C.c_double
        L.oracle_rng_normal.argtypes = [C.c_uint64] * 2
        L.oracle_rng_poisson.restype = C.c_int
        L.oracle_rng_poisson.argtypes = [C.c_uint64, C.c_uint64, C.c_double]
        L.oracle_seq_normals.argtypes = [C.c_uint64, C.c_uint64, C.c_size_t, C.POINTER(C.c_double)]
        L.oracle_create.restype = P
        L.oracle_create.argtypes = [C.POINTER(abi.Config), C.c_int]
        L.oracle_create_with_biology.restype = P
        L.oracle_create_with_biology.argtypes = [C.POINTER(abi.Config), C.c_int, C.POINTER(C.c_char_p),
                                                 C.POINTER(C.c_double), C.c_size_t]
        L.oracle_create_with_csr.restype = P
        L.oracle_create_with_csr.argtypes = [C.POINTER(abi.Config), C.c_int] + [u32p] * 8
        L.oracle_destroy.argtypes = [P]
        L.oracle_step.argtypes = [P, C.c_int64]
        L.oracle_summary.argtypes = [P, C.POINTER(abi.Summary)]
        L.oracle_get_state.restype = C.c_int64
        L.oracle_get_state.argtypes = [P, C.c_int, C.POINTER(C.c_double), C.c_size_t]
        L.oracle_get_csr.argtypes = [P, C.c_int, u32p, u32p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]
        L.oracle_spike_counts.argtypes = [P, C.c_int64, C.c_int64, u32p]
        L.oracle_raster.argtypes = [P, u32p, C.c_size_t]
        L.oracle_build_seconds.restype = C.c_double
        L.oracle_build_seconds.argtypes = [P]
        L.oracle_set_exp_perturbation.argtypes = [P, C.c_double]
        L.oracle_set_contraction.argtypes = [P, C.c_int]
        _lib = L
    return _lib


def _u32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def rng_bits(seed, stream, counter):
    return lib().oracle_rng_bits(seed, stream, counter)


def rng_uniform(seed, stream, counter):
    return lib().oracle_rng_uniform(seed, stream, counter)


def rng_normal(seed, stream):
    return lib().oracle_rng_normal(seed, stream)


def rng_poisson(seed, stream, lam):
    return lib().oracle_rng_poisson(seed, stream, lam)


def seq_normals(seed, stream, n):
    out = np.empty(n, dtype=np.float64)
    lib().oracle_seq_normals(seed, stream, n, out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


class OracleSim:
    """One FP64 network on the host, stepped exactly as the reference's time loop."""

    def __init__(self, cfg=None, threads=0, csrs=None, biology=None, **overrides):
        """`biology`: {name: value} overrides of the biology constants (flags as bool)."""
        self.cfg = cfg if cfg is not None else abi.default_config(**overrides)
        L = lib()
        if biology:
            names = (C.c_char_p * len(biology))(*[k.encode() for k in biology])
            values = (C.c_double * len(biology))(*[float(v) for v in biology.values()])
            self._h = L.oracle_create_with_biology(C.byref(self.cfg), threads, names, values, len(biology))
        elif csrs is None:
            self._h = L.oracle_create(C.byref(self.cfg), threads)
        else:
            arrs = []
            for k in ("exc", "inh", "sic", "e2a"):
                rs, src = csrs[k]
                arrs += [np.ascontiguousarray(rs, dtype=np.uint32), np.ascontiguousarray(src, dtype=np.uint32)]
            self._keep = arrs
            self._h = L.oracle_create_with_csr(C.byref(self.cfg), threads, *[_u32p(a) for a in arrs])
        if not self._h:
            raise ValueError("oracle_create rejected the configuration")
        n_exc, n_inh, n_astro, _ = abi.scaling(self.cfg.n_total)
        self.n_neurons = n_exc + n_inh
        self.n_astro = n_astro
        self.steps_done = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def perturb_exp(self, rate):
        """Moves the AdEx exponential one ulp for a fraction `rate` of its arguments (0: off)."""
        lib().oracle_set_exp_perturbation(self._h, float(rate))

    def contract(self, on=True):
        """Evaluates the neuron update with fused multiply-adds (a second correct rounding)."""
        lib().oracle_set_contraction(self._h, 1 if on else 0)

    def step(self, n):
        lib().oracle_step(self._h, n)
        self.steps_done += n

    def summary(self):
        s = abi.Summary()
        lib().oracle_summary(self._h, C.byref(s))
        return s.as_dict()

    def state(self, name):
        which = abi.STATE[name]
        n = lib().oracle_get_state(self._h, which, None, 0)
        out = np.empty(n, dtype=np.float64)
        lib().oracle_get_state(self._h, which, out.ctypes.data_as(C.POINTER(C.c_double)), n)
        return out

    def csr(self, name):
        which = abi.CSR[name]
        nt, ne = C.c_uint32(), C.c_uint64()
        lib().oracle_get_csr(self._h, which, None, None, C.byref(nt), C.byref(ne))
        rs = np.empty(nt.value + 1, dtype=np.uint32)
        src = np.empty(ne.value, dtype=np.uint32)
        lib().oracle_get_csr(self._h, which, _u32p(rs), _u32p(src), None, None)
        return rs, src

    def spike_counts(self, first=0, n=None):
        n = self.steps_done - first if n is None else n
        out = np.empty(n, dtype=np.uint32)
        if lib().oracle_spike_counts(self._h, first, n, _u32p(out)) != 0:
            raise ValueError("steps not done")
        return out

    def raster(self):
        words = (self.n_neurons + 31) // 32
        out = np.zeros(words * max(0, self.cfg.raster_steps), dtype=np.uint32)
        if out.size:
            lib().oracle_raster(self._h, _u32p(out), out.size)
        return out.reshape(max(0, self.cfg.raster_steps), words)

    def build_seconds(self):
        return lib().oracle_build_seconds(self._h)
