"""B200-native tripartite neuron-astrocyte network simulator.

Python host side of the C ABI in include/astrosim.h (library
``lib/libastrosim_b200.so``, built by ``make -C astrosimgpu_cuda_b200`` or
``__graft_entry__.build()``).  The reference program (src/astrosim_fused.cu)
exposes only a CLI; :class:`Simulation` mirrors its run structure
(create -> step -> summary) on top of the library, and every computation runs in
the library's CUDA kernels.  There is no CPU path: importing works without a
GPU, but creating a simulation needs the built library and a CUDA device.
"""
import ctypes as C
import json
import math
import os
import subprocess

import numpy as np

from . import abi
from .abi import default_config, scaling  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libastrosim_b200.so")
CLI_PATH = os.path.join(LIB_DIR, "astrosim")

_lib = None


class AstrosimError(RuntimeError):
    """A library call returned a non-zero status."""

    def __init__(self, code, msg):
        super().__init__(f"astrosim error {code}: {msg}")
        self.code = code


def build(jobs=8):
    """Compiles the CUDA library and the CLI for sm_100a (nvcc; no GPU needed)."""
    subprocess.run(["make", "-s", "-C", HERE, f"-j{jobs}"], check=True)


def library_path():
    """The library this process uses: lib/libastrosim_b200.so, or the path in
    ASTROSIM_LIBRARY (e.g. the FP32 measurement build lib/libastrosim_b200_fp32ieee.so)."""
    return os.environ.get("ASTROSIM_LIBRARY") or LIB_PATH


def lib():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `make -C {HERE}` "
                          "(the simulator has no CPU fallback)")
    L = C.CDLL(path)
    P = C.c_void_p
    u32p = C.POINTER(C.c_uint32)
    L.astrosim_config_default.argtypes = [C.POINTER(abi.Config)]
    L.astrosim_config_default.restype = None
    L.astrosim_last_error.restype = C.c_char_p
    L.astrosim_abi_version.restype = C.c_int
    L.astrosim_create.argtypes = [C.POINTER(abi.Config), C.POINTER(P)]
    L.astrosim_step.argtypes = [P, C.c_int64]
    L.astrosim_summary.argtypes = [P, C.POINTER(abi.Summary)]
    L.astrosim_destroy.argtypes = [P]
    L.astrosim_spike_counts.argtypes = [P, C.c_int64, C.c_int64, u32p]
    L.astrosim_raster.argtypes = [P, u32p, C.c_size_t]
    L.astrosim_get_state.argtypes = [P, C.c_int, C.POINTER(C.c_double), C.c_size_t]
    L.astrosim_get_csr.argtypes = [P, C.c_int, u32p, C.c_size_t, u32p, C.c_size_t,
                                   C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]
    L.astrosim_dump_edges.argtypes = [P, C.c_char_p]
    L.astrosim_last_step_ms.argtypes = [P, C.POINTER(C.c_double)]
    L.astrosim_device_info.argtypes = [C.c_int, C.c_char_p, C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    E = C.c_void_p
    L.astrosim_ensemble_create.argtypes = [C.POINTER(abi.Config), C.c_uint32, C.POINTER(E)]
    L.astrosim_ensemble_step.argtypes = [E, C.c_int64]
    L.astrosim_ensemble_summary.argtypes = [E, C.c_uint32, C.POINTER(abi.Summary)]
    L.astrosim_ensemble_get_state.argtypes = [E, C.c_uint32, C.c_int, C.POINTER(C.c_double), C.c_size_t]
    L.astrosim_ensemble_spike_counts.argtypes = [E, C.c_uint32, C.c_int64, C.c_int64, u32p]
    L.astrosim_ensemble_last_step_ms.argtypes = [E, C.POINTER(C.c_double)]
    L.astrosim_ensemble_build_seconds.argtypes = [E, C.POINTER(C.c_double)]
    L.astrosim_ensemble_shared_constants.argtypes = [E, C.POINTER(C.c_int)]
    L.astrosim_ensemble_destroy.argtypes = [E]
    for name in ("astrosim_ensemble_create", "astrosim_ensemble_step", "astrosim_ensemble_summary",
                 "astrosim_ensemble_get_state", "astrosim_ensemble_spike_counts", "astrosim_ensemble_last_step_ms",
                 "astrosim_ensemble_build_seconds", "astrosim_ensemble_shared_constants",
                 "astrosim_ensemble_destroy"):
        getattr(L, name).restype = C.c_int
    S = C.c_void_p
    L.astrosim_server_create.argtypes = [C.c_int, C.c_int, C.c_uint64, C.c_int, C.POINTER(S)]
    L.astrosim_server_submit.argtypes = [S, C.POINTER(abi.Config), C.POINTER(C.c_uint64)]
    L.astrosim_server_pump.argtypes = [S, C.c_int64]
    L.astrosim_server_result.argtypes = [S, C.c_uint64, C.POINTER(abi.RequestResult), C.POINTER(C.c_int)]
    L.astrosim_server_get_stats.argtypes = [S, C.POINTER(abi.ServerStats)]
    L.astrosim_server_destroy.argtypes = [S]
    L.astrosim_selfcheck_division.argtypes = [C.c_int, C.POINTER(C.c_double), C.c_size_t, C.c_uint64, C.c_uint64,
                                              C.POINTER(C.c_uint64)]
    L.astrosim_selfcheck_division.restype = C.c_int
    L.astrosim_record_calcium.argtypes = [P, C.c_int64, C.c_uint32, C.c_uint32, C.c_int64]
    L.astrosim_calcium_samples.argtypes = [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.astrosim_copy_calcium.argtypes = [P, C.c_int64, C.c_int64, C.POINTER(C.c_double), C.c_int]
    L.astrosim_sync.argtypes = [P]
    L.astrosim_create_with_biology.argtypes = [C.POINTER(abi.Config), C.c_char_p, C.POINTER(P)]
    L.astrosim_create_with_biology.restype = C.c_int
    L.astrosim_biology_names.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
    L.astrosim_biology_names.restype = C.c_int
    L.astrosim_biology_value.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(C.c_double)]
    L.astrosim_biology_value.restype = C.c_int
    L.astrosim_ensemble_create_with_biology.argtypes = [C.POINTER(abi.Config), C.c_uint32, C.POINTER(C.c_char_p),
                                                        C.POINTER(P)]
    L.astrosim_ensemble_create_with_biology.restype = C.c_int
    L.astrosim_server_submit_with_biology.argtypes = [P, C.POINTER(abi.Config), C.c_char_p, C.POINTER(C.c_uint64)]
    L.astrosim_server_submit_with_biology.restype = C.c_int
    for name in ("astrosim_record_calcium", "astrosim_calcium_samples", "astrosim_copy_calcium", "astrosim_sync"):
        getattr(L, name).restype = C.c_int
    for name in ("astrosim_server_create", "astrosim_server_submit", "astrosim_server_pump", "astrosim_server_result",
                 "astrosim_server_get_stats", "astrosim_server_destroy"):
        getattr(L, name).restype = C.c_int
    for name in ("astrosim_create", "astrosim_step", "astrosim_summary", "astrosim_destroy",
                 "astrosim_spike_counts", "astrosim_raster", "astrosim_get_state", "astrosim_get_csr",
                 "astrosim_dump_edges", "astrosim_last_step_ms", "astrosim_device_info"):
        getattr(L, name).restype = C.c_int
    if L.astrosim_abi_version() != abi.ABI_VERSION:
        raise ImportError("libastrosim_b200.so ABI version mismatch")
    _lib = L
    return L


def check(code):
    if code != abi.OK:
        raise AstrosimError(code, lib().astrosim_last_error().decode())


def _biology_json(biology):
    if biology is None:
        return None
    if isinstance(biology, (str, bytes)):
        return biology.encode() if isinstance(biology, str) else biology
    return json.dumps(biology).encode()


def biology_names():
    """Names of the biology constants that astrosim_create_with_biology accepts."""
    need = C.c_size_t()
    check(lib().astrosim_biology_names(None, 0, C.byref(need)))
    buf = C.create_string_buffer(need.value)
    check(lib().astrosim_biology_names(buf, need.value, None))
    return buf.value.decode().split(",")


def biology_value(name, biology=None):
    """A biology constant's value after `biology` overrides (defaults when None)."""
    v = C.c_double()
    check(lib().astrosim_biology_value(_biology_json(biology), name.encode(), C.byref(v)))
    return v.value


def selfcheck_division(divisors, samples=1 << 20, seed=1, device=0):
    """Mismatches between the FP64 path's division by a constant and IEEE x / y on the device."""
    d = np.ascontiguousarray(divisors, dtype=np.float64)
    out = C.c_uint64(0)
    check(lib().astrosim_selfcheck_division(device, d.ctypes.data_as(C.POINTER(C.c_double)), d.size, samples, seed,
                                            C.byref(out)))
    return int(out.value)


def _u32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def device_info(device=0):
    name = C.create_string_buffer(256)
    major, minor = C.c_int(), C.c_int()
    check(lib().astrosim_device_info(device, name, 256, C.byref(major), C.byref(minor)))
    return name.value.decode(), major.value, minor.value


class Simulation:
    """One network resident on the GPU (astrosim_create / step / summary / destroy)."""

    def __init__(self, cfg=None, biology=None, **overrides):
        """`biology`: overrides of the biology constants, a {name: value} dict or JSON text."""
        self.cfg = cfg if cfg is not None else default_config(**overrides)
        self._h = C.c_void_p()
        check(lib().astrosim_create_with_biology(C.byref(self.cfg), _biology_json(biology), C.byref(self._h)))
        n_exc, n_inh, n_astro, _ = scaling(self.cfg.n_total)
        self.n_exc, self.n_inh, self.n_astro = n_exc, n_inh, n_astro
        self.n_neurons = n_exc + n_inh

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().astrosim_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n):
        check(lib().astrosim_step(self._h, int(n)))

    def summary(self):
        s = abi.Summary()
        check(lib().astrosim_summary(self._h, C.byref(s)))
        return s.as_dict()

    def last_step_ms(self):
        ms = C.c_double()
        check(lib().astrosim_last_step_ms(self._h, C.byref(ms)))
        return ms.value

    def spike_counts(self, first=0, n=None):
        if n is None:
            n = self.summary()["steps_done"] - first
        out = np.empty(n, dtype=np.uint32)
        check(lib().astrosim_spike_counts(self._h, first, n, _u32p(out)))
        return out

    def raster(self):
        words = (self.n_neurons + 31) // 32
        steps = self.cfg.raster_steps
        out = np.zeros(max(1, words * steps), dtype=np.uint32)
        check(lib().astrosim_raster(self._h, _u32p(out), out.size))
        return out[: words * steps].reshape(steps, words)

    def state(self, name):
        n = self.n_astro if name in abi.ASTRO_STATES else self.n_neurons
        out = np.empty(n, dtype=np.float64)
        check(lib().astrosim_get_state(self._h, abi.STATE[name], out.ctypes.data_as(C.POINTER(C.c_double)), n))
        return out

    def csr(self, name):
        which = abi.CSR[name]
        nt, ne = C.c_uint32(), C.c_uint64()
        check(lib().astrosim_get_csr(self._h, which, None, 0, None, 0, C.byref(nt), C.byref(ne)))
        rs = np.empty(nt.value + 1, dtype=np.uint32)
        src = np.empty(max(1, ne.value), dtype=np.uint32)
        check(lib().astrosim_get_csr(self._h, which, _u32p(rs), rs.size, _u32p(src), src.size, None, None))
        return rs, src[: ne.value]

    def dump_edges(self, path):
        check(lib().astrosim_dump_edges(self._h, os.fsencode(path)))

    def record_calcium(self, every, first=0, n=None, max_samples=1024):
        """Records Ca of astrocytes [first, first + n) after every `every`-th step, from the next step on."""
        n = self.n_astro - first if n is None else n
        check(lib().astrosim_record_calcium(self._h, int(every), int(first), int(n), int(max_samples)))
        self._rec_n = n

    def calcium_samples(self):
        """(samples recorded so far, the step after which sample 0 was taken)."""
        k, t0 = C.c_int64(), C.c_int64()
        check(lib().astrosim_calcium_samples(self._h, C.byref(k), C.byref(t0)))
        return k.value, t0.value

    def calcium(self, first=0, n=None):
        """Recorded samples [first, first + n) as an array [n, n_astro_recorded]."""
        if n is None:
            n = self.calcium_samples()[0] - first
        out = np.empty((n, self._rec_n), dtype=np.float64)
        check(lib().astrosim_copy_calcium(self._h, first, n, out.ctypes.data_as(C.POINTER(C.c_double)), 1))
        return out


class Ensemble:
    """Many independent networks stepped together (astrosim_ensemble_*)."""

    def __init__(self, cfgs, biology=None):
        """`biology`: None, or one override (dict / JSON text / None) per network."""
        self.cfgs = list(cfgs)
        arr = (abi.Config * len(self.cfgs))(*self.cfgs)
        self._h = C.c_void_p()
        if biology is None:
            check(lib().astrosim_ensemble_create(arr, len(self.cfgs), C.byref(self._h)))
        else:
            texts = (C.c_char_p * len(self.cfgs))(*[_biology_json(b) for b in biology])
            check(lib().astrosim_ensemble_create_with_biology(arr, len(self.cfgs), texts, C.byref(self._h)))
        self.sizes = [scaling(c.n_total) for c in self.cfgs]

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().astrosim_ensemble_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.cfgs)

    def step(self, n):
        check(lib().astrosim_ensemble_step(self._h, int(n)))

    def summary(self, i):
        s = abi.Summary()
        check(lib().astrosim_ensemble_summary(self._h, i, C.byref(s)))
        return s.as_dict()

    def state(self, i, name):
        n_exc, n_inh, n_astro, _ = self.sizes[i]
        n = n_astro if name in abi.ASTRO_STATES else n_exc + n_inh
        out = np.empty(n, dtype=np.float64)
        check(lib().astrosim_ensemble_get_state(self._h, i, abi.STATE[name],
                                                out.ctypes.data_as(C.POINTER(C.c_double)), n))
        return out

    def spike_counts(self, i, first=0, n=None):
        if n is None:
            n = self.summary(i)["steps_done"] - first
        out = np.empty(n, dtype=np.uint32)
        check(lib().astrosim_ensemble_spike_counts(self._h, i, first, n, _u32p(out)))
        return out

    def last_step_ms(self):
        ms = C.c_double()
        check(lib().astrosim_ensemble_last_step_ms(self._h, C.byref(ms)))
        return ms.value

    def build_seconds(self):
        s = C.c_double()
        check(lib().astrosim_ensemble_build_seconds(self._h, C.byref(s)))
        return s.value

    def shared_constants(self):
        """True when the networks differ only in seed, sizes, drive rates and w_a2n."""
        v = C.c_int()
        check(lib().astrosim_ensemble_shared_constants(self._h, C.byref(v)))
        return bool(v.value)


class Server:
    """Continuous-batching request loop (astrosim_server_*)."""

    def __init__(self, precision="fp32", device=0, budget_bytes=0, builders=8):
        prec = {"fp64": abi.PRECISION_FP64, "fp32": abi.PRECISION_FP32}[precision]
        self.precision = precision
        self._h = C.c_void_p()
        check(lib().astrosim_server_create(device, prec, budget_bytes, builders, C.byref(self._h)))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().astrosim_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, cfg=None, biology=None, **overrides):
        cfg = cfg if cfg is not None else default_config(precision=self.precision, **overrides)
        rid = C.c_uint64()
        check(lib().astrosim_server_submit_with_biology(self._h, C.byref(cfg), _biology_json(biology), C.byref(rid)))
        return rid.value

    def pump(self, windows=10):
        check(lib().astrosim_server_pump(self._h, int(windows)))

    def result(self, rid):
        r = abi.RequestResult()
        done = C.c_int()
        check(lib().astrosim_server_result(self._h, rid, C.byref(r), C.byref(done)))
        if not done.value:
            return None
        out = r.summary.as_dict()
        out.update(latency_s=r.latency_s, queue_s=r.queue_s, build_s=r.build_s, run_s=r.run_s)
        return out

    def stats(self):
        s = abi.ServerStats()
        check(lib().astrosim_server_get_stats(self._h, C.byref(s)))
        return s.as_dict()


def rate_hz(spikes, n_neurons, ms):
    return spikes / (n_neurons * ms * 1e-3) if ms > 0 else math.nan
