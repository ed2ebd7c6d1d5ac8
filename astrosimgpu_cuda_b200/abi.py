"""ctypes mirror of the C ABI types declared in include/astrosim.h.

Pure layout definitions: importing this module loads no library.
"""
import ctypes as C
import math

ABI_VERSION = 1

OK = 0
ERR_INVALID_ARG = 1
ERR_CUDA = 2
ERR_OUT_OF_MEMORY = 3
ERR_UNSUPPORTED = 4
ERR_NO_DEVICE = 5
ERR_TIMEOUT = 6
ERR_STATE = 7
ERR_IO = 8
ERR_PEER = 9

PRECISION_FP64 = 0
PRECISION_FP32 = 1

STATE = {
    "Ca": 0, "IP3": 1, "h": 2, "V": 3, "w": 4, "g_ex": 5, "dg_ex": 6, "g_in": 7, "dg_in": 8,
    "I_sic": 9, "stp_x": 10, "stp_u": 11, "stp_t_last": 12, "Ca_tot": 13, "IP3_0": 14,
    "tau_IP3": 15, "delta_IP3": 16, "V_reset": 17, "b": 18, "sic_factor": 19,
}
ASTRO_STATES = ("Ca", "IP3", "h", "Ca_tot", "IP3_0", "tau_IP3", "delta_IP3", "sic_factor")

CSR = {"exc": 0, "inh": 1, "sic": 2, "e2a": 3}


class Config(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("n_total", C.c_uint32),
        ("seed", C.c_uint64),
        ("dt", C.c_double),
        ("substeps", C.c_int32),
        ("block", C.c_int32),
        ("pre_ms", C.c_double),
        ("sim_ms", C.c_double),
        ("w_n2a", C.c_double),
        ("w_a2n", C.c_double),
        ("stp_enabled", C.c_int32),
        ("precision", C.c_int32),
        ("neuron_drive_scale", C.c_double),
        ("device", C.c_int32),
        ("raster_steps", C.c_int32),
        ("reserved", C.c_int32 * 8),
    ]


class Summary(C.Structure):
    _fields_ = [
        ("n_total", C.c_uint32), ("n_exc", C.c_uint32), ("n_inh", C.c_uint32), ("n_astro", C.c_uint32),
        ("p_primary", C.c_double),
        ("n_exc_edges", C.c_uint64), ("n_inh_edges", C.c_uint64),
        ("n_e2a_edges", C.c_uint64), ("n_sic_edges", C.c_uint64),
        ("pre_steps", C.c_int64), ("sim_steps", C.c_int64),
        ("total_steps", C.c_int64), ("steps_done", C.c_int64),
        ("spikes_total", C.c_uint64), ("spikes_measured", C.c_uint64),
        ("mean_rate_hz", C.c_double), ("mean_ca", C.c_double),
        ("active_astro", C.c_uint32), ("engaged_astro", C.c_uint32),
        ("sic_th", C.c_double), ("build_seconds", C.c_double), ("run_seconds", C.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class RequestResult(C.Structure):
    _fields_ = [("summary", Summary), ("latency_s", C.c_double), ("queue_s", C.c_double), ("build_s", C.c_double),
                ("run_s", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("done", C.c_uint64), ("failed", C.c_uint64), ("pending", C.c_uint64),
                ("building", C.c_uint64), ("running", C.c_uint64), ("bytes_in_use", C.c_uint64),
                ("budget_bytes", C.c_uint64), ("uptime_s", C.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


def default_config(**overrides):
    """Python-side twin of astrosim_config_default (reference defaults, src/astrosim_fused.cu:792-805)."""
    cfg = Config()
    cfg.struct_size = C.sizeof(Config)
    cfg.n_total = 1000
    cfg.seed = 1
    cfg.dt = 0.1
    cfg.substeps = 1
    cfg.block = 0  # autotuned; the reference launches 128-thread blocks (--block 128)
    cfg.pre_ms = 1000.0
    cfg.sim_ms = 5000.0
    cfg.w_n2a = math.nan
    cfg.w_a2n = math.nan
    cfg.stp_enabled = 1
    cfg.precision = PRECISION_FP64
    cfg.neuron_drive_scale = 1.0
    cfg.device = 0
    cfg.raster_steps = 0
    for k, v in overrides.items():
        if k == "precision" and isinstance(v, str):
            v = {"fp64": PRECISION_FP64, "fp32": PRECISION_FP32}[v.lower()]
        if not hasattr(cfg, k):
            raise AttributeError(f"astrosim_config has no field {k!r}")
        setattr(cfg, k, v)
    return cfg


def scaling(n_total):
    """Fixed-in-degree scaling law, src/astrosim_fused.cu:606-614."""
    def lround(x):
        return int(math.floor(x + 0.5))
    n_exc = max(1, lround(n_total * 0.8))
    n_inh = max(1, n_total - n_exc)
    n_astro = max(1, lround(n_total / 5.0))
    p = min(1.0, 80.0 / n_exc)
    return n_exc, n_inh, n_astro, p
