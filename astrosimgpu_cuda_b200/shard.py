"""One network split across GPUs (astrosim_shard_* / astrosim_shard_group_* in
include/astrosim.h).

:class:`ShardGroup` runs every rank in this process (rank r on ``devices[r]``);
:class:`ShardedSimulation` is one rank per process, with torch.distributed as the
plumbing: it checks that all ranks describe the same network, builds this rank's
part, makes sure every rank succeeded before anyone joins the NCCL communicator,
and hands rank 0's NCCL id to the others.  Both give results bit-identical to a
single-GPU :class:`~astrosimgpu_cuda_b200.Simulation` of the same configuration.
"""
import ctypes as C

import numpy as np

from . import abi, check, default_config, lib, scaling, _biology_json, _u32p

_ARGS_SET = False


def _lib():
    global _ARGS_SET
    L = lib()
    if not _ARGS_SET:
        P, u32p = C.c_void_p, C.POINTER(C.c_uint32)
        L.astrosim_shard_plan.argtypes = [C.c_uint32, C.c_int, C.c_int, u32p, u32p, u32p, u32p]
        L.astrosim_shard_unique_id.argtypes = [C.c_char_p]
        L.astrosim_shard_create.argtypes = [C.POINTER(abi.Config), C.c_char_p, C.c_int, C.c_int, C.POINTER(P)]
        L.astrosim_shard_connect.argtypes = [P, C.c_char_p]
        L.astrosim_shard_step.argtypes = [P, C.c_int64]
        L.astrosim_shard_summary.argtypes = [P, C.POINTER(abi.Summary)]
        L.astrosim_shard_get_state.argtypes = [P, C.c_int, C.POINTER(C.c_double), C.c_size_t]
        L.astrosim_shard_spike_counts.argtypes = [P, C.c_int64, C.c_int64, u32p]
        L.astrosim_shard_last_step_ms.argtypes = [P, C.POINTER(C.c_double)]
        L.astrosim_shard_destroy.argtypes = [P]
        L.astrosim_shard_set_timeout.argtypes = [P, C.c_double]
        L.astrosim_shard_selftest_wait.argtypes = [C.c_int, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                                   C.POINTER(C.c_double)]
        L.astrosim_shard_group_create.argtypes = [C.POINTER(abi.Config), C.c_char_p, C.c_int,
                                                  C.POINTER(C.c_int), C.POINTER(P)]
        L.astrosim_shard_group_step.argtypes = [P, C.c_int64]
        L.astrosim_shard_group_summary.argtypes = [P, C.POINTER(abi.Summary)]
        L.astrosim_shard_group_get_state.argtypes = [P, C.c_int, C.POINTER(C.c_double), C.c_size_t]
        L.astrosim_shard_group_spike_counts.argtypes = [P, C.c_int64, C.c_int64, u32p]
        L.astrosim_shard_group_destroy.argtypes = [P]
        L.astrosim_shard_group_get_csr.argtypes = [P, C.c_int, C.c_int, u32p, C.c_size_t, u32p, C.c_size_t, u32p,
                                                   u32p, C.POINTER(C.c_uint64)]
        for name in ("astrosim_shard_plan", "astrosim_shard_unique_id", "astrosim_shard_create",
                     "astrosim_shard_connect", "astrosim_shard_step", "astrosim_shard_summary",
                     "astrosim_shard_get_state", "astrosim_shard_spike_counts", "astrosim_shard_last_step_ms",
                     "astrosim_shard_destroy", "astrosim_shard_group_create", "astrosim_shard_group_step",
                     "astrosim_shard_group_summary", "astrosim_shard_group_get_state",
                     "astrosim_shard_group_spike_counts", "astrosim_shard_group_destroy",
                     "astrosim_shard_group_get_csr"):
            getattr(L, name).restype = C.c_int
        _ARGS_SET = True
    return L


def shard_plan(n_total, rank, world):
    """(neuron_lo, neuron_hi, astro_lo, astro_hi) owned by `rank` of `world` (no device needed)."""
    v = [C.c_uint32() for _ in range(4)]
    check(_lib().astrosim_shard_plan(n_total, rank, world, *[C.byref(x) for x in v]))
    return tuple(x.value for x in v)


def selftest_wait(scenario, timeout_s):
    """The deadline logic of the ranks' waits on a stand-in communicator (no device):
    (status, windows completed, stand-in aborted, seconds).  Scenarios as
    astrosim_shard_selftest_wait in include/astrosim.h."""
    done, aborted, waited = C.c_int(), C.c_int(), C.c_double()
    rc = _lib().astrosim_shard_selftest_wait(int(scenario), float(timeout_s), C.byref(done), C.byref(aborted),
                                             C.byref(waited))
    return rc, done.value, bool(aborted.value), waited.value


def unique_id():
    """A fresh 128-byte NCCL id (rank 0 makes it; every rank connects with the same bytes)."""
    buf = C.create_string_buffer(128)
    check(_lib().astrosim_shard_unique_id(buf))
    return buf.raw


def _state_array(get, h, name, n_neurons, n_astro):
    n = n_astro if name in abi.ASTRO_STATES else n_neurons
    out = np.empty(n, dtype=np.float64)
    check(get(h, abi.STATE[name], out.ctypes.data_as(C.POINTER(C.c_double)), n))
    return out


class ShardGroup:
    """Every rank of one sharded network in this process; rank r on devices[r]."""

    def __init__(self, cfg=None, world=2, devices=None, biology=None, **overrides):
        self.cfg = cfg if cfg is not None else default_config(**overrides)
        n_exc, n_inh, self.n_astro, _ = scaling(self.cfg.n_total)
        self.n_neurons = n_exc + n_inh
        self.world = world
        devs = None if devices is None else (C.c_int * world)(*devices)
        self._h = C.c_void_p()
        check(_lib().astrosim_shard_group_create(C.byref(self.cfg), _biology_json(biology), world, devs,
                                                 C.byref(self._h)))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib().astrosim_shard_group_destroy(self._h)
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
        check(_lib().astrosim_shard_group_step(self._h, int(n)))

    def summary(self):
        s = abi.Summary()
        check(_lib().astrosim_shard_group_summary(self._h, C.byref(s)))
        return s.as_dict()

    def state(self, name):
        return _state_array(_lib().astrosim_shard_group_get_state, self._h, name, self.n_neurons, self.n_astro)

    def spike_counts(self, first=0, n=None):
        if n is None:
            n = self.summary()["steps_done"] - first
        out = np.empty(n, dtype=np.uint32)
        check(_lib().astrosim_shard_group_spike_counts(self._h, first, n, _u32p(out)))
        return out

    def csr(self, rank, name):
        """(first_row, row_start, src) of CSR `name` as rank `rank` keeps it: the rows of its own cells."""
        which = abi.CSR[name]
        first, nr, ne = C.c_uint32(), C.c_uint32(), C.c_uint64()
        f = _lib().astrosim_shard_group_get_csr
        check(f(self._h, rank, which, None, 0, None, 0, C.byref(first), C.byref(nr), C.byref(ne)))
        rs = np.empty(nr.value + 1, dtype=np.uint32)
        src = np.empty(max(1, ne.value), dtype=np.uint32)
        check(f(self._h, rank, which, _u32p(rs), rs.size, _u32p(src), src.size, None, None, None))
        return first.value, rs, src[: ne.value]


def agree_on_config(cfg, biology, group=None):
    """Raises on every rank unless all ranks describe the same network (cfg.device aside)."""
    import torch.distributed as dist
    desc = {name: getattr(cfg, name) for name, _ in abi.Config._fields_ if name not in ("device", "reserved")}
    desc["biology"] = _biology_json(biology)
    world = dist.get_world_size(group)
    got = [None] * world
    dist.all_gather_object(got, desc, group=group)
    for r, d in enumerate(got):
        diff = sorted(k for k in desc if d.get(k) != desc[k] and not (d.get(k) != d.get(k) and desc[k] != desc[k]))
        if diff:
            raise ValueError(f"rank {r} describes a different network: {', '.join(diff)}")


def all_ranks_ok(ok, message, group=None):
    """True when `ok` holds on every rank; otherwise every rank raises with the failures."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    got = [None] * world
    dist.all_gather_object(got, (bool(ok), message), group=group)
    bad = [(r, m) for r, (o, m) in enumerate(got) if not o]
    if bad:
        raise RuntimeError("sharded network not created: " + "; ".join(f"rank {r}: {m}" for r, m in bad))
    return True


def share_id(make_id=unique_id, group=None):
    """Rank 0's id (from make_id) on every rank."""
    import torch.distributed as dist
    box = [make_id() if dist.get_rank(group) == 0 else None]
    dist.broadcast_object_list(box, src=0, group=group)
    return box[0]


class ShardedSimulation:
    """This process's rank of one network split across the torch.distributed group."""

    def __init__(self, cfg=None, biology=None, group=None, timeout_s=None, **overrides):
        """`timeout_s`: deadline of every wait on the other ranks (astrosim_shard_set_timeout);
        a rank that died or left then makes the others raise instead of hanging."""
        import torch.distributed as dist
        self.cfg = cfg if cfg is not None else default_config(**overrides)
        if dist.is_available() and dist.is_initialized():
            self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        else:
            self.rank, self.world = 0, 1  # no process group: the whole network on this process's GPU
        n_exc, n_inh, self.n_astro, _ = scaling(self.cfg.n_total)
        self.n_neurons = n_exc + n_inh
        if self.world > 1:
            agree_on_config(self.cfg, biology, group)
        self._h = C.c_void_p()
        rc = _lib().astrosim_shard_create(C.byref(self.cfg), _biology_json(biology), self.rank, self.world,
                                          C.byref(self._h))
        msg = "" if rc == abi.OK else lib().astrosim_last_error().decode()
        if self.world > 1:
            all_ranks_ok(rc == abi.OK, msg, group)  # nobody joins the communicator if a rank failed
        else:
            check(rc)
        if timeout_s is not None:
            check(_lib().astrosim_shard_set_timeout(self._h, float(timeout_s)))
        ident = share_id(group=group) if self.world > 1 else b"\0" * 128
        check(_lib().astrosim_shard_connect(self._h, ident))
        self.plan = shard_plan(self.cfg.n_total, self.rank, self.world)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _lib().astrosim_shard_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def step(self, n):
        check(_lib().astrosim_shard_step(self._h, int(n)))

    def summary(self):
        s = abi.Summary()
        check(_lib().astrosim_shard_summary(self._h, C.byref(s)))
        return s.as_dict()

    def state(self, name):
        return _state_array(_lib().astrosim_shard_get_state, self._h, name, self.n_neurons, self.n_astro)

    def last_step_ms(self):
        ms = C.c_double()
        check(_lib().astrosim_shard_last_step_ms(self._h, C.byref(ms)))
        return ms.value

    def spike_counts(self, first=0, n=None):
        if n is None:
            n = self.summary()["steps_done"] - first
        out = np.empty(n, dtype=np.uint32)
        check(_lib().astrosim_shard_spike_counts(self._h, first, n, _u32p(out)))
        return out
