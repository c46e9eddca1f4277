"""Slab decomposition of a uniform mesh over GPUs, one part per GPU along the slowest axis (z on a 3-D mesh, y on a 2-D
one), as the reference's MPI strips split it (SimulationRun.cpp:1011-1446 run_mpi, MPIDecomposition.cpp:114-242).

A part (``Part``, over fvg_create_part) holds its own planes plus ghost planes beyond each interface. Its step is a fixed
sequence of phases (fvg_part_phase); between two phases the parts either exchange their boundary planes with their
neighbours or all-reduce (MAX) a wave speed, on the parts' streams. Two exchangers carry that out:

* ``LocalExchange``: all parts in this process (one GPU or several), by device copies between their buffers; this is how
  a decomposition is checked against the whole run on a single GPU;
* ``DistExchange``: one part per process, torch.distributed point-to-point sends / receives and all-reduce (NCCL
  between GPUs, enqueued on the part's stream: no host synchronisation; gloo on CPU tensors in the host tests);
* ``HostStagedExchange``: one part per process with the planes staged through pinned host memory and moved by a CPU
  process group (gloo): processes that share a GPU, or GPUs without a device-to-device path, exchange this way (each
  communication point waits on the host for the part's stream; no kernel ever waits for another process).

Every part takes the same phases and the same communication in the same order. The cells beyond an interface are the
neighbour's, and dt comes from the all-reduced speed, so a decomposed run reproduces the whole run's bits.
"""
import ctypes

import numpy as np

from .runtime import FVG_OK, Run

COMM_DONE, COMM_EXCHANGE, COMM_ALLREDUCE = 0, 1, 2


def split_axis(params):
    """The split axis of a mesh: 2 (z) in 3-D, 1 (y) in 2-D."""
    return 2 if int(params.get("nz", 1)) > 1 else 1


def part_range(n, nparts, index):
    """(first, count) of part `index` of `nparts` over n planes: the first n % nparts parts hold one plane more (the
    rule of fvg_create_part)."""
    q, r = divmod(n, nparts)
    return index * q + min(index, r), q + (1 if index < r else 0)


def split_state(params, U, nparts):
    """The states of the parts of a whole state (cells of 5 doubles in the reference's order)."""
    nx, ny, nz = int(params["nx"]), int(params["ny"]), int(params.get("nz", 1))
    ax = split_axis(params)
    grid = np.asarray(U).reshape(nz, ny, nx, 5)
    n = nz if ax == 2 else ny
    out = []
    for p in range(nparts):
        f, c = part_range(n, nparts, p)
        sl = grid[f:f + c] if ax == 2 else grid[:, f:f + c]
        out.append(np.ascontiguousarray(sl).reshape(-1, 5))
    return out


def join_states(params, states):
    """The whole state of the parts' states (the inverse of split_state)."""
    nx, ny, nz = int(params["nx"]), int(params["ny"]), int(params.get("nz", 1))
    ax = split_axis(params)
    if ax == 2:
        return np.concatenate([np.asarray(s).reshape(-1, ny, nx, 5) for s in states], axis=0).reshape(-1, 5)
    return np.concatenate([np.asarray(s).reshape(nz, -1, nx, 5) for s in states], axis=1).reshape(-1, 5)


class _DeviceArray:
    """__cuda_array_interface__ of a float64 device array the library owns (torch.as_tensor views it without a copy)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8", "data": (int(ptr), False), "version": 3}


class Part(Run):
    """Part `index` of `nparts` of the run of `params` (fvg_create_part)."""

    def __init__(self, params, nparts, index, U=None, precision=0, device=0):
        super().__init__(params, U=None, precision=precision, device=device, part=(nparts, index))
        self.nparts, self.index, self.device = int(nparts), int(index), int(device)
        vals = [ctypes.c_int() for _ in range(6)]
        self.lib.fvg_part_info(self.h, *[ctypes.byref(v) for v in vals])
        self.axis, self.first, self.count, self.depth, lo, hi = (v.value for v in vals)
        self.peer_lo, self.peer_hi = bool(lo), bool(hi)
        ptrs = [ctypes.POINTER(ctypes.c_double)() for _ in range(5)]
        n = ctypes.c_longlong()
        self._check(self.lib.fvg_part_buffers(self.h, ctypes.byref(ptrs[0]), ctypes.byref(ptrs[1]), ctypes.byref(ptrs[2]), ctypes.byref(ptrs[3]),
                                              ctypes.byref(n), ctypes.byref(ptrs[4])), "part buffers")
        self.xcount = n.value
        self._ptrs = [ctypes.cast(p, ctypes.c_void_p).value for p in ptrs]
        self._tensors = None
        if U is not None:
            self.set_state(U)

    def tensors(self):
        """torch views of the device buffers: send_lo, send_hi, recv_lo, recv_hi (xcount doubles each), reduce (2)."""
        if self._tensors is None:
            import torch

            dev = torch.device("cuda", self.device)
            counts = [self.xcount] * 4 + [2]
            self._tensors = [torch.as_tensor(_DeviceArray(p, c), device=dev) for p, c in zip(self._ptrs, counts)]
        return self._tensors

    def begin(self, t_end, max_steps=0):
        self._check(self.lib.fvg_part_begin(self.h, float(t_end), int(max_steps)), "part begin")

    def phase(self, i):
        comm, n = ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.fvg_part_phase(self.h, int(i), ctypes.byref(comm), ctypes.byref(n)), f"part phase {i}")
        return comm.value, n.value

    def status(self):
        """(active, steps, t, dt, s_max) of the part's control block (synchronises its stream)."""
        a, st = ctypes.c_int(), ctypes.c_int()
        t, dt, s = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.fvg_part_status(self.h, ctypes.byref(a), ctypes.byref(st), ctypes.byref(t), ctypes.byref(dt), ctypes.byref(s)),
                    "part status")
        return bool(a.value), st.value, t.value, dt.value, s.value


class LocalExchange:
    """The communication of all parts of a decomposition held by this process, ordered on the parts' CUDA streams with
    events (no host synchronisation): a part's receive buffers are filled by copies on its own stream once the sending
    part's stream has packed them, and a sender's later work (its next pack) waits for those copies; the all-reduce runs
    on the first part's stream once every part has written its values and every part waits for its result."""

    def __init__(self, parts):
        import torch

        self.parts = list(parts)
        self.streams = [torch.cuda.ExternalStream(p.stream(), device=torch.device("cuda", p.device)) for p in self.parts]
        self.ready = [torch.cuda.Event() for _ in self.parts]
        self.copied = [torch.cuda.Event() for _ in self.parts]
        self.reduced = torch.cuda.Event()

    def _record_ready(self):
        for s, ev in zip(self.streams, self.ready):
            ev.record(s)

    def exchange(self):
        import torch

        self._record_ready()
        n = len(self.parts)
        for i, p in enumerate(self.parts):
            s = self.streams[i]
            with torch.cuda.stream(s):
                if p.peer_lo:   # the low neighbour's send_hi -> my recv_lo
                    j = (i - 1) % n
                    s.wait_event(self.ready[j])
                    p.tensors()[2].copy_(self.parts[j].tensors()[1])
                if p.peer_hi:   # the high neighbour's send_lo -> my recv_hi
                    j = (i + 1) % n
                    s.wait_event(self.ready[j])
                    p.tensors()[3].copy_(self.parts[j].tensors()[0])
            self.copied[i].record(s)
        for i, p in enumerate(self.parts):   # the sender's send buffers are free again once its receivers have copied them
            if p.peer_lo:
                self.streams[i].wait_event(self.copied[(i - 1) % n])
            if p.peer_hi:
                self.streams[i].wait_event(self.copied[(i + 1) % n])

    def allreduce(self, count):
        import torch

        self._record_ready()
        s0 = self.streams[0]
        with torch.cuda.stream(s0):
            for ev in self.ready:
                s0.wait_event(ev)
            red = torch.stack([p.tensors()[4][:count] for p in self.parts]).amax(dim=0)
            for p in self.parts:
                p.tensors()[4][:count].copy_(red)
        self.reduced.record(s0)
        for s in self.streams:
            s.wait_event(self.reduced)


class DistExchange:
    """The communication of this process's part with the other processes' parts (torch.distributed, one part per rank,
    rank = part index). `bufs` are the part's five tensors (send_lo, send_hi, recv_lo, recv_hi, reduce) and `stream` the
    CUDA stream its kernels run on (None for CPU tensors)."""

    def __init__(self, bufs, peer_lo, peer_hi, stream=None, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.bufs = bufs
        self.peer_lo, self.peer_hi = peer_lo, peer_hi
        self.stream = stream
        self.lo = (self.rank - 1) % self.world
        self.hi = (self.rank + 1) % self.world

    @classmethod
    def for_part(cls, part, group=None):
        import torch

        return cls(part.tensors(), part.peer_lo, part.peer_hi, torch.cuda.ExternalStream(part.stream(), device=torch.device("cuda", part.device)),
                   group)

    def _ctx(self):
        import contextlib

        import torch

        return torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext()

    def exchange(self):
        send_lo, send_hi, recv_lo, recv_hi, _ = self.bufs
        with self._ctx():
            if self.world == 1:   # a periodic axis on one part: its own planes
                if self.peer_lo:
                    recv_hi.copy_(send_lo)
                if self.peer_hi:
                    recv_lo.copy_(send_hi)
                return
            # sends first to the low then the high neighbour, receives first from the high then the low one: between
            # any two ranks the k-th send meets the k-th receive (also when both neighbours are one rank, world = 2)
            d = self.dist
            ops = []
            if self.peer_lo:
                ops.append(d.P2POp(d.isend, send_lo, self.lo, self.group))
            if self.peer_hi:
                ops.append(d.P2POp(d.isend, send_hi, self.hi, self.group))
            if self.peer_hi:
                ops.append(d.P2POp(d.irecv, recv_hi, self.hi, self.group))
            if self.peer_lo:
                ops.append(d.P2POp(d.irecv, recv_lo, self.lo, self.group))
            if ops:
                for r in d.batch_isend_irecv(ops):
                    r.wait()

    def allreduce(self, count):
        with self._ctx():
            if self.world > 1:
                self.dist.all_reduce(self.bufs[4][:count], op=self.dist.ReduceOp.MAX, group=self.group)


class HostStagedExchange:
    """DistExchange's communication through pinned host memory and a CPU (gloo) process group: before each exchange or
    all-reduce the part's stream is waited for, its send planes (or reduce slots) are copied to the host, moved between
    the processes, and the received planes copied back on the part's stream. The same pairing of sends and receives as
    DistExchange, so any number of ranks on any number of GPUs (several ranks may share one)."""

    def __init__(self, part, group=None):
        import torch
        import torch.distributed as dist

        self.dist, self.group, self.part = dist, group, part
        self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        self.lo, self.hi = (self.rank - 1) % self.world, (self.rank + 1) % self.world
        self.dev = part.tensors()
        self.stream = torch.cuda.ExternalStream(part.stream(), device=torch.device("cuda", part.device))
        self.host = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in self.dev]

    def exchange(self):
        import torch

        send_lo, send_hi, recv_lo, recv_hi, _ = self.dev
        h_send_lo, h_send_hi, h_recv_lo, h_recv_hi, _ = self.host
        p = self.part
        with torch.cuda.stream(self.stream):
            if p.peer_lo:
                h_send_lo.copy_(send_lo, non_blocking=True)
            if p.peer_hi:
                h_send_hi.copy_(send_hi, non_blocking=True)
        self.stream.synchronize()
        if self.world == 1:
            if p.peer_lo:
                h_recv_hi.copy_(h_send_lo)
            if p.peer_hi:
                h_recv_lo.copy_(h_send_hi)
        else:
            d = self.dist
            ops = []
            if p.peer_lo:
                ops.append(d.P2POp(d.isend, h_send_lo, self.lo, self.group))
            if p.peer_hi:
                ops.append(d.P2POp(d.isend, h_send_hi, self.hi, self.group))
            if p.peer_hi:
                ops.append(d.P2POp(d.irecv, h_recv_hi, self.hi, self.group))
            if p.peer_lo:
                ops.append(d.P2POp(d.irecv, h_recv_lo, self.lo, self.group))
            if ops:
                for r in d.batch_isend_irecv(ops):
                    r.wait()
        with torch.cuda.stream(self.stream):
            if p.peer_hi:
                recv_hi.copy_(h_recv_hi, non_blocking=True)
            if p.peer_lo:
                recv_lo.copy_(h_recv_lo, non_blocking=True)

    def allreduce(self, count):
        import torch

        red, h_red = self.dev[4], self.host[4]
        with torch.cuda.stream(self.stream):
            h_red[:count].copy_(red[:count], non_blocking=True)
        self.stream.synchronize()
        if self.world > 1:
            self.dist.all_reduce(h_red[:count], op=self.dist.ReduceOp.MAX, group=self.group)
        with torch.cuda.stream(self.stream):
            red[:count].copy_(h_red[:count], non_blocking=True)


def advance(parts, exchanger, t_end, max_steps=0, check_every=1):
    """Advances the parts of this process (one part per process with DistExchange or HostStagedExchange, all of them
    with LocalExchange) toward t_end, at most max_steps steps (0: no limit); returns (steps, t). The parts' clocks are
    read (a host synchronisation) every `check_every` steps: steps past t_end or the step limit are gated off on the
    device on every part alike, so enqueuing a few more only costs their empty launches. Raises as fvg_run_until on
    divergence."""
    for p in parts:
        p.begin(t_end, max_steps)
    if any(p.cfg.time_scheme == 3 for p in parts):   # MUSCL-Hancock swaps its state buffers on the host every step
        check_every = 1
    while True:
        st = [p.status() for p in parts]
        active, steps, t = st[0][0], st[0][1], st[0][2]
        if any(s[:3] != st[0][:3] for s in st):
            raise RuntimeError(f"the parts' clocks differ: {st}")
        if not active:
            return steps, t
        for _ in range(max(1, int(check_every))):
            phase = 0
            while True:
                comms = [p.phase(phase) for p in parts]
                comm, n = comms[0]
                if comm == COMM_DONE:
                    break
                if comm == COMM_EXCHANGE:
                    exchanger.exchange()
                else:
                    exchanger.allreduce(n)
                phase += 1


def run_decomposed(params, U, nparts, t_end, max_steps=0, precision=0, device=0):
    """The whole run of `params` from state U as nparts parts in this process (LocalExchange); returns (state, steps, t)."""
    parts = [Part(params, nparts, i, U=s, precision=precision, device=device) for i, s in enumerate(split_state(params, U, nparts))]
    try:
        steps, t = advance(parts, LocalExchange(parts), t_end, max_steps)
        return join_states(params, [p.state() for p in parts]), steps, t
    finally:
        for p in parts:
            p.close()


__all__ = ["Part", "LocalExchange", "DistExchange", "HostStagedExchange", "advance", "run_decomposed", "split_state", "join_states", "part_range", "split_axis", "FVG_OK"]
