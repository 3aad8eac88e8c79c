"""Slices sharded across processes, one process per GPU.

The loop of main.cpp:92-156 with the bunch split into contiguous slice
blocks (boundary.cpp:33-46: the first sliceN % N processes hold one slice
more).  Every slice's step is local, except the slippage shift: the slice that
leaves a block enters the next one (MPI_Transfer1F_Zplus of
fieldShareZ.cpp:39-78; the first block receives zeros).  Diagnostics are
reduced as the reference reduces them: the field energies and the twiss sums
are summed over processes (updateTotalEnergy.cpp:56-68, twiss.cpp:62-64), the
bunching factor stays process-local (saveFile.cpp:109-172).

The exchange is one send and one receive of 2 H planes per shifted iteration.
With the NCCL backend and GPU engines it stays in device memory: the planes
are read and written where the handle keeps them (felis_first_planes_device),
and the send, the receive and the copies are queued on the handle's own
stream, so nothing waits on the host and the planes cross NVLink once.  With
any other backend (gloo on CPU) the planes go through host buffers.
`exchange_in_process` does the same hand-over in device memory for blocks
held by one process.  Engines: `GpuEngine` (felis_b200.Handle in exchange
mode) and `OracleEngine` (the CPU restatement, used by the multi-process
tests).
"""
from __future__ import annotations

import numpy as np

from . import TIME_DEPENDENT


def slice_blocks(slice_n: int, world: int) -> list[tuple[int, int]]:
    """[(min_i, max_i)] per process (boundary.cpp:33-46)."""
    base, remain = divmod(slice_n, world)
    out, lo = [], 0
    for r in range(world):
        n = base + 1 if r < remain else base
        out.append((lo, lo + n))
        lo += n
    return out


def split_beam(beam: dict, lo: int, hi: int) -> dict:
    """Particles of slices [lo, hi) of a slice-major beam, offsets rebased."""
    off = np.asarray(beam["offsets"])
    a, b = int(off[lo]), int(off[hi])
    out = {k: np.asarray(beam[k])[a:b] for k in ("x", "y", "px", "py", "theta", "gamma")}
    out["offsets"] = off[lo:hi + 1] - a
    out["weights"] = np.asarray(beam["weights"])[lo:hi]
    return out


def split_field(field: np.ndarray, lo: int, hi: int) -> np.ndarray:
    """Planes of slices [lo, hi) of a full field [(S + 2), ny, nx] with zero
    ghost planes around them."""
    out = np.zeros((hi - lo + 2,) + field.shape[1:], dtype=field.dtype)
    out[1:-1] = field[1 + lo:1 + hi]
    return out


def twiss_from_sums(s: np.ndarray, species: int) -> np.ndarray:
    """twiss.cpp:66-80 on summed (x^2, y^2, x'^2, y'^2, x x', y y', count)."""
    out = np.zeros(6 * species)
    for sp in range(species):
        a = s[7 * sp:7 * sp + 7]
        cnt = a[6]
        if cnt > 0:
            ax2, ay2, axp, ayp, cx, cy = a[0] / cnt, a[1] / cnt, a[2] / cnt, a[3] / cnt, a[4] / cnt, a[5] / cnt
            ex, ey = np.sqrt(ax2 * axp - cx * cx), np.sqrt(ay2 * ayp - cy * cy)
            out[6 * sp:6 * sp + 6] = [ex, ax2 / ex, -cx / ex, ey, ay2 / ey, -cy / ey]
    return out


class _DeviceArray:
    """A complex128 vector in device memory, for torch.as_tensor (no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<c16", "data": (ptr, False), "version": 3,
                                         "strides": None}


class GpuEngine:
    """felis_b200.Handle of one slice block, in exchange mode."""

    def __init__(self, handle):
        self.h = handle
        self.h.set_slice_exchange(True)
        self.H, self.species, self.mode = handle.H, handle.species, handle.mode

    def plane_views(self):
        """torch views of the block's first-slice planes in device memory
        ([h][pol] order), valid until the next shift."""
        import torch

        n = self.h.nx * self.h.ny
        return [torch.as_tensor(_DeviceArray(p, n), device="cuda") for p in self.h.first_planes_device()]

    def stream(self):
        import torch

        return torch.cuda.ExternalStream(self.h.stream())

    def energy(self, it: int) -> np.ndarray:
        return self.h.total_energy(it)

    def sums(self, it: int) -> np.ndarray:
        return self.h.diagnostic_sums(it)

    def step(self, it: int) -> bool:
        self.h.step(it)
        lat = self.h.lattice()
        return not lat.drift_flag and self.mode == TIME_DEPENDENT

    def outgoing(self) -> np.ndarray:
        return self.h.first_planes()

    def incoming(self, planes: np.ndarray):
        self.h.set_first_planes(planes)


class OracleEngine:
    """The CPU restatement of one slice block, driven function by function in
    the order of main.cpp:117-155."""

    def __init__(self, oracle, mode: int):
        self.o = oracle
        self.H, self.species, self.mode = oracle.H, oracle.species, mode

    def energy(self, it: int) -> np.ndarray:
        return self.o.total_energy()

    def sums(self, it: int) -> np.ndarray:
        return self.o.diagnostic_sums()

    def step(self, it: int) -> bool:
        o = self.o
        o.solve_field()
        o.update_lattice(it, 0.0)
        o.transverse_push()
        o.update_lattice(it, 0.5)
        o.transverse_push()
        lat = o.lattice()
        if not lat.drift_flag:
            o.push_theta_gamma()
        else:
            o.drift_theta_gamma()
        o.periodic_particles()
        shifted = not lat.drift_flag and self.mode == TIME_DEPENDENT
        if shifted:
            o.shift_field()
        return shifted

    def outgoing(self) -> np.ndarray:
        # after shiftField the slice that left the block sits in the upper ghost plane
        return np.stack([np.stack([self.o.get_field(h, pol)[-1] for pol in (0, 1)]) for h in range(self.H)])

    def incoming(self, planes: np.ndarray):
        for h in range(self.H):
            for pol in (0, 1):
                f = self.o.get_field(h, pol)
                f[1] = planes[h, pol]
                self.o.set_field(h, pol, f)


class ShardedLoop:
    """Iterations of one process's slice block with the halo exchange and the
    cross-process reductions; every process calls run() with the same range."""

    def __init__(self, engine, dist, rank: int, world: int):
        self.e, self.dist, self.rank, self.world = engine, dist, rank, world
        self.device = None
        try:
            if dist.get_backend() == "nccl":
                import torch

                self.device = torch.device("cuda", torch.cuda.current_device())
        except Exception:
            self.device = None

    def _tensor(self, a: np.ndarray):
        import torch

        t = torch.from_numpy(np.ascontiguousarray(a))
        return t.to(self.device) if self.device is not None else t

    def _allreduce(self, a: np.ndarray) -> np.ndarray:
        t = self._tensor(a.astype(np.float64))
        self.dist.all_reduce(t)
        return t.cpu().numpy()

    def exchange(self):
        if self.device is not None and isinstance(self.e, GpuEngine):
            return self._exchange_device()
        out = self.e.outgoing()
        buf = np.ascontiguousarray(out.view(np.float64))
        req = None
        if self.rank + 1 < self.world:
            req = self.dist.isend(self._tensor(buf), self.rank + 1)
        recv = np.zeros_like(buf)
        if self.rank > 0:
            t = self._tensor(recv)
            self.dist.recv(t, self.rank - 1)
            recv = t.cpu().numpy()
        if req is not None:
            req.wait()
        self.e.incoming(recv.view(np.complex128).reshape(out.shape))

    def _exchange_device(self):
        """MPI_Transfer1F_Zplus in device memory over NCCL, on the handle's
        stream: the outgoing planes packed into one buffer and sent to rank +
        1; the planes of rank - 1 received and copied into place (zeros on
        rank 0)."""
        import torch

        views = self.e.plane_views()
        with torch.cuda.stream(self.e.stream()):
            ops, recv = [], None
            if self.rank + 1 < self.world:
                send = torch.view_as_real(torch.stack(views))
                ops.append(self.dist.P2POp(self.dist.isend, send, self.rank + 1))
            if self.rank > 0:
                recv = torch.empty((len(views), views[0].numel(), 2), dtype=torch.float64, device=views[0].device)
                ops.append(self.dist.P2POp(self.dist.irecv, recv, self.rank - 1))
            if ops:
                for req in self.dist.batch_isend_irecv(ops):
                    req.wait()
            for k, v in enumerate(views):
                if recv is None:
                    v.zero_()
                else:
                    v.copy_(torch.view_as_complex(recv[k]))

    def run(self, it0: int, it1: int):
        """Returns per-iteration (energy, twiss, bfactor) of the state at the
        start of each iteration, as main.cpp:117-124 writes them: energy and
        twiss of the whole bunch, the bunching factor of this block.  The
        block's unfinished bunching sums (2 H, then the weight) are kept in
        self.bunching_sums for callers that want the whole-bunch value."""
        H, ns = self.e.H, self.e.species
        E, T, B, self.bunching_sums = [], [], [], []
        for it in range(it0, it1):
            E.append(self._allreduce(self.e.energy(it)))
            s = self.e.sums(it)
            tw = self._allreduce(s[:7 * ns])
            T.append(twiss_from_sums(tw, ns))
            b = s[7 * ns:7 * ns + 2 * H + 1]
            self.bunching_sums.append(b)
            B.append(b[:-1] / b[-1])
            if self.e.step(it):
                self.exchange()
        self.bunching_sums = np.array(self.bunching_sums)
        return np.array(E), np.array(T), np.array(B)


def exchange_in_process(engines: list) -> None:
    """The slippage hand-over between consecutive slice blocks held by one
    process (GpuEngines on one GPU, or on several with peer access), in
    device memory: every block's outgoing planes are copied on its own stream,
    block r + 1 waits for that copy and takes it, block 0 takes zeros."""
    import torch

    outs, events = [], []
    for e in engines:
        st = e.stream()
        with torch.cuda.stream(st):
            outs.append(torch.stack(e.plane_views()))
            ev = torch.cuda.Event()
            ev.record(st)
        events.append(ev)
    for r, e in enumerate(engines):
        st = e.stream()
        with torch.cuda.stream(st):
            views = e.plane_views()
            if r == 0:
                for v in views:
                    v.zero_()
            else:
                st.wait_event(events[r - 1])
                outs[r - 1].record_stream(st)  # read on this stream: keep it until then
                for k, v in enumerate(views):
                    v.copy_(outs[r - 1][k], non_blocking=True)
