"""Streaming independent particle states from host memory through the GPU.

``HostPipeline`` serves callers whose particle states live in (pinned) host
memory -- an ensemble of scenes, a parameter sweep, states handed over by a
CPU host application -- and that step each state once per submission: copy
the state in, run one substep, copy it back out.  Each of ``depth`` solvers
of the same scene owns its device state and runs on its own CUDA stream, so
the host->device copy of one submission, the substep of another and the
device->host copy of a third proceed at the same time (the two copy engines
and the SMs); a step's copies are never overlapped with its own compute.

The state of a submission is the solver's storage-order particle arrays
(positions (n,3), velocities (n,3), affine matrices (n,3,3) and particle ids
(n,)), the layout ``FlipSolver3D`` keeps between substeps; ``state_tensors``
returns a solver's.  All solvers of a pipeline have the same grid, solids
and settings, so any state stepped by one may be submitted to another.
"""
from __future__ import annotations

from typing import Callable, List, Sequence

import torch


class HostPipeline:
    """``depth`` copies of a scene, each on its own stream.

    ``factory()`` builds one ``FlipSolver3D`` (the same scene every call); its
    particle count fixes the state size of every submission."""

    def __init__(self, factory: Callable[[], object], depth: int = 3):
        if depth < 1:
            raise ValueError("depth must be >= 1")
        self.solvers = [factory() for _ in range(depth)]
        n = {s.n_particles for s in self.solvers}
        if len(n) != 1:
            raise ValueError("the factory must build the same scene every call")
        self.n = n.pop()
        dev = self.solvers[0].device
        self.streams = [torch.cuda.Stream(device=dev) for _ in range(depth)]
        self._k = 0

    @staticmethod
    def state_tensors(solver) -> List[torch.Tensor]:
        """The solver's device state in storage order: pos, vel, C, pid."""
        return [solver._pos, solver._vel, solver._C, solver._pid]

    def state_bytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in self.state_tensors(self.solvers[0]))

    def host_buffers(self) -> List[torch.Tensor]:
        """A pinned host copy of the state layout (for inputs or outputs)."""
        return [torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
                for t in self.state_tensors(self.solvers[0])]

    def submit(self, host_in: Sequence[torch.Tensor], host_out: Sequence[torch.Tensor],
               dt: float, **step_kw) -> torch.cuda.Event:
        """Queue one submission: host_in -> device, one substep, device ->
        host_out (pinned host tensors of the state layout).  Returns an event
        that completes when host_out holds the result.  host_out must not be
        reused before then; host_in may be reused once the call returns only
        if the caller synchronises on the event first."""
        i = self._k % len(self.solvers)
        s, st = self.solvers[i], self.streams[i]
        dev = self.state_tensors(s)
        if len(host_in) != 4 or len(host_out) != 4:
            raise ValueError("a state is (pos, vel, C, pid)")
        for d, h, o in zip(dev, host_in, host_out):
            if h.shape != d.shape or o.shape != d.shape:
                raise ValueError(f"state shape {tuple(h.shape)} != {tuple(d.shape)}")
        with torch.cuda.stream(st):
            for d, h in zip(dev, host_in):
                d.copy_(h, non_blocking=True)
            s.step(dt, **step_kw)
            for d, h in zip(dev, host_out):
                h.copy_(d, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(st)
        self._k += 1
        return ev

    def wait_all(self, stream: torch.cuda.Stream = None) -> None:
        """Make ``stream`` (default: the current stream) wait for every
        submission queued so far."""
        cur = stream or torch.cuda.current_stream(self.solvers[0].device)
        for st in self.streams:
            cur.wait_stream(st)

    def synchronize(self) -> None:
        for st in self.streams:
            st.synchronize()
