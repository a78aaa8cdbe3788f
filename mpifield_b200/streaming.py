"""Gather and scatter of markers that live in host memory, with the copies overlapped.

A step over N host-resident markers (positions (ndim, N), values (ncomp_v, N) in pinned
host memory) that gathers a device field at the markers into a host result and deposits
the values into a device field cuts the markers into chunks and runs three streams:
host-to-device copies of chunk c + 1, the kernels on chunk c, and the device-to-host copy
of chunk c - 1's result, so that both copy directions of the link and the kernels work at
once. Two device slots hold the chunks in flight; events order the slots' reuse. The
kernels are the public gather and scatter (``mpf_gather`` / ``mpf_scatter``); their
results are the same as one call over all markers (the scatter adds chunk after chunk).
"""

from __future__ import annotations

import torch

from mpifield_b200 import kernels as K


class HostPipeline:
    """Reusable device slots and streams for `step` (chunks of ``chunk`` markers)."""

    def __init__(self, device, ndim: int, gather_components: int, value_components: int,
                 dtype=torch.float64, chunk: int = 1 << 22, slots: int = 2):
        self.device = torch.device(device)
        self.chunk = chunk
        self.slots = [
            {"pos": torch.empty((ndim, chunk), dtype=dtype, device=self.device),
             "val": torch.empty((value_components, chunk), dtype=dtype, device=self.device),
             "res": torch.empty((gather_components, chunk), dtype=dtype, device=self.device),
             "loaded": torch.cuda.Event(), "computed": torch.cuda.Event(), "stored": torch.cuda.Event(),
             "used": False}
            for _ in range(slots)]
        self.h2d = torch.cuda.Stream(self.device)
        self.compute = torch.cuda.Stream(self.device)
        self.d2h = torch.cuda.Stream(self.device)

    def step(self, kind: int, degree: int, host_positions: torch.Tensor, host_values: torch.Tensor,
             field: torch.Tensor, density: torch.Tensor, host_result: torch.Tensor, geometry,
             host_density: torch.Tensor | None = None) -> torch.cuda.Event:
        """host_result = gather(field) at the host markers; density += their deposit; then
        (optionally) host_density = density. Returns the event of the last copy."""
        n = host_positions.shape[1]
        start = torch.cuda.current_stream(self.device)
        for s in (self.h2d, self.compute, self.d2h):
            s.wait_stream(start)
        for k, first in enumerate(range(0, n, self.chunk)):
            m = min(self.chunk, n - first)
            slot = self.slots[k % len(self.slots)]
            pos, val, res = slot["pos"][:, :m], slot["val"][:, :m], slot["res"][:, :m]
            with torch.cuda.stream(self.h2d):
                if slot["used"]:
                    self.h2d.wait_event(slot["computed"])  # the slot's markers were consumed
                for r in range(pos.shape[0]):  # one contiguous copy per row
                    pos[r].copy_(host_positions[r, first:first + m], non_blocking=True)
                for r in range(val.shape[0]):
                    val[r].copy_(host_values[r, first:first + m], non_blocking=True)
                slot["loaded"].record(self.h2d)
            with torch.cuda.stream(self.compute):
                self.compute.wait_event(slot["loaded"])
                if slot["used"]:
                    self.compute.wait_event(slot["stored"])  # the slot's result was copied out
                K.gather(kind, degree, pos, field, res, geometry)
                K.scatter(kind, degree, pos, val, density, geometry)
                slot["computed"].record(self.compute)
            with torch.cuda.stream(self.d2h):
                self.d2h.wait_event(slot["computed"])
                for r in range(res.shape[0]):
                    host_result[r, first:first + m].copy_(res[r], non_blocking=True)
                slot["stored"].record(self.d2h)
            slot["used"] = True
        done = torch.cuda.Event()
        with torch.cuda.stream(self.d2h):
            self.d2h.wait_stream(self.compute)
            if host_density is not None:
                host_density.copy_(density, non_blocking=True)
            done.record(self.d2h)
        start.wait_event(done)
        return done
