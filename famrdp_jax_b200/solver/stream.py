"""Time steps whose states arrive from and return to host memory, with the
transfers overlapped with the steps.

A caller that feeds states from the host (a service stepping independent
requests, or a loop that checkpoints every state to host memory) pays a
host-to-device copy before and a device-to-host copy after every step.
``HostStepper`` pipelines them over two device buffer sets and three streams:
while step n runs, the input of step n+1 is copied in and the result of step
n-1 is copied out.  Host buffers must be pinned for the copies to overlap.

    stepper = HostStepper(StepPlan(state, cfg))
    stepper.run(host_inputs, host_outputs, dt)   # lists over steps of lists over blocks
    torch.cuda.current_stream().synchronize()    # host_outputs are complete
"""
from __future__ import annotations

import torch

from famrdp_jax_b200.solver.step import StepPlan


class HostStepper:
    """Pipelined host -> device -> step -> host stepping with one plan."""

    def __init__(self, plan: StepPlan, depth: int = 2):
        if depth < 1:
            raise ValueError("depth must be >= 1")
        self.plan = plan
        dev = plan.device
        self.depth = depth
        self.h2d, self.comp, self.d2h = (torch.cuda.Stream(dev) for _ in range(3))

        def buffers():
            return [[torch.empty(s, dtype=torch.float64, device=dev) for s in plan.shapes] for _ in range(depth)]

        self.din, self.dout = buffers(), buffers()
        ev = lambda: [torch.cuda.Event() for _ in range(depth)]  # noqa: E731
        self.in_ready, self.in_free, self.out_ready, self.out_free = ev(), ev(), ev(), ev()

    def run(self, host_in, host_out, dt: float, graph: bool = True) -> None:
        """Steps host_in[i] (a list of per-block (5, ni, nj, nk) float64 host
        tensors) into host_out[i] for every i, asynchronously on the caller's
        current stream: work starts after what the stream has queued, and the
        stream waits for the last copy out."""
        if len(host_in) != len(host_out):
            raise ValueError("host_in and host_out differ in length")
        dev = self.plan.device
        cur = torch.cuda.current_stream(dev)
        for s in (self.h2d, self.comp, self.d2h):
            s.wait_stream(cur)
        for i, (hin, hout) in enumerate(zip(host_in, host_out)):
            k = i % self.depth
            with torch.cuda.stream(self.h2d):
                self.h2d.wait_event(self.in_free[k])  # the step that last read din[k] is done
                for d, h in zip(self.din[k], hin):
                    d.copy_(h, non_blocking=True)
                self.in_ready[k].record(self.h2d)
            with torch.cuda.stream(self.comp):
                self.comp.wait_event(self.in_ready[k])
                self.comp.wait_event(self.out_free[k])  # dout[k] has been copied out
                self.plan.run(self.din[k], self.dout[k], dt, graph=graph)
                self.in_free[k].record(self.comp)
                self.out_ready[k].record(self.comp)
            with torch.cuda.stream(self.d2h):
                self.d2h.wait_event(self.out_ready[k])
                for h, d in zip(hout, self.dout[k]):
                    h.copy_(d, non_blocking=True)
                self.out_free[k].record(self.d2h)
        cur.wait_stream(self.comp)
        cur.wait_stream(self.d2h)
