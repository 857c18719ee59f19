"""A time loop over particle state kept in pinned host memory, with the
host<->device copies overlapped with the steps (no counterpart in the
reference, whose state stays on the device).

Every step copies its inputs in (fluid SoA and labels, wall SoA) and the moved
fluid state and labels out, so that each step's inputs are the previous
step's outputs.  The copies run on a copy stream and the step waits only for
what it reads (lsmps_ctx_set_step_events):

* the fluid positions go to one of two device position buffers, alternating
  per step, so the next step's positions travel while the current step's
  neighbour rebuild and labels still read its own buffer;
* the wall geometry follows (the mixed step first reads it after its fluid
  moment sums), then the velocities, pressure, labels and wall velocities
  (read from the provision stage on), once the previous step is done with
  those buffers;
* the new positions, velocities and pressure go back as soon as the pressure
  correction is done (while the rebuild and the labels run), the labels
  when the step is done.

The neighbour tables, cell lists and moment/PPE workspaces stay on the device
and are shared by both position buffers (both hold the same positions when a
step starts).
"""

from __future__ import annotations

FIRST = ("x", "y", "z")
GEOMETRY = ("x", "y", "z", "normal_x", "normal_y", "normal_z")
SECOND_FLUID = ("vx", "vy", "vz", "pressure", "surface_type")
SECOND_WALLS = ("vx", "vy", "vz")
OUT_EARLY = ("x", "y", "z", "vx", "vy", "vz", "pressure")


class HostResidentLoop:
    """Steps `buffers` (api.StepBuffers) with the particle state in pinned
    host memory (`host_fluid`, `host_walls`: the buffers' current contents
    at construction).  step() queues one step and its copies; sync() waits
    for everything queued and leaves the host arrays holding the last
    step's outputs; close() clears the context's step events.  Queue it on
    the context's own stream (the current torch stream at construction) and
    put the context in asynchronous mode (Context.set_synchronous(False)):
    a synchronous context waits at the end of every step, which still gives
    the same results but leaves less to overlap."""

    def __init__(self, ctx, buffers, params):
        import torch

        self.torch = torch
        self.ctx, self.dev, self.params = ctx, buffers, params
        self.stream = torch.cuda.current_stream()
        self.copy = torch.cuda.Stream(self.stream.device)
        fl, wl = buffers.fluid, buffers.walls
        self.host_fluid = {k: fl[k].detach().to("cpu").pin_memory() for k in FIRST + SECOND_FLUID}
        self.host_walls = {k: wl[k].detach().to("cpu").pin_memory() for k in GEOMETRY + SECOND_WALLS}
        # the second device position buffer and the step state that uses it
        self.pos = [{k: fl[k] for k in FIRST}, {k: torch.empty_like(fl[k]) for k in FIRST}]
        self.states = [buffers.step_state(params), buffers.step_state(params)]
        b = self.states[1].fluid
        b.x, b.y, b.z = (self.pos[1][k].data_ptr() for k in FIRST)
        self.h2d_bytes = sum(t.numel() * t.element_size() for t in list(self.host_fluid.values()) +
                             list(self.host_walls.values()))
        self.d2h_bytes = sum(self.host_fluid[k].numel() * self.host_fluid[k].element_size()
                             for k in OUT_EARLY + ("surface_type",))
        self.ev_pos, self.ev_wall, self.ev_in, self.ev_out, self.ev_end = (torch.cuda.Event() for _ in range(5))
        for ev in (self.ev_pos, self.ev_wall, self.ev_in):
            ev.record(self.copy)  # creates the events before their handles are passed on
        for ev in (self.ev_out, self.ev_end):
            ev.record(self.stream)
        ctx.set_step_events(self.ev_wall.cuda_event, self.ev_in.cuda_event, self.ev_out.cuda_event)
        self.count = 0
        self.labels_pending = False

    def step(self) -> None:
        torch = self.torch
        cur = self.count & 1
        fl, wl = self.dev.fluid, self.dev.walls
        with torch.cuda.stream(self.copy):
            # this step's positions (the previous step's outputs: queued
            # earlier on this stream) into this step's buffer, while the
            # previous step may still run on the other one
            for k in FIRST:
                self.pos[cur][k].copy_(self.host_fluid[k], non_blocking=True)
            self.ev_pos.record(self.copy)
            # the rest once the previous step is done with those buffers
            self.copy.wait_event(self.ev_end)
            if self.labels_pending:
                self.host_fluid["surface_type"].copy_(fl["surface_type"], non_blocking=True)
            for k in GEOMETRY:
                wl[k].copy_(self.host_walls[k], non_blocking=True)
            self.ev_wall.record(self.copy)
            for k in SECOND_FLUID:
                fl[k].copy_(self.host_fluid[k], non_blocking=True)
            for k in SECOND_WALLS:
                wl[k].copy_(self.host_walls[k], non_blocking=True)
            self.ev_in.record(self.copy)
        self.stream.wait_event(self.ev_pos)
        self.ctx.step(self.dev, self.params, self.states[cur])
        self.ev_end.record(self.stream)
        self.copy.wait_event(self.ev_out)
        with torch.cuda.stream(self.copy):
            for k in OUT_EARLY:
                src = self.pos[cur][k] if k in FIRST else fl[k]
                self.host_fluid[k].copy_(src, non_blocking=True)
        self.labels_pending = True
        self.count += 1

    def sync(self) -> None:
        """Queue the last step's labels out and join the copy stream into
        the step stream (then wait with the caller's own synchronisation)."""
        torch = self.torch
        if self.labels_pending:
            with torch.cuda.stream(self.copy):
                self.copy.wait_event(self.ev_end)
                self.host_fluid["surface_type"].copy_(self.dev.fluid["surface_type"], non_blocking=True)
            self.labels_pending = False
        self.stream.wait_stream(self.copy)

    def close(self) -> None:
        self.ctx.set_step_events(None, None, None)
