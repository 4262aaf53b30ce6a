"""project! for basin states kept in host memory, with the copies overlapped with the solves.

A caller whose FlipBasin arrays live in (pinned) host memory pays, per projection, the
upload of u, v, w, types, phi and P and the download of u, v, w, fu, fv, fw and P: about
670 MB at 256^3, more than the solve itself takes to move over PCIe. :class:`HostPipeline`
hides most of it. It keeps three device copies of the basin's arrays and three CUDA
streams: while projection i runs on the compute stream, projection i+1's inputs go up on
one copy stream and projection i-1's outputs come down on the other, so the two copy
directions and the solve all run at once. Events order them: a buffer set is uploaded
only after its previous download has finished, solved only after its upload, and
downloaded only after its solve. Each array moves with one cudaMemcpyAsync (torch's
``copy_`` with ``non_blocking``) from and to page-locked host memory.

The solve is libmpp's ``mpp_project`` (through :class:`mpp.Projector`), one call per
projection; nothing here computes.
"""
from __future__ import annotations

IN_NAMES = ("u", "v", "w", "types", "phi", "P")
OUT_NAMES = ("u", "v", "w", "fu", "fv", "fw", "P")


class HostPipeline:
    """Projections of host-resident basin states through one :class:`mpp.Projector`.

    ``run(inputs, outputs, volume0, dt)`` projects ``len(inputs)`` states: ``inputs[i]`` is
    a dict of pinned host tensors named as :data:`IN_NAMES` (the state projection i starts
    from), ``outputs[i]`` a dict of pinned host tensors named as :data:`OUT_NAMES` that
    receives its result. Returns the list of :class:`mpp.Result` (one per projection), after
    every copy has completed.
    """

    def __init__(self, projector, device=None, depth=3):
        import torch

        self.proj = projector
        g = projector.grid
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        faces = [int(g.face_shape(a)[0] * g.face_shape(a)[1] * g.face_shape(a)[2]) for a in range(3)]
        N = g.ncells
        self.depth = depth
        self.sets = []
        for _ in range(depth):
            f = lambda n, dt: torch.empty(n, dtype=dt, device=self.device)
            self.sets.append({"u": f(faces[0], torch.float32), "v": f(faces[1], torch.float32),
                              "w": f(faces[2], torch.float32), "fu": f(faces[0], torch.uint8),
                              "fv": f(faces[1], torch.uint8), "fw": f(faces[2], torch.uint8),
                              "P": f(N, torch.float32), "types": f(N, torch.uint8), "phi": f(N, torch.float32)})
        self.up = torch.cuda.Stream(self.device)
        self.down = torch.cuda.Stream(self.device)

    @staticmethod
    def bytes_per_step(inputs, outputs):
        """Host-to-device and device-to-host bytes of one projection."""
        h2d = sum(t.numel() * t.element_size() for t in (inputs[k] for k in IN_NAMES))
        d2h = sum(t.numel() * t.element_size() for t in (outputs[k] for k in OUT_NAMES))
        return h2d, d2h

    def run(self, inputs, outputs, volume0, dt, recover=0.5, stream=None):
        import torch

        n = len(inputs)
        if len(outputs) != n:
            raise ValueError("one output set per input set")
        for h in list(inputs) + list(outputs):
            for t in h.values():
                if t.is_cuda or not t.is_pinned():
                    raise ValueError("host arrays must be page-locked CPU tensors (pin_memory())")
        compute = stream if stream is not None else torch.cuda.current_stream(self.device)
        # nothing moves before the work already queued on the compute stream (which may
        # still use the buffer sets, and which a caller's timing event may close)
        self.up.wait_stream(compute)
        self.down.wait_stream(compute)
        freed = [None] * self.depth  # per set: its last download done
        ready = [None] * self.depth  # per set: its upload done

        def upload(i):
            k = i % self.depth
            d = self.sets[k]
            with torch.cuda.stream(self.up):
                if freed[k] is not None:
                    self.up.wait_event(freed[k])
                for name in IN_NAMES:
                    d[name].copy_(inputs[i][name], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.up)
                ready[k] = ev

        def download(i):
            k = i % self.depth
            d = self.sets[k]
            solved = torch.cuda.Event()
            solved.record(compute)
            with torch.cuda.stream(self.down):
                self.down.wait_event(solved)
                for name in OUT_NAMES:
                    outputs[i][name].copy_(d[name], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.down)
                freed[k] = ev

        results = []
        if n:
            upload(0)
        for i in range(n):
            if i + 1 < n:
                upload(i + 1)  # rides beside this projection's solve
            k = i % self.depth
            d = self.sets[k]
            compute.wait_event(ready[k])
            # the solve (the call returns once this projection's result is read back)
            results.append(self.proj.project(d["u"], d["v"], d["w"], d["fu"], d["fv"], d["fw"], d["P"], d["types"],
                                             d["phi"], volume0, dt, recover, stream=compute))
            download(i)  # rides beside the next projection's solve
        for ev in freed:
            if ev is not None:
                compute.wait_event(ev)
        return results
