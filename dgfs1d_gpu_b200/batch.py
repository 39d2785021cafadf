"""Many independent problems advanced as one CUDA graph per stage.

Problems of different velocity grids (N = 16/24/32), sphere rules, point
counts and species (VHS and VSS) cannot share one persistent kernel without
paying the largest variant's shared memory and registers in every CTA: the
kernels are specialised per N at compile time.  Instead each problem's
stage is enqueued on its own stream, forked from and joined to one capture
stream, and the whole stage is captured once into a CUDA graph; a stage is
then a single graph launch whose branches the GPU schedules concurrently.
"""
import torch


class StageGraph:
    """Capture ``[fn_0, ..., fn_k]`` (callables enqueuing work on the current
    stream) as concurrent branches of one CUDA graph."""

    def __init__(self, fns, device='cuda'):
        self.fns = list(fns)
        self.device = device
        self.streams = [torch.cuda.Stream(device=device) for _ in self.fns]
        self.graph = None

    def run_eager(self):
        """The same branches without a graph (for comparison)."""
        main = torch.cuda.current_stream()
        for fn, st in zip(self.fns, self.streams):
            st.wait_stream(main)
            with torch.cuda.stream(st):
                fn()
        for st in self.streams:
            main.wait_stream(st)

    def capture(self, warmup=1):
        for _ in range(warmup):
            self.run_eager()
        torch.cuda.synchronize()
        cap = torch.cuda.Stream(device=self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(cap):
            with torch.cuda.graph(g, stream=cap):
                for fn, st in zip(self.fns, self.streams):
                    st.wait_stream(cap)
                    with torch.cuda.stream(st):
                        fn()
                for st in self.streams:
                    cap.wait_stream(st)
        self.graph = g
        return g

    def replay(self):
        self.graph.replay()
