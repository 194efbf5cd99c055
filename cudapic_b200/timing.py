"""CUDA-event timing helpers shared by the benchmark, the autotuner and the
microbenchmark.

L2 flush between timed launches: a 256 MB buffer (twice the B200's 126 MB L2)
is READ, so the L2 ends up holding clean lines of an unrelated buffer.
Writing the buffer instead would leave ~126 MB of dirty lines whose
write-back the next (timed) kernel would pay for.
"""
import statistics


class L2Flusher:
    def __init__(self, nbytes=256 << 20):
        import torch
        self.buf = torch.ones(nbytes // 4, dtype=torch.int32, device="cuda")

    def __call__(self):
        self.buf.sum()


def time_launch(fn, stream, reps, flush=None, pre=None):
    """Median time (s) of `fn` over `reps` launches, CUDA events on `stream`."""
    import torch
    ts = []
    for _ in range(reps):
        if flush is not None:
            flush()
        if pre is not None:
            pre()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1) * 1e-3)
    return statistics.median(ts)
