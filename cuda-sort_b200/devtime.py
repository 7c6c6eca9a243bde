"""Device timing shared by the tuner and the side-by-side baselines.

One measurement = one pass: an L2-evicting write (a buffer twice the 126 MB
L2), then `launches` called back to back between two CUDA events on the
current stream; the per-launch time is the pass time over the number of
launches.  Each launch is expected to work on its own buffer set, so that no
launch reads what the previous one left in L2.  Batching many launches per
event pair keeps the event clock's granularity (about 2 us on a B200) to a
small fraction of the measured time, which a single launch between two events
does not.
"""
import statistics

import torch

L2_BYTES = 126 * 1024 * 1024


class Flusher:
    def __init__(self, device=None):
        self.buf = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device=device or "cuda")
        self.k = 0

    def __call__(self):
        self.k = (self.k + 1) & 0xFF
        self.buf.fill_(self.k)


def batched_us(launches, flush, passes=5, before_pass=None):
    """Median per-launch time in microseconds over `passes` passes, with the
    relative spread (max - min) / median of the passes.  `launches` is a list
    of callables; a callable returning a non-zero status aborts the
    measurement (returns (None, None)).  `before_pass` (optional) runs before
    the flush of each pass, e.g. to restore in-place inputs."""
    st = torch.cuda.current_stream()
    # one untimed launch first: module loading and per-kernel attribute setup
    # happen on a kernel's first use and must not land in a timed pass
    if before_pass is not None:
        before_pass()
    if launches and launches[0]() not in (0, None):
        torch.cuda.synchronize()
        return None, None
    torch.cuda.synchronize()
    times = []
    for _ in range(passes):
        if before_pass is not None:
            before_pass()
        flush()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for fn in launches:
            rc = fn()
            if rc not in (0, None):
                torch.cuda.synchronize()
                return None, None
        e1.record(st)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) * 1e3 / len(launches))
    med = statistics.median(times)
    return med, (max(times) - min(times)) / med if med > 0 else 0.0


def sets_for(batch_bytes, minimum=20):
    """Buffer sets so that a full rotation moves at least twice the L2."""
    return max(minimum, -(-2 * L2_BYTES // max(1, batch_bytes)) + 1)
