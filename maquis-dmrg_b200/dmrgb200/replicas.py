"""Replica aggregation for one-process-per-GPU runs.

The hot path is one GPU per site problem, so N GPUs run N independent replicas
of the same work (no data-path collective).  Timing follows the rule of the
benchmark: every rank measures its own device time, the job time is the
maximum over ranks, and the job throughput is the total work of all ranks over
that time.  The process group (NCCL on GPUs, gloo on CPUs) carries only the
barrier and the max-reduction of the timings."""
from __future__ import annotations


def job_throughput(per_rank_ms, work_per_rank: float, world: int, dist=None, device=None):
    """Return (max ms over ranks, whole-job work per second) for the given
    per-rank times (a float or a list of floats reduced element-wise)."""
    import torch

    vals = per_rank_ms if isinstance(per_rank_ms, (list, tuple)) else [per_rank_ms]
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    if dist is not None and world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = [float(x) for x in t.cpu()]
    rates = [world * work_per_rank / (m * 1e-3) if m > 0 else 0.0 for m in ms]
    if not isinstance(per_rank_ms, (list, tuple)):
        return ms[0], rates[0]
    return ms, rates
