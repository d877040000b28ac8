"""Multi-GPU plumbing for the halo-finding path: tiles are sharded across ranks, nothing is
exchanged on the data path, and the catalog is gathered once at the end.

* Tile assignment is round-robin, worker w (1-based) taking the tiles i with
  mod1(i, n_workers) == w (MultiResolution.jl:1303-1311).  One rank per GPU stands in for
  the reference's one Julia task per GPU; the tiles of a rank run back to back.
* Within one tile the peaks are independent (the mask writes of the collapse are
  idempotent, ext/CUDAExt.jl:1879), so a tile's peak list may also be split into
  contiguous ranges across ranks that hold the same fields (`peak_range`).
* The catalog gather mirrors the MPI path (MPIExt.jl:1041-1063): an all-gather of the
  per-rank record counts, then a variable-size gather of the Float32 records to rank 0.
  torch.distributed provides both (NCCL on GPUs, gloo on CPU).
* HaloRecord packing follows MultiResolution.jl:1164-1219: peaks with RTHL <= 0 are
  skipped; RTHL is converted to Mpc/h with alatt; Sbar is scaled by the growth factor D
  and Sbar2 by -3/7 Om(a)^(-1/143) D^2 when ilpt >= 2.

No collective runs inside a step; `max_over_ranks` is the end-of-run timing reduction.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np
import torch

HALO_FIELDS = ("x", "y", "z", "vx", "vy", "vz", "RTHL", "vx2", "vy2", "vz2", "overdensity")


def tiles_for_rank(ntiles: int, rank: int, world: int) -> list:
    """0-based tile indices rank `rank` of `world` processes (MultiResolution.jl:1305)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return [t for t in range(ntiles) if t % world == rank]


def peak_range(npeaks: int, rank: int, world: int) -> tuple:
    """Contiguous [lo, hi) share of a tile's peak list for one rank; the first
    npeaks % world ranks take one peak more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(npeaks, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def halo_records(x, y, z, results: dict, alatt: float, *, D: float = 1.0,
                 coef2: float = 0.0, ilpt: int = 2) -> np.ndarray:
    """(nhalo, 11) Float32 HaloRecord rows of the collapsed peaks (RTHL > 0), in peak
    order (MultiResolution.jl:1164-1219; field order IO/Catalog.jl:4-10).

    x, y, z: physical peak positions (PeakCandidate.x/y/z); results: the host or device
    result arrays of one collapse call (RTHL, Fbarx, Sbar and Sbar2 rows of 3 per peak);
    D: linear growth factor at the peak's redshift; coef2: the 2LPT coefficient
    -3/7 Om(a)^(-1/143) D^2 (used when ilpt >= 2)."""
    as_np = lambda t: t.detach().cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)
    rthl = as_np(results["RTHL"]).astype(np.float32)
    npk = len(np.asarray(x))
    rthl = rthl[:npk]
    keep = rthl > 0
    sbar = as_np(results["Sbar"]).reshape(-1, 3)[:npk][keep].astype(np.float32)
    sbar2 = as_np(results["Sbar2"]).reshape(-1, 3)[:npk][keep].astype(np.float32)
    out = np.zeros((int(keep.sum()), len(HALO_FIELDS)), np.float32)
    out[:, 0] = np.asarray(x, np.float64)[keep].astype(np.float32)
    out[:, 1] = np.asarray(y, np.float64)[keep].astype(np.float32)
    out[:, 2] = np.asarray(z, np.float64)[keep].astype(np.float32)
    out[:, 3:6] = sbar * np.float32(D)
    out[:, 6] = (rthl[keep].astype(np.float64) * alatt).astype(np.float32)
    if ilpt >= 2:
        out[:, 7:10] = sbar2 * np.float32(coef2)
    out[:, 10] = as_np(results["Fbarx"]).astype(np.float32)[:npk][keep]
    return out


def gather_records(local: np.ndarray, group=None, dst: int = 0) -> Optional[np.ndarray]:
    """Gather every rank's (n_r, nfields) Float32 records to rank `dst` in rank order
    (MPIExt.jl:1041-1063: Allgather of the counts, then Gatherv).  Returns the
    concatenation on `dst` and None elsewhere.  With no process group (one process) the
    local records are returned unchanged."""
    import torch.distributed as dist
    local = np.ascontiguousarray(local, dtype=np.float32)
    if not (dist.is_available() and dist.is_initialized()):
        return local
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    backend = dist.get_backend(group)
    dev = (torch.device("cuda", torch.cuda.current_device()) if backend == "nccl"
           else torch.device("cpu"))
    nf = local.shape[1] if local.ndim == 2 else 1
    cnt = torch.tensor([local.size], dtype=torch.int64, device=dev)
    counts = [torch.zeros_like(cnt) for _ in range(world)]
    dist.all_gather(counts, cnt, group=group)
    counts = [int(c.item()) for c in counts]
    cap = max(max(counts), 1)
    buf = torch.zeros(cap, dtype=torch.float32, device=dev)
    if local.size:
        buf[:local.size] = torch.from_numpy(local.reshape(-1)).to(dev)
    # Padded all-gather: every rank takes the same collective steps; only dst keeps them.
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    if rank != dst:
        return None
    flat = np.concatenate([p[:c].cpu().numpy() for p, c in zip(parts, counts)])
    return flat.reshape(-1, nf)


def max_over_ranks(value: float, group=None) -> float:
    """Largest `value` over all ranks (per-step device time is reported as the max)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    backend = dist.get_backend(group)
    dev = (torch.device("cuda", torch.cuda.current_device()) if backend == "nccl"
           else torch.device("cpu"))
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sum_over_ranks(value: float, group=None) -> float:
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    backend = dist.get_backend(group)
    dev = (torch.device("cuda", torch.cuda.current_device()) if backend == "nccl"
           else torch.device("cpu"))
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())


def aggregate_e2e(e2e: dict, group=None) -> dict:
    """The whole job's end-to-end line from every rank's own (value = units per second over
    `steps` steps of `ms_per_step`, bytes copied per step): the units of all ranks over the
    slowest rank's time, the copied bytes summed over ranks.  Every rank calls it (it holds
    collectives); without an initialised process group it returns the line unchanged."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return dict(e2e)
    out = dict(e2e)
    steps = e2e["steps"]
    units = e2e["value"] * e2e["ms_per_step"] * steps / 1e3
    ms = max_over_ranks(e2e["ms_per_step"], group)
    out["ms_per_step"] = ms
    out["value"] = sum_over_ranks(units, group) / (ms * steps / 1e3)
    out["h2d_bytes_per_step"] = int(sum_over_ranks(e2e["h2d_bytes_per_step"], group))
    out["d2h_bytes_per_step"] = int(sum_over_ranks(e2e["d2h_bytes_per_step"], group))
    out["ranks"] = dist.get_world_size(group)
    return out


def merge_catalog(parts: Sequence[np.ndarray]) -> np.ndarray:
    """Rank-order concatenation of per-rank records (halo order across workers carries no
    meaning, MultiResolution.jl:1338)."""
    parts = [np.asarray(p, np.float32).reshape(-1, len(HALO_FIELDS)) for p in parts]
    return np.concatenate(parts) if parts else np.zeros((0, len(HALO_FIELDS)), np.float32)
