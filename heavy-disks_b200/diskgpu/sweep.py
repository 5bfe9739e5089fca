"""Parameter sweeps over many independent disks: the parameter law, sharding across
ranks, and the result gather.

The path shards over independent disks: every rank advances its own subset and the only
collective is the final gather of a few numbers per disk (gamma, Omega_p, saturated
|C2|/|C0|).  The draw uses a counter-based generator (splitmix64) so any disk's
parameters follow from (seed, index) alone, whatever the rank layout.
"""
from __future__ import annotations

import math
from dataclasses import asdict, dataclass

MASK64 = (1 << 64) - 1
GRIDS = (128, 256, 384, 512)


def splitmix64(x: int) -> int:
    """One output of the splitmix64 sequence at counter x (Steele, Lea, Flood 2014)."""
    z = (x + 0x9E3779B97F4A7C15) & MASK64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return z ^ (z >> 31)


def uniform(seed: int, index: int, stream: int) -> float:
    """U[0, 1) for (seed, disk index, parameter stream)."""
    return (splitmix64((seed * 0x100000001B3) ^ (index << 8) ^ stream) >> 11) * (1.0 / (1 << 53))


@dataclass
class SweepPoint:
    index: int
    N: int                # grid N x N (log R x phi)
    Qmin: float           # target minimum Toomre Q over the disk body
    mass_ratio: float     # M_d / M_*
    soft_over_r: float    # softening / r  (eps = (s/r)^2)
    gamma: float          # EOS index
    phase0: float         # m=2 seed phase
    amp: float = 1e-3

    def as_dict(self):
        return asdict(self)


def draw(n: int, seed: int = 12345, grids=GRIDS) -> list[SweepPoint]:
    """The sweep law: grid uniform over `grids`, Q_min ~ U[1,2], M_d/M_* ~ U[0.2,1],
    softening/r ~ U[0.05,0.2], Gamma ~ U[1.5,2], seed phase ~ U[0, pi)."""
    pts = []
    for k in range(n):
        u = [uniform(seed, k, s) for s in range(6)]
        pts.append(SweepPoint(index=k, N=grids[min(int(u[0] * len(grids)), len(grids) - 1)],
                              Qmin=1.0 + u[1], mass_ratio=0.2 + 0.8 * u[2], soft_over_r=0.05 + 0.15 * u[3],
                              gamma=1.5 + 0.5 * u[4], phase0=math.pi * u[5]))
    return pts


def cost(pt: SweepPoint, tlim: float = 1.0) -> float:
    """Relative work of a disk: zones x steps, steps ~ N (CFL) -> N^3."""
    return float(pt.N) ** 3 * tlim


def shard(points, world: int, rank: int, tlim: float = 1.0):
    """Longest-processing-time assignment of disks to ranks (deterministic): every rank
    gets a disjoint subset, the union is everything, and the loads are balanced."""
    order = sorted(points, key=lambda p: (-cost(p, tlim), p.index))
    load = [0.0] * world
    mine = []
    for p in order:
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += cost(p, tlim)
        if r == rank:
            mine.append(p)
    return sorted(mine, key=lambda p: p.index)


def gather(local_results, group=None):
    """All-gather per-disk result dicts (small) from every rank, merged by disk index."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return sorted(local_results, key=lambda r: r["index"])
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, local_results, group=group)
    merged = [r for part in parts for r in part]
    return sorted(merged, key=lambda r: r["index"])


def run_point(pt: SweepPoint, tlim: float, precision: str = "mixed", device: int = -1, dtout: float = 0.25,
              fit_window=(None, None)):
    """Advance one sweep disk on the GPU and fit gamma, Omega_p and the saturated ratio."""
    from . import Disk, params_physical
    from .analysis import fit_growth, saturation_ratio

    p, qach = params_physical(pt.Qmin, pt.mass_ratio, pt.soft_over_r, pt.gamma)
    with Disk(pt.N, pt.N, params=p, amp=pt.amp, phase0=pt.phase0, precision=precision, device=device) as d:
        d.init_standard()
        rec, t, steps = d.advance(tlim, dtout=dtout)
    lo, hi = fit_window
    try:
        g, w, _ = fit_growth(rec[:, 0], rec[:, 2], rec[:, 3], tmin=lo, tmax=hi)
    except ValueError:
        g, w = float("nan"), float("nan")
    return {"index": pt.index, "gamma": g, "omega_p": w, "sat_ratio": saturation_ratio(rec[:, 1], rec[:, 2]),
            "Qmin_achieved": qach, "steps": int(steps), "t": t}


def point_params(pt: SweepPoint, precision: str = "mixed", device: int = -1):
    """The dg_params of a sweep disk: the physics dg_params_physical maps (Q_min,
    M_d/M_*, softening/r, Gamma) to, on the point's grid, with its seed."""
    from . import FP64, MIXED, params_physical

    p, _ = params_physical(pt.Qmin, pt.mass_ratio, pt.soft_over_r, pt.gamma)
    p.Nu = p.Nphi = pt.N
    p.amp, p.phase0, p.device = pt.amp, pt.phase0, device
    p.precision = {"fp64": FP64, "mixed": MIXED}[precision] if isinstance(precision, str) else precision
    return p


def write_sweep_file(path, points, precision: str = "mixed", device: int = -1):
    """Describe a sweep outside Python: the plain-text parameter file (dg_params_write),
    one disk per line with every dg_params field, readable by dg_params_read."""
    from . import write_params

    write_params(path, [point_params(pt, precision, device) for pt in points])


def read_sweep_file(path):
    """The disks of a parameter file (dg_params_read), ready for Batch or Disk(params=...)."""
    from . import read_params

    return read_params(path)
