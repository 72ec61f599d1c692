"""k-point sharding of the SCF over ranks (one process per GPU).

k-points are independent in op_H, Kprec and the eigensolvers; the exchange
steps of an SCF iteration are the sum over k of calc_rhoe (calc_rhoe.jl:51-78),
of the band energies (calc_energies.jl:7-58, 342-375), and the eigenvalues of
every k-point for the Fermi level (occupations.jl:126-192).  Each rank owns
a set of k-points balanced by Ngw_k x Nstates; those three exchanges are
all-reduce sums over the default torch.distributed group (NCCL between
GPUs), and every rank then runs the same mixing and update! steps.
"""


def shard_kpoints(costs, world):
    """k-point lists per rank: longest first onto the least-loaded rank (ties
    to the lower rank), each list sorted."""
    loads = [0.0] * world
    own = [[] for _ in range(world)]
    for ik in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(world), key=lambda q: (loads[q], q))
        own[r].append(ik)
        loads[r] += costs[ik]
    return [sorted(o) for o in own]


class KShards:
    """This rank's k-points and the all-reduce of the SCF exchange steps.
    world = 1 (no process group) keeps every k-point and reduces nothing."""

    def __init__(self, Ngw, Nstates):
        import torch.distributed as dist
        self.dist = dist if dist.is_available() and dist.is_initialized() else None
        self.world = self.dist.get_world_size() if self.dist else 1
        self.rank = self.dist.get_rank() if self.dist else 0
        self.owned = shard_kpoints([float(n) * Nstates for n in Ngw], self.world)
        self.mine = self.owned[self.rank]

    kind = "kpoints"

    def sum_(self, t):
        """In-place sum over ranks of a tensor."""
        if self.dist is not None:
            self.dist.all_reduce(t)
        return t

    def reduce_evals(self, evals):
        """Each rank filled the columns of its own k-points: sum them."""
        if self.world > 1:
            import torch
            t = torch.from_numpy(evals.copy())
            if self.dist.get_backend() == "nccl":
                t = t.cuda()
            evals[:] = self.sum_(t).cpu().numpy()
        return evals


def make_shards(Ngw, Nstates):
    """The SCF's work split over the default process group: by k-points, or
    for a single k-point with more than one rank, inside the Gamma point
    (pwb200.gshard: bands for op_H and the density, plane-wave rows for the
    Rayleigh-Ritz products)."""
    import torch.distributed as dist
    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    if world > 1 and len(Ngw) == 1:
        from .gshard import GammaShards
        return GammaShards()
    return KShards(Ngw, Nstates)
