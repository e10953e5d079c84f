"""Multi-GPU form of the search: independent replicas over disjoint K ranges.

The per-K search has no exchange step (every K is searched independently), so
N GPUs run N replicas, each on its own K range, with no collective on the
data path.  The only cross-rank steps are host-side: the partial result
hashes are combined (the reference's result hash is an additive sum reduced
by 2e9, src/common/AP26.cpp:557-561) and device times are reduced with max.
"""
MAXINTV = 2_000_000_000


def rank_range(kmin, k_per_rank, rank):
    """[first, last] K of rank `rank` (weak scaling: k_per_rank each)."""
    a = kmin + k_per_rank * rank
    return a, a + k_per_rank - 1


def split_range(kmin, kmax, world, rank):
    """[first, last] K of rank `rank` when one workunit [kmin, kmax] is split
    over `world` ranks (strong scaling); empty ranges come back as (a, a-1)."""
    n = kmax - kmin + 1
    a = kmin + n * rank // world
    b = kmin + n * (rank + 1) // world - 1
    return a, b


def merge_hash(partials):
    """Combine per-rank result hashes exactly as one process accumulating all
    reports would: every partial is in [0, 2e9], the sum is reduced by 2e9
    whenever it passes it."""
    h = 0
    for p in partials:
        h += int(p)
        if h > MAXINTV:
            h -= MAXINTV
    return h
