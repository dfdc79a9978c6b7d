"""Multi-GPU sharding of the triplet search: one process per GPU, each holding a full
replica of the dataset, each scanning a contiguous range of first indices i, then ONE
exchange step that keeps the lowest (score, triplet index) over all ranks.

The reference runs on one device and has no multi-device path; the partition follows the
work model of its search loops (the triplets with first index i number C(M-1-i, 2),
GPU/v4.cpp:286-290 and CPU/v4_popc_avx512.cpp:287-300 iterate i < j < k), and the
exchange keeps its tie rule (a strict `<` over the flat index gives the lowest-index
triplet, GPU/v2.cpp:558-565).

The exchange is two MIN all-reduces of one int64 each, so it is exact for any backend
that supports MIN on int64 (NCCL on the GPU, gloo on the CPU):
  1. the minimum of the float32 score bit patterns (positive floats order like their bits);
  2. the minimum packed index (i<<42 | j<<21 | k) among the ranks that hold that score.
"""
import struct

NO_SCORE_BITS = 0x7F800000  # +inf: a rank whose shard holds no triplet
NO_INDEX = (1 << 63) - 1


def triplets_of_first(m, i):
    """Triplets (i, j, k), i < j < k < m, with first index i."""
    return ((m - 1 - i) * (m - 2 - i)) // 2 if i <= m - 3 else 0


def triplets_in(m, lo, hi):
    return sum(triplets_of_first(m, i) for i in range(lo, hi))


def shard_bounds(m, parts):
    """Cut first indices [0, m) into `parts` contiguous ranges of near-equal triplet count
    (each range is off the even split by less than the work of one first index)."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    work = [triplets_of_first(m, i) for i in range(m)]
    total = sum(work)
    bounds, acc, lo = [], 0, 0
    for i in range(m):
        acc += work[i]
        if len(bounds) < parts - 1 and acc * parts >= total * (len(bounds) + 1):
            bounds.append((lo, i + 1))
            lo = i + 1
    bounds.append((lo, m))
    while len(bounds) < parts:
        bounds.append((m, m))
    return bounds


def score_bits(score):
    return struct.unpack("<I", struct.pack("<f", score))[0]


def bits_score(bits):
    return struct.unpack("<f", struct.pack("<I", bits))[0]


def pack_index(i, j, k):
    return (int(i) << 42) | (int(j) << 21) | int(k)


def unpack_index(key):
    return (key >> 42) & 0x1FFFFF, (key >> 21) & 0x1FFFFF, key & 0x1FFFFF


def better(a, b):
    """Strict order of (score, (i, j, k)) candidates: lower score, then lower index."""
    sa, sb = score_bits(a[0]), score_bits(b[0])
    if sa != sb:
        return sa < sb
    return pack_index(*a[1]) < pack_index(*b[1])


def exchange_best(score, ijk, group=None, device=None):
    """Lowest (score, triplet) over all ranks of `group`.  `score` None (or ijk None)
    means this rank has no triplet.  Returns (score, (i, j, k)), or (None, None) when no
    rank has one.  `device`: where the collective's tensors live ("cuda:N" for NCCL;
    default: the CPU for gloo, the current CUDA device for NCCL)."""
    import torch
    import torch.distributed as dist
    if device is None:
        device = "cpu"
        if dist.get_backend(group) == "nccl":
            device = f"cuda:{torch.cuda.current_device()}"
    have = score is not None and ijk is not None
    sb = score_bits(score) if have else NO_SCORE_BITS
    t = torch.tensor([sb], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    best_bits = int(t.item())
    key = pack_index(*ijk) if have and sb == best_bits else NO_INDEX
    t = torch.tensor([key], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    key = int(t.item())
    if key == NO_INDEX:
        return None, None
    return bits_score(best_bits), unpack_index(key)


def scan_sharded(ctx, dataset, rank, world, group=None, parts=None, **opts):
    """Search this rank's share of `dataset` (resident in `ctx` on this rank's GPU) and
    exchange: every rank returns the global best (score, (i, j, k)).  `parts` (default
    `world`) cuts the first indices finer; rank r scans parts r, r+world, ..."""
    m = ctx.info(dataset)["n_snps"]
    parts = parts or world
    bounds = shard_bounds(m, parts)
    best = None
    for p in range(rank, parts, world):
        lo, hi = bounds[p]
        if triplets_in(m, lo, hi) == 0:
            continue
        b = ctx.scan(dataset, snp_begin=lo, snp_end=hi, **opts)
        cand = (b.score, b.ijk)
        if best is None or better(cand, best):
            best = cand
    return exchange_best(best[0] if best else None, best[1] if best else None, group)
