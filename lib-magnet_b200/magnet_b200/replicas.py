"""Replica placement across GPUs: independent layouts (the batched form) and served requests (the served form)
need no data-path collective, so a job of N ranks splits the work, each rank runs its share on its own GPU, and
the results are gathered at the end. One fitted layout stays resident per GPU for the served form.

* ``place``: a deterministic greedy placement of items of known device bytes onto ranks by free HBM: items in
  decreasing size, each to the rank with the most free bytes left (lowest rank on ties), so every rank computes
  the same placement from the same inputs without exchanging it;
* ``free_bytes``: every rank's free device memory, gathered with one collective (all ranks call it);
* ``gather_results``: the ranks' (item index, result) pairs merged on every rank, in item order.
"""


def place(item_bytes, free_bytes):
    """rank of every item (list of ints): decreasing size first, each to the rank with the most free bytes left;
    raises ValueError when an item fits no rank"""
    item_bytes = [int(b) for b in item_bytes]
    left = [int(f) for f in free_bytes]
    if not left:
        raise ValueError("no ranks to place on")
    owner = [0] * len(item_bytes)
    for i in sorted(range(len(item_bytes)), key=lambda j: (-item_bytes[j], j)):
        r = max(range(len(left)), key=lambda k: (left[k], -k))
        if item_bytes[i] > left[r]:
            raise ValueError("item %d (%d bytes) fits no rank (largest free: %d)" % (i, item_bytes[i], left[r]))
        left[r] -= item_bytes[i]
        owner[i] = r
    return owner


def share(owner, rank):
    """the indices of the items placed on `rank`, in item order"""
    return [i for i, r in enumerate(owner) if r == rank]


def free_bytes(dist=None, device=None, budget_fraction=1.0):
    """every rank's free device bytes (times budget_fraction), the same list on every rank"""
    import torch
    free = int(torch.cuda.mem_get_info(device)[0] * budget_fraction) if torch.cuda.is_available() else 0
    if dist is None:
        return [free]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, free)
    return out


def gather_results(pairs, dist=None):
    """[(index, result), ...] of this rank -> the results of all ranks, ordered by index, on every rank"""
    if dist is None:
        return [r for _, r in sorted(pairs, key=lambda p: p[0])]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, list(pairs))
    merged = [p for part in out for p in part]
    idx = [i for i, _ in merged]
    if len(set(idx)) != len(idx):
        raise RuntimeError("an item was run on two ranks")
    return [r for _, r in sorted(merged, key=lambda p: p[0])]


def layout_bytes(n, nnz, dim=2):
    """device bytes of one t-SNE layout of n points and nnz affinities (positions, update, gains, the CSR) plus
    its share of the FFT grid buffers, for placement"""
    return int(n * dim * 4 * 4 + nnz * 8 + (n + 1) * 4 + 64 * n + (1 << 22))


__all__ = ["place", "share", "free_bytes", "gather_results", "layout_bytes"]
