"""Split one structured block into p blocks (integer factorisation).

Restates the idea of ClassPartitionMethod's IF method
(src/base/method_partition.f90:576-666): factorise p into three integers
(px, py, pz) (factorize_number_sub), keep the factorisation with the least
block-to-block communication (the cut planes' area, the t_b2b_if cost) and
cut the block into px x py x pz near-equal boxes. On one GPU the pieces feed
the work queue as ordinary blocks; their interfaces become connections.
"""
from __future__ import annotations

from . import abi, cases


def factorizations(p: int):
    """All ordered triples (a, b, c) with a*b*c == p."""
    out = []
    for a in range(1, p + 1):
        if p % a:
            continue
        for b in range(1, p // a + 1):
            if (p // a) % b:
                continue
            out.append((a, b, p // a // b))
    return out


def cut_area(n, f) -> int:
    """Cells on the cut planes: the ghost exchange the split creates."""
    return (f[0] - 1) * n[1] * n[2] + (f[1] - 1) * n[0] * n[2] + (f[2] - 1) * n[0] * n[1]


def integer_factorize(n, p: int, min_cells: int = 3):
    """Best (px, py, pz) for splitting an n[0] x n[1] x n[2] block into p
    pieces: least cut area, every piece at least `min_cells` wide."""
    best = None
    for f in factorizations(p):
        if any(n[a] // f[a] < min_cells for a in range(3)):
            continue
        c = cut_area(n, f)
        if best is None or c < best[0]:
            best = (c, f)
    if best is None:
        raise ValueError(f"cannot split {tuple(n)} into {p} pieces of at least {min_cells} cells")
    return best[1]


def split_boxes(n, f):
    """Near-equal boxes (lo, hi) of the factorisation f, x fastest."""
    def cuts(m, k):
        return [m * i // k for i in range(k + 1)]
    cx, cy, cz = cuts(n[0], f[0]), cuts(n[1], f[1]), cuts(n[2], f[2])
    boxes = []
    for k in range(f[2]):
        for j in range(f[1]):
            for i in range(f[0]):
                boxes.append(((cx[i], cy[j], cz[k]), (cx[i + 1], cy[j + 1], cz[k + 1])))
    return boxes


def partition_case(case: cases.Case, p: int, periodic=(False, False, False)) -> cases.Case:
    """The single-block `case` as p blocks: interfaces connected, outer faces
    periodic where `periodic` says so and transmissive otherwise."""
    if len(case.blocks) != 1:
        raise ValueError("partition_case splits single-block cases")
    (n, dr), q = case.blocks[0], case.states[0]
    f = integer_factorize(n, p)
    boxes = split_boxes(n, f)
    conns, bcs = cases.periodic_box_connections(n, boxes, periodic)
    out = cases.Case(name=f"{case.name}_x{p}", cfg=dict(case.cfg), meta=dict(case.meta))
    out.meta["factorization"] = f
    for lo, hi in boxes:
        out.blocks.append((tuple(hi[a] - lo[a] for a in range(3)), dr))
        out.origins.append(lo)
        out.states.append(q[:, lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]].copy())
    out.conns = conns
    out.bcs = bcs
    return out
