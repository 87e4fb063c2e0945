"""Host logic of the case builders: block layouts tile their boxes, every
ghost cell of a connected face has exactly one donor, state conversions."""
import numpy as np

from fvm3d import cases


def test_vortex_blocks_tile_box():
    for N in (16, 32, 128):
        boxes = cases.vortex_blocks(N)
        cover = np.zeros((N, N, N), dtype=int)
        for lo, hi in boxes:
            cover[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += 1
        assert (cover == 1).all()
    assert sum(np.prod([h - l for l, h in zip(lo, hi)]) for lo, hi in cases.vortex_blocks(128)) == 128 ** 3


def test_connections_cover_every_ghost_cell_once():
    N = 32
    boxes = cases.vortex_blocks(N)
    conns, bcs = cases.periodic_box_connections((N, N, N), boxes)
    assert not bcs
    for b, (lo, hi) in enumerate(boxes):
        n = [hi[a] - lo[a] for a in range(3)]
        for a in range(3):
            t = [d for d in range(3) if d != a]
            for side in (0, 1):
                cnt = np.zeros((3, n[t[0]], n[t[1]]), dtype=int)
                for (bb, rng, d, drng, dt) in conns:
                    if bb != b:
                        continue
                    lo_a, hi_a = rng[a]
                    if side == 0 and hi_a >= 0:
                        continue
                    if side == 1 and lo_a < n[a]:
                        continue
                    for l in range(lo_a, hi_a + 1):
                        layer = -1 - l if side == 0 else l - n[a]
                        cnt[layer, rng[t[0]][0]:rng[t[0]][1] + 1, rng[t[1]][0]:rng[t[1]][1] + 1] += 1
                        # donor maps to the wrapped global cell
                        g = [0, 0, 0]
                        g[a] = (lo[a] + l) % N
                        dg = boxes[d][0][a] + drng[a][0] + (l - lo_a)
                        assert dg == g[a]
                assert (cnt == 1).all()


def test_prim_cons_roundtrip():
    rng = np.random.default_rng(0)
    p = np.stack([rng.uniform(0.2, 2, 50), rng.normal(size=50), rng.normal(size=50), rng.normal(size=50),
                  rng.uniform(0.1, 5, 50)])
    q = cases.prim_to_cons(*p)
    np.testing.assert_allclose(cases.cons_to_prim(q), p, rtol=1e-13, atol=1e-14)


def test_riemann_seed_ranges():
    c = cases.riemann2d(n=32, seed=5)
    for rho, u, v, w, p in c.meta["quadrants"]:
        assert 0.5 <= rho <= 1.5 and 0.3 <= p <= 1.5 and -0.5 <= u <= 0.5 and -0.5 <= v <= 0.5


def test_integer_factorization_prefers_small_cuts():
    from fvm3d import partition

    assert partition.integer_factorize((128, 128, 128), 8) == (2, 2, 2)
    assert partition.integer_factorize((256, 32, 32), 4) == (4, 1, 1)
    with __import__("pytest").raises(ValueError):
        partition.integer_factorize((4, 4, 4), 8, min_cells=3)


def test_partitioned_case_equals_single_block():
    import oracle as orc
    from fvm3d import abi, partition

    c1 = cases.isentropic_vortex(N=24, layout="single", rk_stages=3, reconstruct=abi.RECON_MUSCL,
                                 limiter=abi.LIMITER_MINMOD, flux_split=abi.FLUX_ROE)
    c6 = partition.partition_case(c1, 6, periodic=(True, True, True))
    assert len(c6.blocks) == 6
    o1 = c1.apply(orc.Oracle(c1.config()))
    o6 = c6.apply(orc.Oracle(c6.config()))
    o1.step(2)
    o6.step(2)
    q6 = cases.assemble(c6, [o6.get_state(b) for b in range(6)])
    assert np.array_equal(q6, o1.get_state(0))
