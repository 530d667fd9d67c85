"""CPU estimate of the subset-test work for other tile shapes (test and
planning infrastructure; nothing on the product path imports it).

On a seeded table it splits the largest partitions into tiles the way the
GPU partitioner's tile phase does (pivot: the unused bit maximising members
holding it x (1 - its table frequency)^12, zeros side first), routes a
seeded query set to each partition by its mask, and counts candidate
(query, tile) pairs: queries holding a tile's 8 rarest AND-mask bits.  It
compares
  * 32-filter tiles, one per warp (the current kernel);
  * the union of two half-tile selectors (one more pivot split per tile);
  * 16- and 8-filter tiles packed 2 or 4 per warp, where a warp's trips are
    set by the largest candidate count among its tiles.

usage: python -m oracle.tile_shape_estimate [filters] [queries] [partitions]
"""
import sys

import numpy as np

from oracle import oracle
from tagmatch_b200 import workload


def main(n=1_000_000, nq=20_000, n_parts=6, max_p=65536):
    f, ko, k = workload.generate_filters(n, 2)
    q = workload.generate_queries(nq, f, 2)
    parts = sorted(oracle.partition(f, max_p), key=len, reverse=True)
    fb = np.unpackbits(f.view(np.uint8), axis=1, bitorder="little").astype(bool)  # [n, 192]
    qb = np.unpackbits(q.view(np.uint8), axis=1, bitorder="little").astype(bool)
    rf = fb.sum(0)
    weight = (1.0 - rf / n) ** 12
    rarest_first = np.argsort(rf, kind="stable")

    def pivot(idx, used):
        fr = fb[idx].sum(0)
        ok = (fr > 0) & (fr < len(idx)) & ~used
        return int(np.argmax(np.where(ok, fr * weight, -1.0).astype(np.float32))) if ok.any() else -1

    def tiles(idx, used, limit):
        if len(idx) <= limit:
            return [idx]
        b = pivot(idx, used)
        if b < 0:
            return [idx[i:i + limit] for i in range(0, len(idx), limit)]
        u = used.copy()
        u[b] = True
        return tiles(idx[~fb[idx, b]], u, limit) + tiles(idx[fb[idx, b]], u, limit)

    def selector(idx):
        am = fb[idx].all(0)
        return np.array([b for b in rarest_first if am[b]][:8], dtype=int)

    def candidates(idx, routed):
        s = selector(idx)
        return qb[routed][:, s].all(1) if len(s) else np.ones(len(routed), bool)

    routed_of = []
    for p in range(min(n_parts, len(parts))):
        idx = np.array(parts[p], dtype=np.int64)
        pm = fb[idx].all(0)
        routed_of.append((idx, np.nonzero(qb[:, pm].all(1))[0] if pm.any() else np.arange(nq)))
    # 32-filter tiles against the union of two half selectors
    whole = halves = useful = 0
    for idx, routed in routed_of:
        for t in tiles(idx, np.zeros(192, bool), 32):
            c = candidates(t, routed)
            whole += int(c.sum())
            b = pivot(t, np.zeros(192, bool)) if len(t) > 1 else -1
            halves += int((candidates(t[~fb[t, b]], routed) | candidates(t[fb[t, b]], routed)).sum()) if b >= 0 else int(c.sum())
            qs = routed[c]
            if len(qs):
                useful += int((~(fb[t][None, :, :] & ~qb[qs][:, None, :]).any(2)).any(1).sum())
    print(f"32-filter tiles: {whole} candidates, {useful / max(whole, 1):.3f} of them match a member; "
          f"union of half selectors: {halves / max(whole, 1):.3f} of the candidates")
    # smaller tiles packed several per warp
    for limit, per_warp in ((32, 1), (16, 2), (8, 4)):
        cand = trips = 0
        for idx, routed in routed_of:
            cs = [int(candidates(t, routed).sum()) for t in tiles(idx, np.zeros(192, bool), limit)]
            cand += sum(cs)
            trips += sum(max(cs[i:i + per_warp]) for i in range(0, len(cs), per_warp))
        print(f"{limit}-filter tiles x{per_warp} per warp: {cand} candidates, {trips} warp trip units")


if __name__ == "__main__":
    main(*(int(a) for a in sys.argv[1:4]))
