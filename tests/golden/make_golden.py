"""Generates tests/golden/golden_vectors.json.

An independent pure-Python restatement of the integer and BVH parts of
tinypt's path (the reference itself cannot be built here: no Rust
toolchain).  The C++ oracle and the product's host BVH builder are checked
against these vectors, so a transcription slip in either one shows up as a
mismatch against a second, separately written restatement.

Restated: Rng::new / next_u32 / next_f64 and seed_for (src/rng.rs:12-47),
interleave_bits / morton2 and the tile task order (src/render.rs:75-100,
284-299), Bvh::build (src/bvh.rs:51-242) with Triangle::bounds and
Aabb::from_points (src/geometry.rs:70-80, 221-230).

Run: python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
from pathlib import Path

M64 = (1 << 64) - 1


# ---- src/rng.rs -------------------------------------------------------------
class Rng:
    def __init__(self, seed: int):
        self.state = 0x9E3779B97F4A7C15 if seed == 0 else seed & M64

    def next_u32(self) -> int:
        old = self.state
        self.state = (old * 6364136223846793005 + 1442695040888963407) & M64
        xs = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xs >> rot) | (xs << ((32 - rot) & 31))) & 0xFFFFFFFF

    def next_f64(self) -> float:
        hi = self.next_u32() << 21
        lo = self.next_u32() & ((1 << 21) - 1)
        return float(hi | lo) * (1.0 / float(1 << 53))


def seed_for(px: int, py: int, s: int) -> int:
    h = 0xD1B54A32D192ED03
    h ^= (px * 0x9E3779B185EBCA87) & M64
    h ^= (py * 0xC2B2AE3D27D4EB4F) & M64
    h ^= (s * 0x165667B19E3779F9) & M64
    return h ^ (h >> 32)


# ---- src/render.rs ---------------------------------------------------------
def interleave_bits(v: int) -> int:
    x = v & 0x00000000FFFFFFFF
    x = (x | (x << 16)) & 0x0000FFFF0000FFFF
    x = (x | (x << 8)) & 0x00FF00FF00FF00FF
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0F
    x = (x | (x << 2)) & 0x3333333333333333
    x = (x | (x << 1)) & 0x5555555555555555
    return x


def tile_order(w, h, tile, morton):
    tasks = []
    for y in range(0, h, tile):
        for x in range(0, w, tile):
            tasks.append((x, y, min(x + tile, w), min(y + tile, h)))
    if morton:
        tx_n, ty_n = (w + tile - 1) // tile, (h + tile - 1) // tile

        def key(t):
            tx = min(t[0] // tile, max(tx_n - 1, 0))
            ty = min(t[1] // tile, max(ty_n - 1, 0))
            return interleave_bits(tx) | (interleave_bits(ty) << 1)

        tasks.sort(key=key)  # stable, like slice::sort_by_key
    return tasks


# ---- src/bvh.rs --------------------------------------------------------------
INF = float("inf")


def tri_bounds(a, b, c):
    lo = [min(min(min(INF, a[k]), b[k]), c[k]) - 1e-9 for k in range(3)]
    hi = [max(max(max(-INF, a[k]), b[k]), c[k]) + 1e-9 for k in range(3)]
    return lo, hi


def bvh_build(pos, tris):
    n_t = len(tris)
    bounds = [tri_bounds(pos[t[0]], pos[t[1]], pos[t[2]]) for t in tris]
    cents = [[(lo[k] + hi[k]) * 0.5 for k in range(3)] for lo, hi in bounds]
    idx = list(range(n_t))
    nodes = []

    def union(bb, lo, hi):
        return [min(bb[0][k], lo[k]) for k in range(3)], [max(bb[1][k], hi[k]) for k in range(3)]

    def empty():
        return [INF] * 3, [-INF] * 3

    def bin_of(cv, minc, inv_extent):
        f = (cv - minc) * inv_extent * 8.0
        b = int(f) if f > 0 else 0
        return min(b, 7)

    def build(start, end):
        n = end - start
        bb, cb = empty(), empty()
        for i in idx[start:end]:
            bb = union(bb, *bounds[i])
            cb = union(cb, cents[i], cents[i])
        node = len(nodes)
        nodes.append([bb, -1, -1, 0, 0])
        if n <= 4:
            nodes[node][3], nodes[node][4] = start, n
            return node
        ext = [cb[1][k] - cb[0][k] for k in range(3)]
        axis = 0 if (ext[0] >= ext[1] and ext[0] >= ext[2]) else (1 if ext[1] >= ext[2] else 2)
        mid = start + n // 2
        if n >= 16:
            minc, maxc = cb[0][axis], cb[1][axis]
            extent = maxc - minc
            if extent > 1e-12:
                inv_extent = 1.0 / extent
                bins = [[empty(), 0] for _ in range(8)]
                for i in idx[start:end]:
                    b = bin_of(cents[i][axis], minc, inv_extent)
                    bins[b][0] = union(bins[b][0], *bounds[i])
                    bins[b][1] += 1
                lb, lc, rb, rc = [None] * 8, [0] * 8, [None] * 8, [0] * 8
                acc, cnt = empty(), 0
                for i in range(8):
                    if bins[i][1] > 0:
                        acc, cnt = union(acc, *bins[i][0]), cnt + bins[i][1]
                    lb[i], lc[i] = acc, cnt
                acc, cnt = empty(), 0
                for i in range(7, -1, -1):
                    if bins[i][1] > 0:
                        acc, cnt = union(acc, *bins[i][0]), cnt + bins[i][1]
                    rb[i], rc[i] = acc, cnt

                def area(b):
                    e = [b[1][k] - b[0][k] for k in range(3)]
                    return 2.0 * (e[0] * e[1] + e[1] * e[2] + e[2] * e[0])

                best, split = INF, 0
                for i in range(7):
                    if lc[i] == 0 or rc[i + 1] == 0:
                        continue
                    cost = area(lb[i]) * float(lc[i]) + area(rb[i + 1]) * float(rc[i + 1])
                    if cost < best:
                        best, split = cost, i + 1
                if math.isfinite(best):
                    idx[start:end] = sorted(idx[start:end], key=lambda i: bin_of(cents[i][axis], minc, inv_extent))
                    lt = sum(bins[i][1] for i in range(split))
                    if 0 < lt < n:
                        mid = start + lt
        left = build(start, mid)
        right = build(mid, end)
        nodes[node][1], nodes[node][2] = left, right
        return node

    if n_t:
        build(0, n_t)
    return nodes, idx


def cube_mesh():
    """Unit cube centred at the origin, edge 1.0, six quads fan-triangulated."""
    v = [(-0.5, -0.5, -0.5), (0.5, -0.5, -0.5), (0.5, 0.5, -0.5), (-0.5, 0.5, -0.5),
         (-0.5, -0.5, 0.5), (0.5, -0.5, 0.5), (0.5, 0.5, 0.5), (-0.5, 0.5, 0.5)]
    quads = [(0, 1, 2, 3), (4, 7, 6, 5), (0, 4, 5, 1), (1, 5, 6, 2), (2, 6, 7, 3), (3, 7, 4, 0)]
    tris = []
    for q in quads:
        for k in range(1, 3):
            tris.append((q[0], q[k], q[k + 1]))
    return [list(p) for p in v], tris


def icosphere(subdiv):
    t = (1.0 + math.sqrt(5.0)) / 2.0
    base = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
            (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]

    def nrm(p):
        l = math.sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2])
        return [p[0] / l, p[1] / l, p[2] / l]

    v = [nrm(p) for p in base]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            k = (min(a, b), max(a, b))
            if k not in cache:
                cache[k] = len(v)
                v.append(nrm([v[a][i] + v[b][i] for i in range(3)]))
            return cache[k]

        nf = []
        for a, b, c in f:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    # A deterministic radial jitter so the centroid bins are uneven.
    r = Rng(99)
    v = [[p[k] * (1.0 + 0.05 * (r.next_f64() - 0.5)) for k in range(3)] for p in v]
    return v, f


def dump_bvh(pos, tris):
    nodes, idx = bvh_build(pos, tris)
    return {
        "positions": [[x.hex() for x in p] for p in pos],
        "tris": tris,
        "bbox": [[x.hex() for x in n[0][0] + n[0][1]] for n in nodes],
        "left_right": [[n[1], n[2]] for n in nodes],
        "start_count": [[n[3], n[4]] for n in nodes],
        "indices": idx,
    }


def main():
    out = {}
    seeds = [0, 1, 42, 0xDEADBEEFCAFEBABE, M64]
    out["rng_u32"] = {str(s): [Rng(s).next_u32() for _ in range(1)] for s in seeds}
    for s in seeds:
        r = Rng(s)
        out["rng_u32"][str(s)] = [r.next_u32() for _ in range(16)]
    out["rng_f64"] = {}
    for s in seeds:
        r = Rng(s)
        out["rng_f64"][str(s)] = [r.next_f64().hex() for _ in range(8)]
    trip = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (17, 33, 0), (1919, 1079, 0), (5, 7, 3), (4294967295, 4294967295, 0)]
    out["seed_for"] = [[a, b, c, seed_for(a, b, c)] for a, b, c in trip]
    vals = [0, 1, 2, 3, 255, 1023, 65535, 0x12345678, 0xFFFFFFFF, 0x1FFFFFFFF]
    out["interleave_bits"] = [[v, interleave_bits(v)] for v in vals]
    out["tile_order"] = []
    for w, h, tile, morton in [(37, 23, 8, True), (37, 23, 8, False), (64, 64, 16, True), (1920, 1080, 16, True)]:
        out["tile_order"].append({"w": w, "h": h, "tile": tile, "morton": morton, "tasks": tile_order(w, h, tile, morton)})
    out["bvh"] = {"cube": dump_bvh(*cube_mesh()), "ico1": dump_bvh(*icosphere(1)), "ico2": dump_bvh(*icosphere(2))}
    path = Path(__file__).with_name("golden_vectors.json")
    path.write_text(json.dumps(out))
    print(path, path.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
