"""Generate kf_mc_tables.h: the marching-cubes triangulation used by this library.

The table is derived here, case by case, instead of being transcribed:

* corner c of a cell sits at offset kCorner[c] (the classic layout), edge e
  joins corners kEdge[e] = (near, far) along one axis;
* for each of the 256 sign cases (bit c set: corner c has tsdf < 0, inside),
  every cube face contributes contour segments: walking the face's corners
  counter-clockwise as seen from outside the cell, each crossing where the
  walk enters the inside is joined to the next crossing where it leaves it.
  On a face with two diagonal inside corners this keeps the inside corners
  apart, a choice that depends on the face alone, so neighbouring cells agree
  and the mesh has no cracks;
* the segments chain into closed loops (each crossed edge starts one segment
  and ends one), and each loop is cut into a triangle fan from its first
  edge.  Triangles are wound so that their normal points from the inside
  (negative) to the outside (positive).

Run `python mc_tables.py` to rewrite the header next to this file.
"""
import itertools
import pathlib

CORNERS = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
EDGES = [(0, 1), (1, 2), (3, 2), (0, 3), (4, 5), (5, 6), (7, 6), (4, 7), (0, 4), (1, 5), (2, 6), (3, 7)]
# faces as corner cycles, counter-clockwise seen from outside the cell
FACES = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (3, 7, 6, 2), (0, 4, 7, 3), (1, 2, 6, 5)]


def edge_of(a, b):
    for e, (p, q) in enumerate(EDGES):
        if {p, q} == {a, b}:
            return e
    raise KeyError((a, b))


def loops_of(case):
    inside = [(case >> c) & 1 for c in range(8)]
    nxt = {}
    for face in FACES:
        walk = [(face[i], face[(i + 1) % 4]) for i in range(4)]
        crossings = [(i, inside[p], edge_of(p, q)) for i, (p, q) in enumerate(walk) if inside[p] != inside[q]]
        for k, (i, p_in, e) in enumerate(crossings):
            if p_in:
                continue  # leaves the inside; it ends a segment
            # enters the inside: join it to the next crossing that leaves it
            for j in range(1, len(crossings) + 1):
                _, q_in, f = crossings[(k + j) % len(crossings)]
                if q_in:
                    assert e not in nxt
                    nxt[e] = f
                    break
    loops, seen = [], set()
    for start in sorted(nxt):
        if start in seen:
            continue
        loop, e = [], start
        while e not in seen:
            seen.add(e)
            loop.append(e)
            e = nxt[e]
        assert e == start
        loops.append(loop)
    return loops


def midpoint(e):
    p, q = EDGES[e]
    return [(CORNERS[p][i] + CORNERS[q][i]) / 2 for i in range(3)]


def sub(a, b):
    return [a[i] - b[i] for i in range(3)]


def cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def dot(a, b):
    return sum(a[i] * b[i] for i in range(3))


def triangles_of(case, flip):
    tris = []
    for loop in loops_of(case):
        for k in range(1, len(loop) - 1):
            t = (loop[0], loop[k], loop[k + 1])
            tris.append((t[0], t[2], t[1]) if flip else t)
    return tris


def field(case, p):
    """Trilinear blend of the corner signs (inside -1, outside +1) at p."""
    value = 0.0
    for c, (cx, cy, cz) in enumerate(CORNERS):
        w = (p[0] if cx else 1 - p[0]) * (p[1] if cy else 1 - p[1]) * (p[2] if cz else 1 - p[2])
        value += w * (-1.0 if (case >> c) & 1 else 1.0)
    return value


def orientation_ok(case, tris):
    """Every triangle's normal has the direction of the blended field's gradient."""
    h = 1e-4
    for t in tris:
        a, b, c = (midpoint(e) for e in t)
        n = cross(sub(b, a), sub(c, a))
        centre = [(a[i] + b[i] + c[i]) / 3 for i in range(3)]
        g = []
        for i in range(3):
            hi, lo = list(centre), list(centre)
            hi[i] += h
            lo[i] -= h
            g.append((field(case, hi) - field(case, lo)) / (2 * h))
        if dot(n, g) <= 0:
            return False
    return True


def build():
    # one global winding convention; check it against the single-corner case
    flip = not orientation_ok(1, triangles_of(1, False))
    masks, table = [], []
    for case in range(256):
        inside = [(case >> c) & 1 for c in range(8)]
        mask = 0
        for e, (p, q) in enumerate(EDGES):
            if inside[p] != inside[q]:
                mask |= 1 << e
        tris = triangles_of(case, flip)
        assert len(tris) <= 5, (case, tris)
        used = {e for t in tris for e in t}
        assert used == {e for e in range(12) if mask >> e & 1}, case
        assert orientation_ok(case, tris), case
        masks.append(mask)
        table.append([e for t in tris for e in t] + [-1] * (16 - 3 * len(tris)))
    return masks, table


def check_watertight(masks, table):
    # every crossed edge of a case is shared by exactly two triangle sides
    for case in range(1, 255):
        count = {}
        tris = [table[case][i:i + 3] for i in range(0, 15, 3) if table[case][i] >= 0]
        for t in tris:
            for a, b in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
                count[(a, b)] = count.get((a, b), 0) + 1
        for (a, b), n in count.items():
            assert n == 1, (case, a, b)  # no doubled directed side


def main():
    masks, table = build()
    check_watertight(masks, table)
    lines = [
        "// kf_mc_tables.h - generated by mc_tables.py; do not edit.",
        "//",
        "// Marching-cubes triangulation of this library: kMcEdgeMask[case] has bit",
        "// e set when cube edge e is crossed; kMcTriangles[case] lists the case's",
        "// triangles as triples of cube edges, wound with the normal pointing from",
        "// the inside (tsdf < 0) to the outside, -1 terminated.  Corner and edge",
        "// numbering: corner c at kMcCorner[c], edge e from kMcEdge[e][0] (near) to",
        "// kMcEdge[e][1] (far) along axis kMcEdge[e][2].",
        "#pragma once",
        "",
        "#include <stdint.h>",
        "",
        "static const uint8_t kMcCorner[8][3] = {" + ", ".join("{%d, %d, %d}" % c for c in CORNERS) + "};",
    ]
    axes = []
    for p, q in EDGES:
        d = [CORNERS[q][i] - CORNERS[p][i] for i in range(3)]
        axes.append(d.index(1))
    lines.append("static const uint8_t kMcEdge[12][3] = {" +
                 ", ".join("{%d, %d, %d}" % (p, q, a) for (p, q), a in zip(EDGES, axes)) + "};")
    lines.append("static const uint16_t kMcEdgeMask[256] = {")
    for i in range(0, 256, 16):
        lines.append("    " + ", ".join("0x%03x" % m for m in masks[i:i + 16]) + ",")
    lines.append("};")
    lines.append("static const int8_t kMcTriangles[256][16] = {")
    for row in table:
        lines.append("    {" + ", ".join("%d" % v for v in row) + "},")
    lines.append("};")
    out = pathlib.Path(__file__).with_name("kf_mc_tables.h")
    out.write_text("\n".join(lines) + "\n")
    return out


if __name__ == "__main__":
    print(main())
