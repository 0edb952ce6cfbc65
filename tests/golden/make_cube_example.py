"""Generates tests/golden/cube_example.json from the reference's own example model
(examples/cube.msh and examples/cube.toml of the reference project): 8 nodes, 6 Tet4, young
200e3, poisson 0.25, node sets x0 (ux = 0), x1 (ux = 0.01), y0 (uy = 0), z0 (uz = 0). The
reference checks it against the analytic field ux = 0.01 x, uy = -0.25 * 0.01 y,
uz = -0.25 * 0.01 z (crates/maille-cli/tests/examples.rs:669-681).

Run where the reference tree is checked out: python tests/golden/make_cube_example.py <reference root>
"""
import json
import os
import sys


def parse_msh41(path):
    lines = open(path).read().split("\n")
    i = 0
    names, point_groups, nodes, tets, point_nodes = {}, {}, {}, [], {}
    while i < len(lines):
        s = lines[i].strip()
        if s == "$PhysicalNames":
            n = int(lines[i + 1])
            for k in range(n):
                dim, tag, name = lines[i + 2 + k].split(maxsplit=2)
                names[(int(dim), int(tag))] = name.strip('"')
            i += n + 2
        elif s == "$Entities":
            npt = int(lines[i + 1].split()[0])
            for k in range(npt):
                f = lines[i + 2 + k].split()
                tag, nphys = int(f[0]), int(f[4])
                point_groups[tag] = [int(t) for t in f[5:5 + nphys]]
            i += 1
        elif s == "$Nodes":
            nblocks = int(lines[i + 1].split()[0])
            j = i + 2
            for _ in range(nblocks):
                _, _, _, count = (int(v) for v in lines[j].split())
                tags = [int(lines[j + 1 + k]) for k in range(count)]
                for k, t in enumerate(tags):
                    nodes[t] = [float(v) for v in lines[j + 1 + count + k].split()]
                j += 1 + 2 * count
            i = j
        elif s == "$Elements":
            nblocks = int(lines[i + 1].split()[0])
            j = i + 2
            for _ in range(nblocks):
                dim, ent, etype, count = (int(v) for v in lines[j].split())
                for k in range(count):
                    f = [int(v) for v in lines[j + 1 + k].split()]
                    if etype == 15:
                        point_nodes.setdefault(ent, []).append(f[1])
                    elif etype == 4:
                        tets.append(f[1:5])
                j += 1 + count
            i = j
        else:
            i += 1
    return names, point_groups, nodes, tets, point_nodes


def main(ref_root):
    names, point_groups, nodes, tets, point_nodes = parse_msh41(
        os.path.join(ref_root, "examples", "cube.msh"))
    order = sorted(nodes)
    index = {t: k for k, t in enumerate(order)}
    coords = [nodes[t] for t in order]
    conn = []
    for t in tets:
        q = [index[v] for v in t]
        p = [coords[v] for v in q]
        a = [p[1][c] - p[0][c] for c in range(3)]
        b = [p[2][c] - p[0][c] for c in range(3)]
        c = [p[3][k] - p[0][k] for k in range(3)]
        six_v = (a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0])
                 + a[2] * (b[0] * c[1] - b[1] * c[0]))
        if six_v < 0:  # maille-io orient(): swap the first two vertices of a reversed tet
            q[0], q[1] = q[1], q[0]
        conn.append(q)
    sets = {}
    for ent, groups in point_groups.items():
        for g in groups:
            sets.setdefault(names[(0, g)], []).extend(index[v] for v in point_nodes.get(ent, []))
    bcs = []
    for name, dof, value in (("x0", 0, 0.0), ("x1", 0, 0.01), ("y0", 1, 0.0), ("z0", 2, 0.0)):
        for v in sorted(set(sets[name])):
            bcs.append([v, dof, value])
    out = dict(source="examples/cube.msh + examples/cube.toml (reference)", young=200e3,
               poisson=0.25, coords=coords, conn=conn, bcs=bcs,
               expected="ux = 0.01 x, uy = -0.25*0.01 y, uz = -0.25*0.01 z within 1e-12")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cube_example.json")
    json.dump(out, open(path, "w"), indent=1)
    print(path)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_cube_example.py <root of the reference project>")
    main(sys.argv[1])
