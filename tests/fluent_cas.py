"""A reader of ASCII Fluent case files (.cas), test infrastructure: the
reference's example grid rae2822_hybrid2d__4.fts was converted from the
Fluent case beside it, so the two files describe the same nodes, faces and
cells, and an independent parse of the case checks the .fts reader.

Sections of the format read here (all indices hexadecimal, 1-based):

* (10 (zone first last type nd)( x y [z] ... ))      nodes
* (13 (zone first last bctype facetype)( ... ))      faces: per face its
  nodes (a count first when facetype is 0, mixed), then the cells on its
  two sides (c0 c1; 0 where there is none)
* (12 (zone first last type elemtype)( ... ))        cells
* (45 (zone type name)())                            zone names
Zone 0 headers are declarations with no data.
"""
from __future__ import annotations

import re

import numpy as np

_HEAD = re.compile(r"\((10|12|13|45) \(([^()]*)\)")

# Fluent face-zone boundary types used by the example case
FLUENT_INTERIOR = 2
FLUENT_WALL = 3
FLUENT_PRESSURE_FAR_FIELD = 9


def read_cas(path: str) -> dict:
    text = open(path).read()
    nodes, faces, cells, names = [], [], 0, {}
    nd = 2
    m = re.search(r"\(2 (\d)\)", text)
    if m:
        nd = int(m.group(1))
    pos = 0
    while True:
        h = _HEAD.search(text, pos)
        if not h:
            break
        kind = int(h.group(1))
        fields = h.group(2).split()
        pos = h.end()
        if kind == 45:
            names[int(fields[0])] = (fields[1], fields[2])
            continue
        zone = int(fields[0], 16)
        first, last = int(fields[1], 16), int(fields[2], 16)
        if zone == 0:
            continue
        if text[pos] != "(":
            continue
        end = text.index(")", pos + 1)
        body = text[pos + 1:end].split()
        pos = end
        if kind == 10:
            xyz = np.array([float(v) for v in body]).reshape(last - first + 1, nd)
            nodes.append((first, xyz))
        elif kind == 13:
            bctype, ftype = int(fields[3], 16), int(fields[4], 16)
            vals = [int(v, 16) for v in body]
            k = 0
            for _ in range(last - first + 1):
                if ftype == 0:
                    nn = vals[k]
                    k += 1
                else:
                    nn = ftype
                fn = vals[k:k + nn]
                c0, c1 = vals[k + nn], vals[k + nn + 1]
                k += nn + 2
                faces.append((zone, bctype, tuple(v - 1 for v in fn), c0 - 1, c1 - 1))
        elif kind == 12:
            cells = max(cells, last)
    nodes.sort()
    xyz = np.concatenate([a for _, a in nodes])
    return {"ndim": nd, "xyz": xyz, "faces": faces, "n_cell": cells, "zone_names": names}
