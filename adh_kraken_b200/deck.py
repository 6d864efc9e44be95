"""Reference file formats on either side of the SW2 time step: the ``.geo`` grid
file and the ``.init`` DATASET restart file, read and written.

Readers follow the reference's own readers card for card:

* ``.geo`` -- sgrid_read (src/structs/sgrid/sgrid_read.c:22-420): header counts
  ``NODES``, ``ELEMS_TRI``, ``ELEMS_SEG``; ``ND gid x y z`` puts node gid-1 at its
  place whatever the line order (sgrid_read_node, :530-590); ``TRI id n1 n2 n3
  [bflag [mat]]`` and ``SEG id n1 n2 [bflag [mat]]`` append elements in file order
  with 1-based node ids (sgrid_read_elem, :597-700).  Every other card is skipped.
  QUAD, TET and PRISM elements are refused: the SW2 path is triangles only.
* ``.init`` -- smodel_super_read_init (src/structs/smodel_super/smodel_super_read_init.c:26-150):
  blocks of ``DATASET`` / ``OBJTYPE`` / ``ND nnodes`` / ``NC`` / ``DIM d`` /
  ``NAME [OLD|OLDER] var`` / ``TS`` / one line of d values per node / ``ENDDS``.
  ``NAME`` picks the level (sol, sol_old, sol_older) and the variable: ``DEPTH``
  (d = 1, dof 3 node) or ``DA_VELOCITY`` (d = 2, dofs 3 node + 1, + 2), the names of
  the SW2 variables in sadh_def.c:28-33.

* ``.params`` time series -- the series pass of smodel_super_read
  (src/structs/smodel_super/smodel_super_read.c:42-61) with sseries_read_allocate
  (src/structs/sseries/sseries.c:46-118): ``SERIES BC id n in_units out_units`` then n
  lines ``t value``; the series gets id - 1, times are scaled by the input unit
  (sdt_get_conversion_factor, src/structs/sdt/sdt.c:50: seconds, minutes, hours, days,
  weeks; units outside 0..4 stop the reference, sdt_check_units :109).  ``SERIES WIND``
  and ``SERIES WAVE`` (two station coordinates, then 2 or 3 values per line) are read past,
  as the reference reads them into lists the SW2 step does not use.

The reference splits ``.geo`` lines on single spaces and copies each into a
100-byte buffer (sgrid_read.c:28); the writer uses single spaces, and its longest
line (an ND card with a 10-digit id and three 24-character ``%.17g`` values) is 88
bytes.  Host code only: nothing here touches the GPU.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, Optional, Sequence

import numpy as np

from .mesh import SW2Case


@dataclass
class GeoGrid:
    xyz: np.ndarray         # (V, 3) float64
    tri: np.ndarray         # (T, 3) int32, 0-based node ids in file order
    seg: np.ndarray         # (S, 2) int32
    tri_bflag: np.ndarray   # (T,) int32, the card's optional bflag (UNSET -> -3)
    seg_bflag: np.ndarray   # (S,) int32


_UNSET_INT = -3             # UNSET_INT, src/include/define.h


def _ints(tok, n, what, line_no):
    try:
        return [int(t) for t in tok[:n]]
    except ValueError as e:
        raise ValueError(f"line {line_no}: bad {what} card") from e


def read_geo(path: str) -> GeoGrid:
    counts = {"NODES": None, "ELEMS_TRI": 0, "ELEMS_SEG": 0}
    nodes: Dict[int, tuple] = {}
    tri, tflag, seg, sflag = [], [], [], []
    with open(path) as f:
        for line_no, line in enumerate(f, 1):
            tok = line.split()
            if not tok:
                continue
            card = tok[0]
            if card in counts:
                counts[card] = int(tok[1])
            elif card in ("ELEMS_QUAD", "ELEMS_TET", "ELEMS_PRISM", "QUAD", "TET", "PRISM"):
                if card.startswith("ELEMS_") and int(tok[1]) == 0:
                    continue
                raise ValueError(f"line {line_no}: {card} elements are not on the SW2 triangle path")
            elif card == "ND":
                gid = int(tok[1])
                if gid in nodes:
                    raise ValueError(f"line {line_no}: node {gid} given twice")
                nodes[gid] = (float(tok[2]), float(tok[3]), float(tok[4]))
            elif card == "TRI":
                v = _ints(tok[1:], 4, "TRI", line_no)
                tri.append([v[1] - 1, v[2] - 1, v[3] - 1])
                tflag.append(int(tok[5]) if len(tok) > 5 else _UNSET_INT)
            elif card == "SEG":
                v = _ints(tok[1:], 3, "SEG", line_no)
                seg.append([v[1] - 1, v[2] - 1])
                sflag.append(int(tok[4]) if len(tok) > 4 else _UNSET_INT)
    V = counts["NODES"]
    if V is None or V <= 0:
        raise ValueError("no NODES count card")
    if sorted(nodes) != list(range(1, V + 1)):
        raise ValueError(f"ND cards do not number the nodes 1..{V}")
    if len(tri) != counts["ELEMS_TRI"] or len(seg) != counts["ELEMS_SEG"]:
        raise ValueError("element counts differ from ELEMS_TRI / ELEMS_SEG")
    xyz = np.array([nodes[i + 1] for i in range(V)], dtype=np.float64).reshape(V, 3)
    tri_a = np.array(tri, dtype=np.int32).reshape(-1, 3)
    seg_a = np.array(seg, dtype=np.int32).reshape(-1, 2)
    for a, what in ((tri_a, "TRI"), (seg_a, "SEG")):
        if a.size and (a.min() < 0 or a.max() >= V):
            raise ValueError(f"{what} card names a node outside 1..{V}")
    return GeoGrid(xyz, tri_a, seg_a, np.array(tflag, np.int32), np.array(sflag, np.int32))


def write_geo(path: str, xyz: np.ndarray, tri: np.ndarray, seg: Optional[np.ndarray] = None,
              seg_bflag: Optional[Sequence[int]] = None) -> None:
    """Write a grid the reference reads back exactly (``%.17g`` coordinates)."""
    xyz = np.asarray(xyz, dtype=np.float64)
    tri = np.asarray(tri)
    seg = np.zeros((0, 2), np.int32) if seg is None else np.asarray(seg)
    with open(path, "w") as f:
        f.write(f"NODES {xyz.shape[0]}\nELEMS_TRI {tri.shape[0]}\nELEMS_SEG {seg.shape[0]}\n")
        for i, (x, y, z) in enumerate(xyz, 1):
            f.write(f"ND {i} {x:.17g} {y:.17g} {z:.17g}\n")
        for e, (a, b, c) in enumerate(tri, 1):
            f.write(f"TRI {e} {a + 1} {b + 1} {c + 1} -1\n")
        for k, (a, b) in enumerate(seg, 1):
            bf = 0 if seg_bflag is None else int(seg_bflag[k - 1])
            f.write(f"SEG {k} {a + 1} {b + 1} {bf}\n")


_LEVELS = {"": 0, "OLD": 1, "OLDER": 2}
_VARS = {"DEPTH": (1, (0,)), "DA_VELOCITY": (2, (1, 2))}


def read_init(path: str, nnodes: int):
    """(sol, sol_old, sol_older) of an ``.init`` file; levels and variables the file
    does not set stay 0, as the reference's zero-initialised arrays do."""
    levels = [np.zeros(3 * nnodes) for _ in range(3)]
    with open(path) as f:
        lines = f.readlines()
    i, n = 0, len(lines)

    def head(card):
        nonlocal i
        if i >= n:
            raise ValueError(f"file ends before {card}")
        tok = lines[i].split()
        if not tok or tok[0] != card:
            raise ValueError(f"line {i + 1}: expected {card}")
        i += 1
        return tok

    while i < n:
        tok = lines[i].split()
        i += 1
        if not tok or tok[0] != "DATASET":
            continue
        head("OBJTYPE")
        nd = int(head("ND")[1])
        if nd != nnodes:
            raise ValueError(f"DATASET has {nd} nodes, the grid {nnodes}")
        head("NC")
        dim = int(head("DIM")[1])
        name = head("NAME")[1:]
        level = 0
        if name and name[0] in ("OLD", "OLDER"):
            level = _LEVELS[name[0]]
            name = name[1:]
        if not name or name[0] not in _VARS:
            raise ValueError(f"line {i}: variable {' '.join(name) or '?'} is not an SW2 variable")
        want, offs = _VARS[name[0]]
        if dim != want:
            raise ValueError(f"line {i}: {name[0]} has DIM {want}, not {dim}")
        head("TS")
        if i + nnodes > n:
            raise ValueError("file ends inside a DATASET")
        vals = np.array([[float(t) for t in lines[i + k].split()] for k in range(nnodes)], dtype=np.float64)
        if vals.shape != (nnodes, dim):
            raise ValueError(f"DATASET {name[0]}: expected {dim} value(s) on each of {nnodes} lines")
        i += nnodes
        head("ENDDS")
        for d, off in enumerate(offs):
            levels[level][off::3] = vals[:, d]
    return tuple(levels)


def write_init(path: str, sol, sol_old, sol_older, nelems: int = 0, t: float = 0.0) -> None:
    """The three levels as six DATASETs (depth and depth-averaged velocity per level)."""
    with open(path, "w") as f:
        for prefix, s in (("", sol), ("OLD ", sol_old), ("OLDER ", sol_older)):
            s = np.asarray(s, dtype=np.float64)
            V = s.size // 3
            for var, (dim, offs) in _VARS.items():
                f.write(f"DATASET\nOBJTYPE \"mesh2d\"\nND {V}\nNC {nelems}\nDIM {dim}\nNAME {prefix}{var}\n")
                f.write(f"TS 0 {t:.17g}\n")
                cols = np.stack([s[o::3] for o in offs], axis=1)
                for row in cols:
                    f.write(" ".join(f"{v:.17g}" for v in row) + "\n")
                f.write("ENDDS\n")


_UNIT_SECONDS = {0: 1, 1: 60, 2: 3600, 3: 86400, 4: 604800}   # sdt_get_conversion_factor (an int)


def _tokens(line: str):
    # get_token / get_next_token (src/tokens/tokens.c:10-40): strtok on " \t\n"
    return line.replace("\t", " ").replace("\n", " ").split(" ")


def read_params_series(path: str) -> Dict[int, tuple]:
    """The ``SERIES BC`` time series of a ``.params`` file as the reference reads them:
    {id (file id - 1): (times in seconds, values)}, in file order."""
    out: Dict[int, tuple] = {}
    with open(path) as fh:
        lines = fh.readlines()
    i = 0
    while i < len(lines):
        tok = [t for t in _tokens(lines[i]) if t]
        i += 1
        if not tok or tok[0] != "SERIES" or len(tok) < 2:
            continue
        kind = tok[1]
        if kind not in ("BC", "WIND", "WAVE"):
            raise ValueError(f"{path}:{i}: series type {kind} not recognised")
        rest = tok[2:]
        sid, n = int(rest[0]) - 1, int(rest[1])
        if kind in ("WIND", "WAVE"):
            rest = rest[2:]             # station x, y
        in_units, out_units = int(rest[2]), int(rest[3])
        for u, what in ((in_units, "input"), (out_units, "output")):
            if u not in _UNIT_SECONDS:
                raise ValueError(f"{path}:{i}: invalid {what} time units {u} (0..4)")
        nval = {"BC": 1, "WIND": 2, "WAVE": 3}[kind]
        times = np.empty(n)
        values = np.empty((n, nval))
        for k in range(n):
            et = [t for t in _tokens(lines[i]) if t]
            i += 1
            times[k] = float(et[0]) * _UNIT_SECONDS[in_units]
            for v in range(nval):
                values[k, v] = float(et[1 + v]) if 1 + v < len(et) else -999.0
        if kind == "BC":
            out[sid] = (times, values[:, 0].copy())
    return out


def case_from_files(name: str, geo_path: str, init_path: str, seg_kind, dt: float, nsteps: int,
                    series, t0: float = 0.0, **kw) -> SW2Case:
    """An SW2Case from a ``.geo`` grid and an ``.init`` state.  ``seg_kind`` gives each
    segment's boundary (0 NB VEL, 1 DEPTH, 2-5 the structure strings): an array over the
    segments, or a dict from the SEG cards' bflag to the kind.  ``series`` is a dict of
    time series or the path of a ``.params`` file to read them from.  The case starts
    from the file's current level."""
    if isinstance(series, str):
        series = read_params_series(series)
    g = read_geo(geo_path)
    if isinstance(seg_kind, dict):
        kinds = np.array([seg_kind[int(b)] for b in g.seg_bflag], dtype=np.int32)
    else:
        kinds = np.asarray(seg_kind, dtype=np.int32)
    if kinds.shape != (g.seg.shape[0],):
        raise ValueError("one boundary kind per segment is needed")
    sol, _, _ = read_init(init_path, g.xyz.shape[0])
    return SW2Case(name, g.xyz, g.tri, g.seg, kinds, sol, dt, nsteps, series, t0=t0, **kw)
