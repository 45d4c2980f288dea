"""Reader and writer of the reference's dump files.

Format of read_dump_information (src/IO/dump-input.cpp:51-214):

    ITEM: TIMESTEP / <int>
    ITEM: NUMBER OF ATOMS / <n>
    ITEM: BOX BOUNDS <bx> <by> <bz>      ("pp" periodic, "ff" open)
    <xmin> <xmax> / <ymin> <ymax> / <zmin> <zmax>
    ITEM: ATOMS type x y z stdvq molarfraction chemicalmultp thermalmultp
                chemicalmultpbcc thermalmultpbcc
    n rows of those 10 columns

Species are atomic numbers (the reference casts the type column to its
AtomicSpecie enum, 193-198).  The orthogonal box becomes origin = lo and
cell = diag(hi - lo).  The writer emits the same layout
(write_dump_information, src/IO/dump-output.cpp:52-157) so a state can be
checkpointed and read back.
"""
from __future__ import annotations

import numpy as np


def read_dump(path):
    with open(path) as f:
        lines = f.read().splitlines()
    it = iter(lines)
    next(it)
    timestep = int(next(it).split()[0])
    next(it)
    n = int(next(it).split()[0])
    bounds = next(it).split()
    bc = bounds[3:6]
    lo, hi = np.zeros(3), np.zeros(3)
    for a in range(3):
        v = next(it).split()
        lo[a], hi[a] = float(v[0]), float(v[1])
    next(it)
    rows = np.array([[float(t) for t in next(it).split()[:10]] for _ in range(n)])
    species = rows[:, 0].astype(np.int32)
    if np.any((species < 1) | (species > 111)):
        raise ValueError("dump: particle type outside 1..111")
    return dict(q=np.ascontiguousarray(rows[:, 1:4]),
                sigma=np.ascontiguousarray(rows[:, 4]),
                x=np.ascontiguousarray(rows[:, 5]),
                gamma=np.ascontiguousarray(rows[:, 6]),
                beta=np.ascontiguousarray(rows[:, 7]),
                gamma_bcc=rows[:, 8].astype(np.int32),
                beta_bcc=rows[:, 9].astype(np.int32),
                species=species,
                origin=lo.copy(), cell=np.diag(hi - lo),
                periodic=np.array([1 if b == "pp" else 0 for b in bc], np.int32),
                timestep=timestep)


def write_dump(path, s, timestep=0):
    cell = np.asarray(s["cell"])
    if np.any(np.abs(cell - np.diag(np.diag(cell))) > 0):
        raise ValueError("dump format holds orthogonal boxes only")
    lo = np.asarray(s["origin"])
    hi = lo + np.diag(cell)
    n = len(s["x"])
    bc = ["pp" if p else "ff" for p in s["periodic"]]
    gb = s.get("gamma_bcc", np.zeros(n))
    bb = s.get("beta_bcc", np.zeros(n))
    with open(path, "w") as f:
        f.write(f"ITEM: TIMESTEP\n{timestep}\nITEM: NUMBER OF ATOMS\n{n}\n")
        f.write(f"ITEM: BOX BOUNDS {bc[0]} {bc[1]} {bc[2]}\n")
        for a in range(3):
            f.write(f"{float(lo[a])!r} {float(hi[a])!r}\n")
        f.write("ITEM: ATOMS type x y z stdvq molarfraction chemicalmultp thermalmultp "
                "chemicalmultpbcc thermalmultpbcc\n")
        for i in range(n):
            vals = [*map(float, s["q"][i]), float(s["sigma"][i]), float(s["x"][i]),
                    float(s["gamma"][i]), float(s["beta"][i]), float(gb[i]), float(bb[i])]
            f.write(f"{int(s['species'][i])} " + " ".join(repr(v) for v in vals) + "\n")
