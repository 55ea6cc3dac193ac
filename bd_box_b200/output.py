"""BD_BOX's trajectory file formats, written from frames taken with
System.frames_take (bdb_frames_*), byte for byte as BD_BOX writes them:

* XYZ (save_xyz, output.c:64-75): the bead count, the line
  "<xyz_filename> time [ps] <curr_time>", then "<name> <x> <y> <z>" per bead,
  all numbers with C's "%f";
* DCD (init_dcd, output.c:97-141, and save_dcd :77-95): a CHARMM-style
  header whose frame count is bdsteps / save_dcd_freq, then per frame the
  x, y and z blocks as float32, each between two 4-byte block sizes;
* energies (init_enr :152-156, save_energy :143-150): a header line, then
  per frame the time, the sum of the terms and the terms, "%15f" and "%15g".

The bytes are pinned against BD_BOX's own output.c by
tests/test_output_format.py.
"""
from __future__ import annotations

import struct

import numpy as np


class XYZWriter:
    """save_xyz: `title` is the xyz_filename string BD_BOX prints in the
    comment line (the deck's value, as given)."""

    def __init__(self, path: str, names, title: str):
        self.f = open(path, "w")
        self.names = list(names)
        self.title = title

    def write(self, time: float, coord: np.ndarray):
        n = len(self.names)
        c = np.asarray(coord, dtype=np.float64).reshape(n, -1)
        lines = [f"{n}\n", f"{self.title} time [ps] {time:f}\n"]
        lines += [f"{self.names[i]} {c[i, 0]:f} {c[i, 1]:f} {c[i, 2]:f}\n" for i in range(n)]
        self.f.write("".join(lines))
        self.f.flush()

    def close(self):
        self.f.close()


class DCDWriter:
    """init_dcd + save_dcd for `n` beads; `header_frames` is the count the
    header announces (BD_BOX: bdsteps / save_dcd_freq)."""

    def __init__(self, path: str, n: int, header_frames: int):
        self.f = open(path, "wb")
        self.n = n
        icntrl = [header_frames, 0, 1, 0, 0, 0, 0, 0, 0]
        # init_dcd writes sizeof(float) bytes of the double DELTA = 1.0: its
        # first four bytes in memory, zero on a little-endian host
        delta = struct.pack("<d", 1.0)[:4]
        title = b"bd_box DCD file".ljust(80, b"\0")
        hdr = struct.pack("<I", 84) + b"CORD" + struct.pack("<9i", *icntrl) + delta
        hdr += struct.pack("<10i", *([0] * 10)) + struct.pack("<I", 84)
        hdr += struct.pack("<I", 84) + struct.pack("<i", 1) + title + struct.pack("<I", 84)
        hdr += struct.pack("<I", 4) + struct.pack("<i", n) + struct.pack("<I", 4)
        self.f.write(hdr)
        self.f.flush()

    def write(self, coord: np.ndarray):
        c = np.asarray(coord, dtype=np.float64).reshape(self.n, -1)
        size = struct.pack("<I", 4 * self.n)
        out = b""
        for k in range(3):
            out += size + c[:, k].astype("<f4").tobytes() + size
        self.f.write(out)
        self.f.flush()

    def close(self):
        self.f.close()


# ENERGY_TYPE indices (data.h:278-289)
E_BOND, E_ANGLE, E_ANGLE_COS, E_DIHE, E_DIHE_ANGLE, E_LJ, E_COULOMB = 1, 2, 3, 4, 5, 6, 7


class ENRWriter:
    """init_enr + save_energy. The columns are BD_BOX's, labels included
    (its DIHE column holds the dihedral-angle term and DIHE_COS the cosine
    dihedral term)."""

    def __init__(self, path: str):
        self.f = open(path, "w")
        self.f.write("#%14s%15s %15s %15s %15s %15s %15s %15s %15s\n" %
                     ("TIME", "ALL", "BOND", "ANG", "ANG_COS", "DIHE", "DIHE_COS", "LJ", "COULOMB"))
        self.f.flush()

    def write(self, time: float, E):
        E = [float(v) for v in E]
        total = E[E_BOND] + E[E_ANGLE] + E[E_ANGLE_COS] + E[E_DIHE_ANGLE] + E[E_DIHE] + E[E_LJ] + E[E_COULOMB]
        self.f.write("%15f%15f %15g %15g %15g %15g %15g %15g %15g\n" %
                     (time, total, E[E_BOND], E[E_ANGLE], E[E_ANGLE_COS], E[E_DIHE_ANGLE], E[E_DIHE], E[E_LJ],
                      E[E_COULOMB]))
        self.f.flush()

    def close(self):
        self.f.close()
