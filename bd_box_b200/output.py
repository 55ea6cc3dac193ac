"""BD_BOX's trajectory file formats, written from frames taken with
System.frames_take (bdb_frames_*), byte for byte as BD_BOX writes them:

* XYZ (save_xyz, output.c:64-75): the bead count, the line
  "<xyz_filename> time [ps] <curr_time>", then "<name> <x> <y> <z>" per bead,
  all numbers with C's "%f";
* DCD (init_dcd, output.c:97-141, and save_dcd :77-95): a CHARMM-style
  header whose frame count is bdsteps / save_dcd_freq, then per frame the
  x, y and z blocks as float32, each between two 4-byte block sizes.

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
