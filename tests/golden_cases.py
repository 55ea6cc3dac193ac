"""Load the golden fixtures (tests/golden/*.npz) as decks + reference outputs."""
import glob
import os
import tempfile

import numpy as np

from bd_box_b200 import decks

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = tempfile.mkdtemp(prefix="golden_")
    with open(os.path.join(d, "c.prm"), "w") as f:
        f.write(str(z["prm"]))
    with open(os.path.join(d, "c.str"), "w") as f:
        f.write(str(z["str"]))
    deck = decks.read_deck(os.path.join(d, "c.prm"))
    return deck, {k: z[k] for k in z.files if k not in ("prm", "str")}
