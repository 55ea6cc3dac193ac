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
    if "cos_dihe" in z.files:
        # cosine dihedrals added through BD_BOX's add_dihe (its .str parser
        # cannot read them): rows (i, j, k, l, k_theta, m, delta), stored as
        # add_dihe stores them, (-k_theta delta, m)
        rows = z["cos_dihe"]
        deck.dihe_pairs = rows[:, :4].astype(np.int32)
        deck.dihe_parms = np.stack([-rows[:, 4] * rows[:, 6], rows[:, 5]], axis=1)
    return deck, {k: z[k] for k in z.files if k not in ("prm", "str")}
