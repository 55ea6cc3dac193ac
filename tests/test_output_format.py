"""The XYZ, DCD and energy writers of bd_box_b200.output against BD_BOX's own
output.c: the reference harness (oracle/_ref/ref_harness, mode "output")
runs steps with the reference's init_save / save_output / free_save and
dumps the coordinates it saved; our writers get the same coordinates and
times and must produce the same bytes."""
import os
import subprocess

import numpy as np
import pytest

from bd_box_b200 import decks, output

HARNESS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "ref_harness")


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("hydro,xyz_freq,dcd_freq,enr_freq,K", [("none", 2, 3, 2, 6), ("geyer", 1, 2, 3, 5)])
def test_writers_match_bd_box_output(tmp_path, hydro, xyz_freq, dcd_freq, enr_freq, K):
    p = decks.write_chain_deck(str(tmp_path), "out", 17, seed=5, hydro=hydro)
    deck = decks.read_deck(p)
    n = deck.n
    np.random.default_rng(3).standard_normal(3 * n * (K + 2)).tofile(tmp_path / "g.bin")
    bdsteps = K + 1
    env = dict(os.environ, BDB_GAUSS_FILE=str(tmp_path / "g.bin"), OMP_NUM_THREADS="1")
    subprocess.run([HARNESS, "out.prm", "output", "coords.bin", str(K), "--xyz_filename=ref.xyz",
                    "--dcd_filename=ref.dcd", "--enr_filename=ref.enr", f"--save_xyz_freq={xyz_freq}",
                    f"--save_dcd_freq={dcd_freq}", f"--save_enr_freq={enr_freq}", f"--bdsteps={bdsteps}"],
                   cwd=tmp_path, env=env, check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    rec = np.fromfile(tmp_path / "coords.bin").reshape(K + 1, 4 * n + 9)
    coords = rec[:, :4 * n].reshape(K + 1, n, 4)
    energies = rec[:, 4 * n:]
    # curr_time accumulates dt step by step (diff_comp.c:216)
    times = [0.0]
    for _ in range(K):
        times.append(times[-1] + deck.prm["dt"])
    xw = output.XYZWriter(str(tmp_path / "ours.xyz"), deck.names, "ref.xyz")
    dw = output.DCDWriter(str(tmp_path / "ours.dcd"), n, bdsteps // dcd_freq)
    ew = output.ENRWriter(str(tmp_path / "ours.enr"))
    for k in range(K + 1):
        if k % xyz_freq == 0:
            xw.write(times[k], coords[k])
        if k % dcd_freq == 0:
            dw.write(coords[k])
        if k % enr_freq == 0:
            ew.write(times[k], energies[k])
    xw.close()
    dw.close()
    ew.close()
    # LJ and Debye-Hueckel terms on every written step, bonds once they
    # stretch (the chain starts at the bond length)
    saved = energies[::enr_freq]
    assert np.all(saved[:, [6, 7]] != 0) and np.any(saved[:, 1] != 0)
    for a, b in (("ours.xyz", "ref.xyz"), ("ours.dcd", "ref.dcd"), ("ours.enr", "ref.enr")):
        assert (tmp_path / a).read_bytes() == (tmp_path / b).read_bytes(), a
