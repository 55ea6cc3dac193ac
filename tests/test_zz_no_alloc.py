"""bdb_stored_matvec_noalloc: the allocation-free variant of the Cholesky
path's per-step products, for callers that cannot call cudaMalloc (a host
whose device memory belongs to its own pool allocator, or a loop that must
not allocate). The caller owns every buffer; the function keeps its partial
sums in a fixed array inside the library.

Checked through the C ABI against the existing entry points of a system on
the same deck (bdb_compute_Rf and bdb_compute_r of the mixed-precision
path), within the mixed path's 1e-5 bound, on two calls in a row. This file
sorts last so that a run stopping at the first failure has run every other
test already.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not gpu_available(), reason="needs a CUDA device")]

from bd_box_b200 import decks, engine  # noqa: E402

KB = 0.001986248532617   # Boltzmann constant in BD_BOX's units (data.h)


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


# (beads, extra row padding): a small case; 3N = 3072, where the partial sums
# fill the fixed array exactly; and 3N = 603, not a multiple of 4, whose edge
# tiles take the scalar loads, with rows padded past the next multiple of 4
@pytest.mark.parametrize("beads,pad", [(200, 0), (1024, 0), (201, 64)])
def test_noalloc_matches_existing_entry_points(tmp_path, beads, pad):
    import torch
    deck = decks.read_deck(decks.write_chain_deck(str(tmp_path), "na", beads, seed=41, hydro="cholesky"))
    n3 = 3 * deck.n
    dt, T = deck.prm["dt"], deck.prm["T"]
    g = np.random.default_rng(3).standard_normal(n3)

    # existing entry points
    s = engine.System(deck, precision=engine.PREC_MIXED, noise=engine.NOISE_HOST)
    F, _, _, _ = s.compute_forces(energies=False)
    Rf_ref = s.compute_Rf()
    Rs_ref = s.compute_r(g)
    D = s.compute_D()

    # caller-owned buffers: M holds D above the diagonal and L on/below it
    L = np.linalg.cholesky(D)
    ld = (n3 + 3) // 4 * 4 + pad
    Mh = np.zeros((n3, ld), dtype=np.float32)
    Mh[:, :n3] = np.triu(D, 1) + L
    dev = torch.device("cuda")
    M = torch.from_numpy(Mh).to(dev)
    dD = torch.from_numpy(np.diag(D).copy()).to(dev)
    Fd = torch.from_numpy(F).to(dev)
    X = torch.from_numpy(g * np.sqrt(2 * dt)).to(dev)
    Rf = torch.empty(n3, dtype=torch.float64, device=dev)
    Rs = torch.empty(n3, dtype=torch.float64, device=dev)
    lib = engine.load_library()
    stream = torch.cuda.current_stream().cuda_stream
    outs = []
    for _ in range(2):
        Rf.fill_(float("nan"))
        Rs.fill_(float("nan"))
        rc = lib.bdb_stored_matvec_noalloc(M.data_ptr(), n3, ld, dD.data_ptr(), Fd.data_ptr(), X.data_ptr(),
                                           dt / (KB * T), Rf.data_ptr(), Rs.data_ptr(), C.c_void_p(stream))
        assert rc == 0, lib.bdb_last_error().decode()
        torch.cuda.synchronize()
        outs.append((Rf.cpu().numpy().copy(), Rs.cpu().numpy().copy()))
    for rf, rs in outs:
        assert rel(rf, Rf_ref) <= 1e-5
        assert rel(rs, Rs_ref) <= 1e-5
    # the second call sees the previous call's scratch contents and must not depend on them
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    lib = engine.load_library()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    rc = lib.bdb_stored_matvec_noalloc(p, 4096, 4096, p, p, p, 1.0, p, p, None)
    assert rc == -1
    assert b"3072" in lib.bdb_last_error()
