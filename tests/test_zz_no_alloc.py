"""The allocation-free pair-list entry point, pgm_pair_list_noalloc, through the C ABI.

It serves callers that cannot allocate device memory (MD engines whose memory pool owns the whole GPU, hosts
that reserve their device memory up front): its scratch is one static device array of the library.
Its pair set must equal the one the engine's own entry point produces (pgm_engine_pairs after an
evaluation), bit for bit, on two calls in a row (the second call finds the first call's scratch contents).
This file runs last so that a failure here comes after every other test has run; it also passes alone.
"""

import numpy as np
import pytest

from conftest import PKG, load_golden_system

pytestmark = pytest.mark.gpu


def pairs_from_rows(slot_atom, counts, neighbors):
    I, J = [], []
    for s in range(len(slot_atom)):
        i = int(slot_atom[s])
        js = neighbors[s, :counts[s]]
        sel = js > i
        I.append(np.full(int(sel.sum()), i))
        J.append(js[sel])
    I = np.concatenate(I).astype(np.int64)
    J = np.concatenate(J).astype(np.int64)
    order = np.lexsort((J, I))
    return I[order], J[order]


def test_noalloc_pair_list_matches_engine():
    import torch
    S, _ = load_golden_system("water216")
    eng = PKG.Engine(PKG.Settings(cutoff=S.cutoff, beta=S.beta, grid=S.grid, order=S.order, tol=1e-10,
                                  max_iter=1000, peek=0.0, predictor=0, precision=PKG.FP64))
    eng.set_system(S)
    eng.compute(S.pos, S.box)
    ei, ej = eng.pairs()
    dev = torch.device("cuda:0")
    cap = 512
    pos = torch.from_numpy(S.pos).to(dev).contiguous()
    slot_atom = torch.empty(S.n, dtype=torch.int32, device=dev)
    counts = torch.empty(S.n, dtype=torch.int32, device=dev)
    nbrs = torch.empty((S.n, cap), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        slot_atom.fill_(-1)
        counts.fill_(-1)
        nbrs.fill_(-1)
        torch.cuda.synchronize()
        mx = PKG.pair_list_noalloc(S.n, pos.data_ptr(), S.box, S.cutoff, cap, slot_atom.data_ptr(),
                                   counts.data_ptr(), nbrs.data_ptr(), stream)
        sa, c, nb = slot_atom.cpu().numpy(), counts.cpu().numpy(), nbrs.cpu().numpy()
        assert sorted(sa.tolist()) == list(range(S.n))
        assert mx == c.max() and 0 < mx <= cap   # the longest row, reported on every call
        pi, pj = pairs_from_rows(sa, c, nb)
        assert np.array_equal(pi, ei) and np.array_equal(pj, ej), call
        assert int(c.sum()) == 2 * len(ei)
    eng.close()


def test_noalloc_rejects_beyond_its_limits():
    import torch
    S, _ = load_golden_system("tiny_triclinic")
    dev = torch.device("cuda:0")
    pos = torch.from_numpy(S.pos).to(dev).contiguous()
    sa = torch.empty(S.n, dtype=torch.int32, device=dev)
    c = torch.empty(S.n, dtype=torch.int32, device=dev)
    nb = torch.empty((S.n, 4), dtype=torch.int32, device=dev)
    with pytest.raises(PKG.PgmError) as ex:   # rows longer than cap: reported, never written past cap
        PKG.pair_list_noalloc(S.n, pos.data_ptr(), S.box, S.cutoff, 4, sa.data_ptr(), c.data_ptr(), nb.data_ptr())
    assert ex.value.status == -4 and ex.value.max_count > 4
    with pytest.raises(PKG.PgmError, match="16384") as ex:
        PKG.pair_list_noalloc(20000, pos.data_ptr(), S.box, S.cutoff, 4, sa.data_ptr(), c.data_ptr(), nb.data_ptr())
    assert ex.value.status == -4
