"""rq_kernel_normalize_sp_noalloc: the normalisation for callers that cannot allocate device
memory, checked through the C ABI against rq_kernel_normalize_sp (which allocates its scratch).

Two calls in a row on two different states: the second call must not see the first call's
per-domain sums, which stay in the library's fixed scratch array between calls.  Bar: the same
tolerance as the normalisation parity test (FP64 sums in a different atomic order can move
f32(norm) by one ulp): max |difference| <= 2e-6 * max |psi|.
"""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def states():
    sys.path.insert(0, GOLD)
    from make_golden import seeded_state
    return [(64, 8.0 / 64, seeded_state(64, 12, 11)), (48, 8.0 / 48, seeded_state(48, 30, 12))]


def test_noalloc_normalize_matches_allocating_entry_point_twice():
    import torch
    from realmolecule_b200 import _lib
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    for NN, h, st in states():  # two calls in a row on the shared scratch
        S = NN + 1
        nA = st["atoms5"].size // 5
        h3 = np.float32(h ** 3)
        Z = torch.from_numpy(st["atoms5"].reshape(nA, 5)[:, 3].copy()).cuda()
        L = torch.from_numpy(st["label"]).cuda()
        U_ref = torch.from_numpy(st["U"].copy()).cuda()
        U_new = torch.from_numpy(st["U"].copy()).cuda()
        assert lib.rq_kernel_normalize_sp(U_ref.data_ptr(), L.data_ptr(), Z.data_ptr(), nA, S, h3, None, stream) == 0
        assert lib.rq_kernel_normalize_sp_noalloc(U_new.data_ptr(), L.data_ptr(), Z.data_ptr(), nA, S, h3,
                                                  stream) == 0
        torch.cuda.synchronize()
        a, b = U_new.cpu().numpy(), U_ref.cpu().numpy()
        assert np.max(np.abs(a - b)) <= 2e-6 * np.max(np.abs(b))
        assert not np.array_equal(b, st["U"])  # the normalisation did change psi


def test_noalloc_rejects_too_many_domains_before_launching():
    from realmolecule_b200 import _lib
    lib = _lib.load()
    S = 17
    import torch
    U = torch.zeros(S ** 3, dtype=torch.float32, device="cuda")
    L = torch.zeros(S ** 3, dtype=torch.int32, device="cuda")
    n = _lib.NOALLOC_MAX_DOMAINS + 1
    Z = torch.ones(n, dtype=torch.float32, device="cuda")
    assert lib.rq_kernel_normalize_sp_noalloc(U.data_ptr(), L.data_ptr(), Z.data_ptr(), n, S, 1.0, None) == \
        _lib.RQ_EINVAL
