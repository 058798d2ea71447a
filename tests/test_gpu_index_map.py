"""Block-cyclic index map on the device (splab_block_cyclic_info) against the
reference's BlockCyclicGenerator::get_block_info, bit for bit (golden fixture
produced from the reference build)."""
import ctypes as ct

import numpy as np
import pytest

import golden_cases as gc

pytestmark = pytest.mark.gpu


def test_block_cyclic_info_matches_reference(spla_lib):
    import torch
    L = spla_lib.lib()
    g = dict(np.load(gc.GOLDEN / "index_map.npz"))
    params, infos = g["params"], g["infos"]
    for pi in np.unique(infos[:, 0]):
        rows = infos[infos[:, 0] == pi]
        rb, cb, gr, gcl, nr, nc, ro, co, _ = (int(v) for v in params[pi])
        ids = torch.from_numpy(np.ascontiguousarray(rows[:, 1])).cuda()
        out = torch.empty(9 * len(rows), dtype=torch.int64, device="cuda")
        rc = L.splab_block_cyclic_info(rb, cb, gr, gcl, nr, nc, ro, co, ids.data_ptr(), len(rows),
                                       out.data_ptr(), None)
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(-1, 9)
        assert np.array_equal(got, rows[:, 2:]), (params[pi])


def test_block_cyclic_info_rejects_bad_grid(spla_lib):
    L = spla_lib.lib()
    assert L.splab_block_cyclic_info(0, 1, 1, 1, 10, 10, 0, 0, None, 1, None, None) == 1
