"""The allocation-free entry point, trisk_weighted_sum_noalloc.

It serves callers that cannot let the library allocate device memory: hosts whose device
memory all comes from their own pool (the Julia side, through CUDA.jl), or code that runs
while a stream is being captured into a CUDA graph. They pass their own device vectors and
the library's static scratch array holds the partial sums.

This file is collected last so that a run that stops at the first failure has run every
other test first. The check: the same total mass as the model's own diagnostics entry
point (trisk_diagnostics), within the 1e-12 relative tolerance of the other parity tests,
on two calls in a row that reuse the static scratch.
"""
import numpy as np
import pytest

import dmplex_b200 as d
from dmplex_b200._lib import check, lib
from conftest import tc2_state, trisk_grid

pytestmark = pytest.mark.gpu


def test_weighted_sum_noalloc_matches_total_mass(require_gpu):
    import torch

    g = trisk_grid(6, True)
    m = d.TRiSKShallowWater(g)
    areas = torch.from_numpy(g.cell_areas.copy()).cuda()
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for seed in (1, 2):  # two calls in a row share the static scratch
        y = tc2_state(g)
        y[g.ne:] += 0.05 * np.random.default_rng(seed).standard_normal(g.nc)
        h = torch.from_numpy(y[g.ne:].copy()).cuda()
        check(lib.trisk_weighted_sum_noalloc(areas.data_ptr(), h.data_ptr(), g.nc, out.data_ptr(), stream))
        torch.cuda.synchronize()
        want = d.total_mass(m, y)
        assert abs(out.item() - want) <= 1e-12 * abs(want)


def test_weighted_sum_noalloc_rejects_oversize(require_gpu):
    import torch

    a = torch.zeros(4, dtype=torch.float64, device="cuda")
    with pytest.raises(d.TriskError) as e:
        check(lib.trisk_weighted_sum_noalloc(a.data_ptr(), a.data_ptr(), 16777217, a.data_ptr(), None))
    assert e.value.status == 1 and "exceeds the maximum" in str(e.value)
