"""b40c_enact_search_no_alloc: the search for callers that must not allocate.

Frameworks whose own allocator owns all device memory, and latency-bound
loops that cannot pay for the synchronisation an allocation may cause, cannot
let a search call cudaMalloc.  This entry point takes the CSR and the label array from the
caller and takes its scratch from a static 32 MiB device array, so these tests
check that its labels and search depth equal those of the ordinary
Reset + EnactSearch path (expand-contract), bit for bit, over calls in a row
that reuse the shared scratch.  The file runs last so that a failure here
cannot stop the rest of the suite.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest


def _no_alloc(nodes, edges, d_row, d_col, src, d_labels, stream=0):
    from back40computing_b200._lib import lib
    depth = ctypes.c_int(-7)
    rc = lib().b40c_enact_search_no_alloc(nodes, edges, ctypes.c_void_p(d_row), ctypes.c_void_p(d_col), src,
                                          ctypes.c_void_p(d_labels), ctypes.byref(depth), ctypes.c_void_p(stream))
    return rc, depth.value


def _existing(g, src):
    """Labels and search depth from the ordinary path (CsrProblem + expand-contract enactor)."""
    import back40computing_b200 as b
    problem = b.CsrProblem(False).from_graph(g)
    en = b.make_enactor(0)
    b.check(problem.Reset(en.GetFrontierType(), 1.0))
    b.check(en.EnactSearch(problem, int(src)))
    labels = problem.labels()
    _, depth, _ = en.GetStatistics()
    problem.close()
    return labels, depth


class DeviceCsr:
    """The caller's own device copy of a CSR; the column array may start off
    a 16-byte boundary to exercise the scalar-load path."""

    def __init__(self, g, misalign=False):
        import torch
        self.g = g
        self.row = torch.from_numpy(g.row_offsets).cuda()
        pad = 1 if misalign else 0
        self._col = torch.zeros(g.edges + pad + 1, dtype=torch.int32, device="cuda")
        self._col[pad:pad + g.edges] = torch.from_numpy(g.column_indices).cuda()
        self.col_ptr = self._col.data_ptr() + 4 * pad
        self.labels = torch.empty(g.nodes, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()

    def search(self, src):
        import torch
        rc, depth = _no_alloc(self.g.nodes, self.g.edges, self.row.data_ptr(), self.col_ptr, int(src),
                              self.labels.data_ptr(), torch.cuda.current_stream().cuda_stream)
        return rc, depth, self.labels.cpu().numpy()


@pytest.mark.gpu
def test_no_alloc_matches_enact_search_on_calls_in_a_row(cuda_device, oracle):
    import back40computing_b200 as b
    from back40computing_b200._lib import last_error
    big = b.rmat(16, 16, seed=11)
    small = b.grid2d(96)
    cases = [(big, False), (big, False), (small, False), (big, True), (small, True)]
    csrs = {}
    for k, (g, misalign) in enumerate(cases):
        key = (g.name, misalign)
        if key not in csrs:
            csrs[key] = DeviceCsr(g, misalign)
        src = int(g.sample_sources(5, 30 + k)[k])
        rc, depth, labels = csrs[key].search(src)
        assert rc == 0, last_error()
        ref_labels, ref_depth = _existing(g, src)
        assert np.array_equal(labels, ref_labels), (k, g.name, src)
        assert depth == ref_depth, (k, depth, ref_depth)
        alone, _ = oracle.bfs(g, src)
        assert oracle.first_mismatch(labels, alone) == -1


@pytest.mark.gpu
def test_no_alloc_same_source_twice(cuda_device):
    """Two identical calls in a row: the second starts from the first's leftovers."""
    import back40computing_b200 as b
    g = b.rmat(15, 8, seed=5)
    csr = DeviceCsr(g)
    src = int(g.sample_sources(1, 3)[0])
    ref_labels, ref_depth = _existing(g, src)
    for _ in range(2):
        rc, depth, labels = csr.search(src)
        assert rc == 0
        assert np.array_equal(labels, ref_labels) and depth == ref_depth


def test_no_alloc_rejects_graphs_beyond_its_scratch():
    """Sizes are checked before the device is touched, so this runs without a GPU."""
    from back40computing_b200._lib import last_error
    from back40computing_b200.bfs import cudaErrorInvalidValue
    for nodes, edges in ((1 << 22, 1 << 26), (1000, (1 << 31) - 1)):
        rc, _ = _no_alloc(nodes, edges, 0, 0, 0, 0)
        assert rc == cudaErrorInvalidValue
        msg = last_error()
        assert "bytes of scratch" in msg and str(32 << 20) in msg, msg
    rc, _ = _no_alloc(0, 0, 0, 0, 0, 0)
    assert rc == cudaErrorInvalidValue
