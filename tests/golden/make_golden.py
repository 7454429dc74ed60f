"""Generates tests/golden/*.npz from the reference's own code.

Every label array here is produced by back40computing's SimpleReferenceBfs
(test/bfs/test_bfs.cu:503-578), compiled from the reference sources into
oracle/_ref/libref_bfs.so by oracle/Makefile.  Graphs come from the
reference's builders (grid2d/grid3d/random/rmat, seeded with srand) and from
this package's generators.  Run from the repository root:

    make -C oracle REFERENCE=<reference tree> && python tests/golden/make_golden.py

Each file holds: row_offsets, column_indices, sources, labels (one row per
source), depths (SimpleReferenceBfs search_depth) and a `builder` string.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

from oracle import ReferenceBfs  # noqa: E402

from back40computing_b200 import graphs  # noqa: E402

OUT = Path(__file__).resolve().parent


def save(name, row, col, sources, ref, builder):
    labels, depths = [], []
    g = graphs.CsrGraph(row, col, name)
    for s in sources:
        lab, d = ref.bfs(g, int(s))
        labels.append(lab)
        depths.append(d)
    np.savez_compressed(OUT / f"{name}.npz", row_offsets=row, column_indices=col,
                        sources=np.asarray(sources, np.int32), labels=np.stack(labels).astype(np.int32),
                        depths=np.asarray(depths, np.int32), builder=np.array(builder))
    print(f"{name}: n={g.nodes} m={g.edges} sources={len(sources)} depths={depths}")


def main():
    ref = ReferenceBfs()
    # Reference builders (with their self-loops), reference BFS.
    row, col = ref.grid2d(32)
    save("ref_grid2d_32", row, col, [16 * 32 + 16, 0, 1023], ref, "BuildGrid2dGraph(32)")
    row, col = ref.grid3d(10)
    save("ref_grid3d_10", row, col, [0, 555, 999], ref, "BuildGrid3dGraph(10)")
    row, col = ref.random(2000, 6000, 1, 7)
    save("ref_random_2000_u", row, col, [0, 17, 1999], ref, "srand(7); BuildRandomGraph(2000, 6000, undirected)")
    row, col = ref.random(3000, 9000, 0, 11)
    save("ref_random_3000_d", row, col, [5, 100, 2500], ref, "srand(11); BuildRandomGraph(3000, 9000, directed)")
    row, col = ref.rmat(4096, 40000, 1, 0.57, 0.19, 0.19, 5)
    save("ref_rmat_4096_u", row, col, [1, 2, 77], ref, "srand(5); BuildRmatGraph(4096, 40000, undirected, .57/.19/.19)")
    # This package's generators, reference BFS.
    g = graphs.rmat(12, 16, seed=1)
    save("pkg_rmat_s12", g.row_offsets, g.column_indices, g.sample_sources(4, 2), ref, "graphs.rmat(12, 16, seed=1)")
    g = graphs.erdos_renyi(5000, 16 / 4999, seed=3)
    save("pkg_er_5000", g.row_offsets, g.column_indices, g.sample_sources(3, 2), ref,
         "graphs.erdos_renyi(5000, 16/4999, seed=3)")
    g = graphs.grid2d(48)
    save("pkg_grid2d_48", g.row_offsets, g.column_indices, [24 * 48 + 24, 0], ref, "graphs.grid2d(48)")
    g = graphs.grid3d(12)
    save("pkg_grid3d_12", g.row_offsets, g.column_indices, [0, 12 ** 3 - 1], ref, "graphs.grid3d(12)")


if __name__ == "__main__":
    main()
