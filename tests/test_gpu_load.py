"""Host loads through the C ABI (pic_load_particles_cells): the load is staged
in chunks of 2^24 particles on a second stream and binned with warp-aggregated
per-tile counters.  A species of 2.5 chunks exported, reloaded and exported
again gives back the same particles, entries with an invalid cell or offset
are dropped (one of them on a chunk boundary), and an empty load leaves an
empty species."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CHUNK = 1 << 24


def export(sim, s):
    n = sim.num_particles(s)
    out = [np.zeros(n, np.int32)] + [np.zeros(n, np.float32) for _ in range(6)]
    assert sim.get_particles_cells(s, out) == n
    return out


def row_keys(arrs):
    """One 64-bit key per particle from all seven fields, sorted: equal
    multisets of rows give equal key arrays."""
    k = arrs[0].astype(np.uint64)
    for a in arrs[1:]:
        k = k * np.uint64(0x9E3779B97F4A7C15) + a.view(np.uint32).astype(np.uint64)
    return np.sort(k)


def make(pkg, cells):
    return pkg.PicSimulation(cells, tuple(c * 0.1 for c in cells), 0.02, pkg.configs.species_table(32),
                             precision="fp32")


def test_chunked_load_round_trip_and_rejects(pkg):
    cells = (320, 64, 64)  # 32 particles per cell: 41.9M particles = 2.5 chunks
    with make(pkg, cells) as a, make(pkg, cells) as b:
        a.init_species(1, 32, (0.0, 0.0, 0.0), 0.02, seed=5)
        a.run(2)
        src = export(a, 1)
        n = src[0].size
        assert n > 2 * CHUNK
        assert b.load_particles_cells(1, *src) == n
        back = export(b, 1)
        assert np.array_equal(row_keys(back), row_keys(src))
        assert np.array_equal(b.cell_counts(), a.cell_counts())
        # invalid entries: an offset of 1, a ghost cell, a cell past the grid,
        # one at the first index of the second chunk
        bad = [x.copy() for x in src]
        bad[1][0] = 1.0
        bad[0][1] = cells[0] * (cells[1] + 2) * (cells[2] + 2)  # i = nx: a ghost plane
        bad[0][2] = 10 ** 9
        bad[3][CHUNK] = -0.5
        assert b.load_particles_cells(1, *bad) == n - 4
        b.step(1)
        assert b.num_particles(1) == n - 4


def test_empty_load(pkg):
    with make(pkg, (8, 8, 8)) as sim:
        empty = [np.zeros(0, np.int32)] + [np.zeros(0, np.float32) for _ in range(6)]
        assert sim.load_particles_cells(0, *empty) == 0
        sim.init_species(1, 4, (0.0, 0.0, 0.0), 0.01, seed=1)
        sim.step(1)
        assert sim.num_particles(0) == 0 and sim.num_particles(1) == 8 * 8 * 8 * 4
