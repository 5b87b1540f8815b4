"""Host loads through the C ABI (pic_load_particles_cells): the load is staged
in chunks of 2^24 particles on a second stream and binned with warp-aggregated
per-tile counters.  A species of 2.5 chunks exported, reloaded and exported
again gives back the same particles, entries with an invalid cell or offset
are dropped (one of them on a chunk boundary), an empty load leaves an
empty species, and the staging that the handle keeps between loads serves
loads of different sizes."""
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


def test_staging_reused_across_loads_of_different_sizes(pkg):
    """The load staging stays with the handle from one load to the next and
    grows when a larger species comes: small, larger (over one chunk), small
    again, and a reload after a step, each exported back unchanged."""
    cells = (160, 64, 64)
    with make(pkg, cells) as a, make(pkg, cells) as b:
        for s, ppc in ((0, 2), (1, 32), (2, 4)):
            a.init_species(s, ppc, (0.0, 0.0, 0.0), 0.02, seed=7 + s)
        src = [export(a, s) for s in range(3)]
        assert src[0][0].size < CHUNK < src[1][0].size
        for s in range(3):
            assert b.load_particles_cells(s, *src[s]) == src[s][0].size
        for s in range(3):
            assert np.array_equal(row_keys(export(b, s)), row_keys(src[s]))
        b.step(1)
        assert b.load_particles_cells(0, *src[0]) == src[0][0].size
        assert np.array_equal(row_keys(export(b, 0)), row_keys(src[0]))
        b.step(2)
        assert b.num_particles() == sum(x[0].size for x in src)
