"""The oracle's restatement of the seeded particle generator against the
library's own host generator (pic_init_species_host): bit for bit, so the CPU
baselines and the reference arm of the benchmark can build their inputs
without loading the product library."""
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
oracle = importlib.import_module("oracle")
pkg = importlib.import_module("0buf_b200")


@pytest.mark.parametrize("cells,species,ppc,drift,vth,seed", [
    ((6, 5, 4), 0, 7, (0.0, 0.0, 0.0), 0.0, 0),
    ((4, 3, 5), 1, 5, (0.0, 0.0, 0.0), 0.02, 1),
    ((5, 4, 3), 2, 3, (0.2, -0.1, 0.05), 0.002, 12345),
    ((3, 3, 3), 1, 4, (0.0, 0.0, 0.0), 0.1, 2 ** 40 + 7),
])
def test_generator_matches_library(cells, species, ppc, drift, vth, seed):
    lengths = tuple(0.1 * c for c in cells)
    ref = pkg.host_species(cells, lengths, species, ppc, drift, vth, seed)
    for threads in (1, 3):
        got = oracle.gen_species(cells, lengths, species, ppc, drift, vth, seed, threads=threads)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)


def test_init_species_equals_add_particles():
    cells, ppc = (6, 4, 5), 6
    lengths = tuple(0.1 * c for c in cells)
    table = pkg.configs.species_table(ppc)
    a = oracle.OracleSim(cells, lengths, 0.02, threads=3)
    b = oracle.OracleSim(cells, lengths, 0.02)
    for i, s in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
        arrs = oracle.gen_species(cells, lengths, i, ppc, s["drift"], s["vth"], 5)
        assert a.init_species(s["sort"], i, ppc, s["drift"], s["vth"], 5, table[i][1], s["q_m"]) == arrs[0].size
        assert b.add_particles(s["sort"], *arrs, table[i][1], s["q_m"]) == arrs[0].size
    pa, pb = a.particles(), b.particles()
    for k in pa:
        assert np.array_equal(pa[k], pb[k]), k
    for _ in range(2):
        assert a.step() == 0 and b.step() == 0
    assert np.array_equal(a.cell_counts(), b.cell_counts())
    assert np.array_equal(a.get_field("Jx"), b.get_field("Jx"))
    a.close()
    b.close()
