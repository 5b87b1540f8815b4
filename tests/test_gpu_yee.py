"""pic_step in the FP32 form against the same step taken through the
reference-facing sub-step calls (pic_b_half, pic_push_deposit, pic_migrate,
pic_j_fold, pic_b_complete, pic_e_update, pic_e_ghosts), on a grid whose z
extent leaves a partial tile.  Without particles the current is exactly zero
and the two paths must agree bit for bit in both ghost modes; with particles
the FP64 current is summed across tiles in no fixed order, so they agree to
FP32 rounding."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SUBSTEPS = ("b_half", "stage_fields", "push_deposit", "migrate", "j_fold", "b_complete", "e_update", "e_ghosts")
FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
CELLS = (24, 12, 20)  # z extent 20 over tiles of 12: a partial tile


def make(pkg, ghosts, ppc=0):
    table = pkg.configs.species_table(max(ppc, 1))
    return pkg.PicSimulation(CELLS, tuple(c * 0.1 for c in CELLS), 0.02, table, precision="fp32", ghosts=ghosts)


def random_fields(pkg, sims, seed):
    rng = np.random.default_rng(seed)
    nodes = int(np.prod([c + 2 for c in CELLS]))
    for f in FIELDS:
        a = rng.normal(0.0, 1e-3, nodes)
        for s in sims:
            s.set_field(f, a)


@pytest.mark.parametrize("ghosts", ["reference", "periodic"])
def test_step_matches_substeps_bitwise(pkg, ghosts):
    with make(pkg, ghosts) as a, make(pkg, ghosts) as b:
        random_fields(pkg, (a, b), 3)
        for st in range(1, 4):
            a.step(st)
            for sub in SUBSTEPS:
                b.substep(sub)
            for f in FIELDS + ("Jx", "Jy", "Jz"):
                assert np.array_equal(a.get_field(f), b.get_field(f)), (st, f)


def test_step_matches_substeps_with_particles(pkg):
    with make(pkg, "reference", 8) as a, make(pkg, "reference", 8) as b:
        for sim in (a, b):
            for i, s in enumerate(pkg.configs.SPECIES_BEAM_PLASMA):
                sim.init_species(i, 8, s["drift"], s["vth"], seed=21 + i)
        random_fields(pkg, (a, b), 4)
        for st in range(1, 6):
            a.step(st)
            for sub in SUBSTEPS:
                b.substep(sub)
        assert np.array_equal(a.cell_counts(), b.cell_counts())
        for f in FIELDS:
            x, y = a.get_field(f), b.get_field(f)
            assert np.max(np.abs(x - y)) <= 1e-5 * np.max(np.abs(y)), f
