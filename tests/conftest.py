import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def pkg():
    return importlib.import_module("0buf_b200")


@pytest.fixture(scope="session")
def oracle_mod():
    return importlib.import_module("oracle")


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def stress_inputs(pkg, cells, lengths, ppc, seed):
    """The stress configuration's species on a small grid, as
    tests/golden/make_golden.py makes them for ref_stress.npz (the fixture
    pins them by a digest): the host generator thinned to the c4 density
    profile for the profiled species, uniform for the beam.  Returns
    [(sort, [x, y, z, px, py, pz], m, q_m)]."""
    import numpy as np
    counts = pkg.profile_counts(cells, dict(pkg.configs.C4_PROFILE, ppc_mean=ppc)).ravel()
    cmax = int(counts.max())
    table = pkg.configs.species_table(ppc, pkg.configs.SPECIES_STRESS)
    out = []
    for i, s in enumerate(pkg.configs.SPECIES_STRESS):
        if "profile" in s:
            arrs = pkg.host_species(cells, lengths, i, cmax, s["drift"], s["vth"], seed)
            keep = (np.arange(cmax)[None, :] < counts[:, None]).ravel()
            arrs = [a[keep] for a in arrs]
        else:
            arrs = pkg.host_species(cells, lengths, i, ppc, s["drift"], s["vth"], seed)
        out.append((s["sort"], arrs, table[i][1], s["q_m"]))
    return out
