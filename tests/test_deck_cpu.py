"""The particle loader's object test runs only on the particles of the cells
that meet each object's bounding box; it must keep exactly the particles
the test over every particle keeps (same random draws, same arithmetic)."""
import numpy as np
import pytest

from pic_b200 import deck


def _load_full(cfg, mesh, species):
    sp, _ = deck.species_params(cfg)
    rng = np.random.default_rng([cfg.seed, species, 7919])
    ncell = cfg.ncx * cfg.ncy
    cell = np.arange(ncell, dtype=np.int64)
    n = ncell * cfg.ppc
    x = (np.repeat(cell // cfg.ncy, cfg.ppc) + rng.random(n)) * mesh.hx
    y = (np.repeat(cell % cfg.ncy, cfg.ppc) + rng.random(n)) * mesh.hy
    keep = np.ones(n, dtype=bool)
    for k in range(mesh.deck.n_objects):
        keep &= ~deck._inside(mesh.deck.objects[k], x, y)
    x, y = x[keep], y[keep]
    v = rng.standard_normal((3, x.size)) * sp[species][3]
    return x, y, v[0], v[1], v[2]


@pytest.mark.parametrize("name,over", [("cfg4", dict(ncx=128, ncy=128, ppc=3)), ("cfg1", dict(ppc=4)),
                                       ("tiny", {})])
def test_bounding_box_loader_matches_full_test(name, over):
    cfg = deck.config(name, **over)
    mesh = deck.Mesh(cfg)
    try:
        for s in range(2):
            a = deck.load_particles(cfg, mesh, s)
            b = _load_full(cfg, mesh, s)
            assert a[0].size < cfg.ncx * cfg.ncy * cfg.ppc  # the objects removed some
            for u, w in zip(a, b):
                assert np.array_equal(u, w)
    finally:
        mesh.close()
