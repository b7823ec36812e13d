"""Gauge-field generation helpers: the even-odd site map and periodic tiling (host code),
and a short pure-gauge HMC run on the GPU (update.cpp:280-339 with the o2mn integrator)."""
import numpy as np
import pytest

from yahmc_b200 import thermalize as th


def test_site_map_roundtrip():
    dims = (4, 6, 2, 4)
    c = th.site_coords(dims)
    V = int(np.prod(dims))
    assert c.shape == (V, 4)
    assert np.array_equal(th.site_index(dims, c), np.arange(V))
    p = c.sum(axis=1) & 1
    assert not p[:V // 2].any() and p[V // 2:].all()            # even sites first


def test_site_map_matches_oracle_geometry():
    from oracle import yahmc_oracle as yo
    dims = (4, 4, 6, 2)
    O = yo.Oracle(yo.Params(dims, 2, "fundamental", "periodic", False, True))
    assert np.array_equal(th.site_coords(dims), O.coord)


def test_tile_is_periodic_copy():
    small, big = (4, 2, 2, 4), (4, 4, 6, 8)
    rng = np.random.default_rng(3)
    Vs = int(np.prod(small))
    U = rng.normal(size=(Vs, 4, 2, 2)) + 1j * rng.normal(size=(Vs, 4, 2, 2))
    Ub = th.tile(U, small, big)
    cb = th.site_coords(big)
    cs = th.site_coords(small)
    lookup = {tuple(c): i for i, c in enumerate(cs)}
    for i in range(0, len(cb), 37):
        j = lookup[tuple(cb[i] % np.array(small))]
        assert np.array_equal(Ub[i], U[j])
    with pytest.raises(ValueError):
        th.tile(U, small, (4, 3, 2, 4))


@pytest.mark.gpu
def test_pure_gauge_hmc_short_run():
    import yahmc_b200 as yg
    lat = yg.Lattice((8, 8, 8, 8), nc=3, repr="fundamental", bc="periodic", clover=False, eo=True)
    lat.set_links(np.broadcast_to(np.eye(3, dtype=complex), (lat.V, 4, 3, 3)).copy())
    hist = th.thermalize(lat, 5.6, 12, steps=20, length=1.0, seed=5, n_warm=4)
    plaq = [h[2] for h in hist]
    acc = [h[0] for h in hist[4:]]
    assert plaq[0] < 1.0 and plaq[-1] < plaq[0]
    assert 0.4 < plaq[-1] < 0.7
    assert np.mean(acc) >= 0.5
    assert all(abs(h[1]) < 5.0 for h in hist[4:])
    U = lat.get_links()
    assert np.abs(U @ np.conj(np.swapaxes(U, -1, -2)) - np.eye(3)).max() < 1e-12
