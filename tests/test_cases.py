"""Synthetic case generators (CPU): the urban DEM's built fraction and block heights, and
the lake-at-rest start raster of the urban case (h + z equal to the level wherever water
stands, as the files are written)."""
import numpy as np

import cases


def test_urban_surface_blocks():
    n = 1 << 10
    base = cases.fbm_surface(n, 0.8, 11, 3.0)
    z = cases.urban_surface(n, 11)
    add = z - base
    built = add > 0
    assert 0.25 <= built.mean() <= 0.35
    assert add[built].min() >= 5.0 and add[built].max() <= 20.0
    np.testing.assert_array_equal(z, cases.urban_surface(n, 11))


def test_urban_catchment_files(tmp_path):
    c = cases.urban_catchment(str(tmp_path), L=7, sim_time=10.0, lake_level=1.0)
    par = open(c.par).read()
    for kw in ("max_ref_lvl   7", "DEMfile       case.dem", "startfile     case.start", "bcifile       case.bci"):
        assert kw in par

    def read(name):
        with open(tmp_path / name) as fp:
            head = [next(fp) for _ in range(6)]
            assert head[0].split()[1] == "128"
            return np.loadtxt(fp)[::-1]

    z, h = read("case.dem"), read("case.start")
    wet = h > 0
    assert 0.0 < wet.mean() < 1.0
    np.testing.assert_allclose((h + z)[wet], 1.0, atol=1e-12)
    assert (z[~wet] >= 1.0 - 1e-12).all()
