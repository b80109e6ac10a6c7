import numpy as np

from graphics_b200.scene import config_dfsph_1m, config_multiphase_500k, config_wcsph_27k, dam_break


def test_config_counts():
    assert config_wcsph_27k().n_fluid == 27000
    s = config_dfsph_1m()
    assert s.n_fluid == 1_000_000
    assert s.n_boundary > 200_000
    m = config_multiphase_500k()
    assert m.n_fluid == 500_094
    assert set(np.unique(m.phase)) == {0, 1}


def test_seeded_and_jitter_bounds():
    a = dam_break((5, 6, 7), 0.01, (0.2, 0.2, 0.2), seed=3)
    b = dam_break((5, 6, 7), 0.01, (0.2, 0.2, 0.2), seed=3)
    c = dam_break((5, 6, 7), 0.01, (0.2, 0.2, 0.2), seed=4)
    assert np.array_equal(a.fluid_pos, b.fluid_pos)
    assert not np.array_equal(a.fluid_pos, c.fluid_pos)
    lat = dam_break((5, 6, 7), 0.01, (0.2, 0.2, 0.2), jitter=0.0).fluid_pos
    assert np.max(np.abs(a.fluid_pos - lat)) <= 0.1 * 0.01 + 1e-7


def test_walls_enclose_fluid():
    s = dam_break((10, 10, 10), 0.01, (0.4, 0.2, 0.2))
    lo, hi = np.array(s.space_min), np.array(s.space_max)
    for p in (s.fluid_pos, s.boundary_pos):
        assert (p >= lo).all() and (p <= hi).all()
