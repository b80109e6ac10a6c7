"""Reading particle files in the reference's .pos format (read_fluid_particles,
fUtility.h:486-510) through the C ABI; no GPU needed.  The file is built
here byte by byte as the reference's write_fluid_particles
(fUtility.h:254-303) writes it."""
import numpy as np

from graphics_b200.sph import read_pos


def _reference_pos_file(path, recs, components, frame, idx, log="scene.log"):
    mask = "<" + "".join(" %s " % c for c in components) + ">"
    with open(path, "wb") as f:
        f.write(('for parameters and scene info, please refer to "%s"\n' % log).encode())
        f.write(("components writed: %s\n" % mask).encode())
        f.write(("%d (frame number), fluid index: %d\n" % (frame, idx)).encode())
        f.write(("%d (num particles)\n" % len(recs)).encode())
        f.write(np.ascontiguousarray(recs, np.float32).tobytes())
    return mask


def test_read_reference_pos_position_only(tmp_path):
    rng = np.random.default_rng(0)
    x = rng.normal(size=(137, 3)).astype(np.float32)
    mask = _reference_pos_file(tmp_path / "a.pos", x, ["position"], 42, 0)
    data, m, frame = read_pos(tmp_path / "a.pos")
    assert frame == 42 and m == mask
    np.testing.assert_array_equal(data, x)


def test_read_reference_pos_several_components(tmp_path):
    rng = np.random.default_rng(1)
    recs = rng.normal(size=(50, 3 + 3 + 1 + 1)).astype(np.float32)  # position velocity density presure
    _reference_pos_file(tmp_path / "b.pos", recs, ["position", "velocity", "density", "presure"], 7, 1)
    data, m, frame = read_pos(tmp_path / "b.pos")
    assert data.shape == (50, 8) and frame == 7
    np.testing.assert_array_equal(data, recs)


def test_read_empty_pos(tmp_path):
    _reference_pos_file(tmp_path / "c.pos", np.zeros((0, 3)), ["position"], 0, 0)
    data, m, frame = read_pos(tmp_path / "c.pos")
    assert data.shape == (0, 3)
