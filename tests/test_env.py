"""Environment maps on the host: the library's Radiance RGBE reader and importance-sampling tables, and the oracle's
restatement of the tables, against the reference's own loadHDR and buildEnvMap outputs (tests/golden/env.npz, made by
its code from two files written by the fixture script); the tables as a probability distribution; bad files."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden


@pytest.fixture(scope="module")
def g():
    return golden("env.npz")


@pytest.mark.parametrize("name", ["big", "small"])
def test_hdr_reader_matches_reference(cwp, g, tmp_path, name):
    """run-length (40x20) and flat (6x4) scanlines decode to the reference's radiance bit for bit"""
    path = tmp_path / f"{name}.hdr"
    path.write_bytes(g[f"{name}_hdr"].tobytes())
    rgb = cwp.hdr_load(path)
    assert rgb.shape == g[f"{name}_rgb"].shape
    assert np.array_equal(rgb.view(np.uint32), g[f"{name}_rgb"].view(np.uint32))


@pytest.mark.parametrize("name", ["big", "small"])
def test_tables_match_reference(cwp, oracle, g, name):
    """texels x strength, marginal and conditional CDFs: the library and the oracle give the reference's floats"""
    rgb = g[f"{name}_rgb"]
    for tex, marg, cond in (cwp.envmap_build(rgb, 1.5), oracle.envmap_build(rgb, 1.5)):
        assert np.array_equal(tex.view(np.uint32), g[f"{name}_tex"].view(np.uint32))
        assert np.array_equal(marg.view(np.uint32), g[f"{name}_marg"].view(np.uint32))
        assert np.array_equal(cond.view(np.uint32), g[f"{name}_cond"].view(np.uint32))


def test_tables_are_a_distribution(cwp, g):
    """CDFs run from 0 to 1 without decreasing; texel probabilities (row x column steps) sum to 1; rows without
    luminance get no probability; a sun-disc texel is far likelier than a sky texel (weight luminance x sin(theta))"""
    tex, marg, cond = cwp.envmap_build(g["big_rgb"], 1.5)
    assert marg[0] == 0.0 and marg[-1] == 1.0 and np.all(np.diff(marg) >= 0)
    assert np.all(cond[:, 0] == 0.0) and np.all(cond[:, -1] == 1.0) and np.all(np.diff(cond, axis=1) >= 0)
    p = np.diff(marg.astype(np.float64))[:, None] * np.diff(cond.astype(np.float64), axis=1)
    assert abs(p.sum() - 1.0) < 1e-6
    assert np.all(p[14:16, :3] == 0.0) and np.all(p[14:16, 9:] == 0.0)   # the dark band (the flat block covers columns 3-8)
    yy, xx = np.mgrid[0:20, 0:40]
    sun = ((yy - 5) ** 2 + (xx - 28) ** 2) < 4
    assert p[sun].mean() > 20 * p[~sun & (p > 0)].mean() and p[sun].sum() > 0.4


def test_uniform_rows_when_black(cwp):
    """a black map: uniform CDFs (the reference's fallback), so sampling still covers the sphere"""
    tex, marg, cond = cwp.envmap_build(np.zeros((3, 5, 3), np.float32), 1.0)
    assert np.allclose(marg, np.arange(4) / 3) and np.allclose(cond, np.tile(np.arange(6) / 5, (3, 1)))


def test_bad_files_and_arguments(cwp, g, tmp_path):
    L = cwp.lib(); w, h = C.c_int32(), C.c_int32()
    bad = tmp_path / "bad.hdr"; bad.write_bytes(b"P6\n2 2\n255\n" + bytes(12))
    assert L.cwp_hdr_load(str(bad).encode(), C.byref(w), C.byref(h), None) == cwp.ERR_IO
    assert L.cwp_hdr_load(str(tmp_path / "missing.hdr").encode(), C.byref(w), C.byref(h), None) == cwp.ERR_IO
    cut = tmp_path / "cut.hdr"; cut.write_bytes(g["big_hdr"].tobytes()[:200])
    assert L.cwp_hdr_load(str(cut).encode(), C.byref(w), C.byref(h), None) == 0            # the header alone is fine
    rgb = np.zeros((h.value, w.value, 3), np.float32)
    assert L.cwp_hdr_load(str(cut).encode(), C.byref(w), C.byref(h), rgb.ctypes.data) == cwp.ERR_IO
    other = tmp_path / "xyz.hdr"; other.write_bytes(b"#?RADIANCE\nFORMAT=32-bit_rle_xyze\n\n-Y 1 +X 1\n" + bytes(4))
    assert L.cwp_hdr_load(str(other).encode(), C.byref(w), C.byref(h), None) == cwp.ERR_IO
    with pytest.raises(cwp.CwpError):
        cwp.envmap_build(np.zeros((2, 2, 3), np.float32), -1.0)


def test_oracle_texture_filtering(cwp, oracle):
    """The oracle's texture lookup: a texel centre returns the texel (linear images exactly, sRGB decoded); halfway
    between two texels, their mean; coordinates wrap"""
    img = np.zeros((4, 6, 4), np.uint8)
    img[..., 0] = np.arange(6)[None, :] * 40; img[..., 1] = np.arange(4)[:, None] * 60; img[..., 2] = 200; img[..., 3] = 255
    tex, keep = cwp.textures_array([(img, False), (img, True)])
    # centre of texel (x=2, y=1) at (u, v) with v up: u = 2.5/6, 1 - v = 1.5/4
    uv = np.array([[2.5 / 6, 1 - 1.5 / 4], [3.0 / 6, 1 - 1.5 / 4], [2.5 / 6 + 1, 1 - 1.5 / 4 - 2]], np.float32)
    lin = oracle.texture_sample(tex, [0, 0, 0], uv)
    assert np.allclose(lin[0], img[1, 2] / 255.0, atol=1e-7)
    assert np.allclose(lin[1], (img[1, 2] / 255.0 + img[1, 3] / 255.0) / 2, atol=1e-6)
    assert np.allclose(lin[2], lin[0], atol=1e-7)                           # wrapped
    near, keep2 = cwp.textures_array([(img, False)], nearest=True)
    assert np.allclose(oracle.texture_sample(near, [0], uv[1:2])[0], img[1, 3] / 255.0, atol=1e-7)   # halfway: the texel right of the edge
    srgb = oracle.texture_sample(tex, [1], uv[:1])[0]
    c = img[1, 2, :3] / 255.0
    assert np.allclose(srgb[:3], np.where(c <= 0.04045, c / 12.92, ((c + 0.055) / 1.055) ** 2.4), atol=1e-6) and abs(srgb[3] - 1.0) < 1e-7


def test_planar_uvs(cwp):
    m = cwp.Mesh.box_field(3, 2)
    uvs, tans = cwp.planar_uvs([m])
    assert uvs.shape == (m.n_tris, 8) and tans.shape == (m.n_tris, 12)
    assert np.all(np.isfinite(uvs)) and np.allclose(np.linalg.norm(tans[:, :3], axis=1), 1.0) and set(np.unique(tans[:, 3])) <= {-1.0, 1.0}
