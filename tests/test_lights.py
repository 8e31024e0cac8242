"""Emissive triangles as area lights of instanced scenes, on the host: the library's light tables (what the server
builds at admission) against the oracle's restatement of the reference's SceneSetup::frameData bit for bit, a case
worked by hand, the tables as a probability distribution (power CDF, uniform area density per material), and bad
arguments."""
import numpy as np
import pytest


def _quad(z=0.0, fm=0):
    v = np.array([[0, 0, z], [1, 0, z], [1, 1, z], [0, 1, z]], np.float32)
    f = np.array([[0, 1, 2], [0, 2, 3]], np.int32)
    return (v, f, np.full(2, fm, np.int32), None)


def _mat(emission=(0, 0, 0)):
    m = np.zeros(16, np.float32)
    m[0:3] = 0.5; m[4:7] = 1.0; m[7] = 0.5; m[8:11] = emission; m[11] = 1.5; m[12] = 1.0
    return m


def emissive_scene(cwp, seed=2, frame=5, scene=1):
    """the serving scenes with every mesh's material 1 emissive (coloured), one scene's instances at one frame"""
    meshes, descs, first, mats, base, boxes = cwp.serving_scenes(n_scenes=3, seed=seed, tris=(200, 3000), instances=(2, 24), blas_per_scene=(1, 3))
    mats = mats.copy()
    for b in base:
        mats[b + 1, 8:11] = (4.0, 3.0, 2.0)
    xf, im = cwp.scene_xforms(descs, first, scene, frame)
    return meshes, base, mats, xf, im


def test_tables_match_oracle(cwp, oracle):
    meshes, base, mats, xf, im = emissive_scene(cwp)
    t, c, p = cwp.emissive_tables(meshes, base, mats, xf, im)
    to, co, po = oracle.emissive_tables(meshes, base, mats, xf, im)
    assert len(t) > 0
    for a, b in ((t, to), (c, co), (p, po)):
        assert a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_hand_worked_case(cwp):
    """two unit quads (white emission, luminance 1; the second mesh red, luminance 0.2126 x 2) under three instances:
    identity, scaled by 2 (four times the area), and the red quad moved; powers 0.5, 0.5, 2, 2, 0.2126, 0.2126"""
    meshes = [_quad(fm=0), _quad(fm=0)]
    mats = np.stack([_mat((1, 1, 1)), _mat((2, 0, 0)), _mat()])
    base = np.array([0, 1], np.int32)
    I = np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], np.float32)
    S2 = np.array([2, 0, 0, 1, 0, 2, 0, 0, 0, 0, 2, 3], np.float32)
    T = np.array([1, 0, 0, 5, 0, 1, 0, 0, 0, 0, 1, 0], np.float32)
    t, c, p = cwp.emissive_tables(meshes, base, mats, [I, S2, T], [0, 0, 1])
    assert len(t) == 6
    pw = np.array([0.5, 0.5, 2.0, 2.0, 0.2126 * 2 * 0.5, 0.2126 * 2 * 0.5])
    tot = pw.sum()
    assert np.allclose(c, np.concatenate([[0], np.cumsum(pw) / tot]), atol=1e-6) and c[-1] == 1.0
    assert np.allclose(p, [1.0 / tot, np.float32(0.2126) * 2 / tot, 0.0], rtol=1e-6)
    # records: world corner, edges, global triangle id (mesh 1's first triangle is 2) and material
    assert np.allclose(t[2, 0:3], [1, 0, 3]) and np.allclose(t[2, 4:7], [2, 0, 0]) and np.allclose(t[2, 8:11], [2, 2, 0])
    assert list(t[:, 3].view(np.int32)) == [0, 1, 0, 1, 2, 3] and list(t[:, 7].view(np.int32)) == [0, 0, 0, 0, 1, 1]


def test_tables_are_a_distribution(cwp):
    """P(triangle) = CDF step = luminance x area / total power, so P / area is the material's area density"""
    meshes, base, mats, xf, im = emissive_scene(cwp, seed=4, frame=9, scene=2)
    t, c, p = cwp.emissive_tables(meshes, base, mats, xf, im)
    assert c[0] == 0.0 and c[-1] == 1.0 and np.all(np.diff(c) >= 0)
    area = 0.5 * np.linalg.norm(np.cross(t[:, 4:7].astype(np.float64), t[:, 8:11].astype(np.float64)), axis=1)
    mat = t[:, 7].view(np.int32)
    step = np.diff(c.astype(np.float64))
    ok = area > 1e-3
    assert np.allclose(step[ok] / area[ok], p[mat[ok]], rtol=1e-3)
    lum = 0.2126 * mats[:, 8] + 0.7152 * mats[:, 9] + 0.0722 * mats[:, 10]
    assert np.allclose(p[lum > 0] / lum[lum > 0], p[lum > 0][0] / lum[lum > 0][0], rtol=1e-6) and np.all(p[lum <= 0] == 0)


def test_no_emitters(cwp, oracle):
    meshes = [_quad(), _quad(1.0)]
    mats = np.stack([_mat(), _mat()])
    I = np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], np.float32)
    t, c, p = cwp.emissive_tables(meshes, [0, 1], mats, [I, I], [0, 1])
    assert len(t) == 0 and len(c) == 0 and np.all(p == 0)
    # emissive, but without area (degenerate instance scale): no light tables either
    mats[0, 8:11] = 1.0
    Z = np.zeros(12, np.float32)
    t, c, p = cwp.emissive_tables(meshes, [0, 1], mats, [Z], [0])
    to, co, po = oracle.emissive_tables(meshes, [0, 1], mats, [Z], [0])
    assert len(t) == len(to) == 0 and np.all(p == 0) and np.all(po == 0)


def test_bad_arguments(cwp):
    meshes = [_quad()]
    mats = np.stack([_mat((1, 1, 1))])
    I = np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], np.float32)
    with pytest.raises(cwp.CwpError):
        cwp.emissive_tables(meshes, [0], mats, [I], [1])          # no mesh 1
    with pytest.raises(cwp.CwpError):
        bad = (np.zeros((4, 3), np.float32), np.array([[0, 1, 7]], np.int32), None, None)
        cwp.emissive_tables([bad], [0], mats, [I], [0])         # vertex index out of range


def test_request_light_options_reach_the_abi(cwp):
    cam = cwp.camera_look_at((0, -5, 2), (0, 0, 0), (0, 0, 1), 0.8, 32, 32)
    r = cwp.make_request(0, cam, 2, light_mode=cwp.LIGHT_NEE, rr=1, rr_depth=2, env_uniform=1)
    assert (r.light_mode, r.rr, r.rr_depth, r.env_uniform) == (1, 1, 2, 1)
    import ctypes as C
    assert C.sizeof(r) == C.sizeof(cwp.Request) and cwp.Request.light_mode.offset == cwp.Request.env_rot_deg.offset + 4
