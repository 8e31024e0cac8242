"""The wavefront renderer on the GPU through the C ABI (cwp_renderer_*) against the oracle's scalar restatement of
the reference's legacy path (same sample streams, same per-vertex decisions) and against the reference's own `pt`
built from its sources (oracle/_ref/pt) on the same scene files."""
import os
import subprocess

import numpy as np
import pytest

from conftest import REF_DIR

pytestmark = pytest.mark.gpu


def render(cwp, mesh, bvh, w, h, spp, batch, variant, tri=1, graph=1, bounces=4, s_base=0):
    p = cwp.frame_params(mesh, w, h, bounces=bounces)
    r = cwp.Renderer()
    r.init(p, bvh, variant=variant, tri=tri, batch=batch, bounces=bounces, graph=graph)
    st = r.render(spp, s_base=s_base)
    return r, p, st, r.read_accum()


@pytest.mark.parametrize("name,variant,bins,spatial", [("boxes12k", 2, 32, 0.0), ("boxes12k", 8, 32, 0.0), ("boxes117k", 8, 128, 1e-3)])
def test_frame_matches_oracle(gpu, cwp, oracle, name, variant, bins, spatial):
    """64x64, 4 spp, depth 4: per-pixel radiance sums agree with the oracle; the only differences come from the order
    of float atomics and ulp-level differences of sin/cos between the GPU and the host's libm (which can change a rare
    path), so the bound is on the image error, stated here: PSNR >= 60 dB in sRGB and >= 99% of the pixels within 1e-4
    relative. Trees: binned SAH on config 1's scene, and the benchmark's SBVH-built CWBVH (128 bins, spatial splits
    at overlap > 1e-3) on config 2's."""
    mesh, bvh = cwp.scene(name, variant=variant, bins=bins, spatial=spatial)
    r, p, st, acc = render(cwp, mesh, bvh, 64, 64, 4, 4, variant)
    ref_acc, counts = oracle.render(p, variant, 1, bvh, 4, 4)
    a = acc[:, :3] / 4; b = ref_acc[:, :3] / 4
    assert cwp.imageio.psnr(a, b) >= 60.0
    rel = np.abs(a - b).max(1) / np.maximum(np.abs(b).max(1), 1e-6)
    assert np.mean(rel <= 1e-4) >= 0.99
    assert abs(st.rays - counts[0]) <= 1e-3 * counts[0] and abs(st.shadow_rays - counts[1]) <= 1e-3 * counts[1]
    assert st.frame_ms > 0 and st.rays >= 64 * 64 * 4


def test_graph_and_host_loop_agree(gpu, cwp):
    mesh, bvh = cwp.scene("boxes12k", variant=8, bins=32)
    _, _, s1, a1 = render(cwp, mesh, bvh, 96, 64, 8, 4, 8, graph=1)
    _, _, s2, a2 = render(cwp, mesh, bvh, 96, 64, 8, 4, 8, graph=0)
    assert s1.rays == s2.rays and s1.shadow_rays == s2.shadow_rays   # every ray's fate is deterministic
    assert np.allclose(a1, a2, rtol=1e-5, atol=1e-6)                  # only the float-atomic order differs


@pytest.mark.parametrize("sort", [1, 2])
def test_regrouped_continuations_render_the_same_frame(gpu, cwp, sort):
    """Regrouping the continuation rays before each bounce only changes the order in which paths are traced: the same
    rays are cast and the image agrees up to the order of float atomics."""
    mesh, bvh = cwp.scene("boxes12k", variant=8, bins=32)
    p = cwp.frame_params(mesh, 96, 64)
    r0 = cwp.Renderer(); r0.init(p, bvh, variant=8, batch=4, bounces=4); s0 = r0.render(8)
    r1 = cwp.Renderer(); r1.init(p, bvh, variant=8, batch=4, bounces=4, sort=sort); s1 = r1.render(8)
    assert s0.rays == s1.rays and s0.shadow_rays == s1.shadow_rays
    assert np.allclose(r0.read_accum(), r1.read_accum(), rtol=1e-5, atol=1e-6)


def test_progressive_accumulation(gpu, cwp):
    """render(8) == render(4, s_base 0) + render(4, s_base 4, clear=False): the sample range is the resume point."""
    mesh, bvh = cwp.scene("boxes12k", variant=2, bins=32)
    p = cwp.frame_params(mesh, 64, 48)
    r = cwp.Renderer(); r.init(p, bvh, variant=2, batch=4, bounces=4)
    r.render(8); full = r.read_accum()
    r.render(4, s_base=0); r.render(4, s_base=4, clear=False); two = r.read_accum()
    assert np.allclose(full, two, rtol=1e-5, atol=1e-6)
    # a different batch size gives the same samples
    r2 = cwp.Renderer(); r2.init(p, bvh, variant=2, batch=2, bounces=4); r2.render(8)
    assert np.allclose(full, r2.read_accum(), rtol=1e-5, atol=1e-6)


def test_layouts_and_triangle_tests_agree(gpu, cwp):
    imgs = []
    for variant in (2, 4, 8):
        for tri in (0, 1):
            mesh, bvh = cwp.scene("boxes12k", variant=variant, bins=32)
            _, _, st, a = render(cwp, mesh, bvh, 64, 64, 4, 4, variant, tri=tri)
            imgs.append(a[:, :3] / 4)
    for x in imgs[1:]:
        assert cwp.imageio.psnr(x, imgs[0]) >= 55.0


def test_renderer_errors(gpu, cwp):
    mesh, bvh = cwp.scene("boxes12k", variant=2, bins=32)
    r = cwp.Renderer()
    with pytest.raises(cwp.CwpError) as e:
        r.render(4)
    assert e.value.code == cwp.ERR_STATE
    p = cwp.frame_params(mesh, 32, 32)
    with pytest.raises(cwp.CwpError):
        r.init(p, bvh, variant=8, batch=4)   # options disagree with the node stride
    r.init(p, bvh, variant=2, batch=4)
    with pytest.raises(cwp.CwpError):
        r.render(6)                          # not a multiple of the batch
    r.render(4)


def test_psnr_vs_reference_pt(gpu, cwp, tmp_path):
    """The reference's own renderer (built from its sources for sm_100) and ours on identical scene files, camera,
    lighting and seed at 256 spp: >= 50 dB in tone-mapped sRGB. The sample streams are the same, but the reference's
    --use_fast_math build rounds directions differently, so paths decorrelate after a bounce or two and the agreement
    is set by Monte Carlo noise (about 38 dB at 16 spp, 55 dB at 256 spp), which is why the bound is taken at 256 spp."""
    pt = os.path.join(REF_DIR, "pt")
    if not os.path.exists(pt):
        pytest.skip("oracle/_ref/pt not built")
    mesh, bvh = cwp.scene("boxes12k", variant=2, bins=16)
    w, h, spp = 256, 256, 256
    p = cwp.frame_params(mesh, w, h)
    args = cwp.reference_inputs(mesh, p, str(tmp_path), w, h, spp, 256)
    out = str(tmp_path / "ref")
    subprocess.run([pt] + args + ["--out", out, "--reps", "1", "--warm", "0"], check=True, capture_output=True, timeout=300)
    ref_img = cwp.imageio.read_pfm(out + ".pfm")
    _, _, st, acc = render(cwp, mesh, bvh, w, h, spp, 256, 2)
    ours = cwp.imageio.accum_to_image(acc, w, h, spp)
    assert cwp.imageio.psnr(ours, ref_img) >= 50.0


def test_display_transform_matches_png_transform(gpu, cwp):
    """cwp_display mode 0 on a rendered accumulation buffer gives the PNG writer's 8-bit sRGB values (host transform
    of sum / spp); the tone-mapped modes stay in range and preserve order."""
    mesh, bvh = cwp.scene("boxes12k", variant=8, bins=32)
    r, p, st, acc = render(cwp, mesh, bvh, 64, 48, 4, 4, 8)
    d_acc = gpu.from_numpy(acc).cuda(); out = gpu.empty((64 * 48, 4), dtype=gpu.uint8, device="cuda")
    cwp.display(d_acc.data_ptr(), out.data_ptr(), 64 * 48, 4, 0.0, 0); gpu.cuda.synchronize()
    got = out.cpu().numpy()
    want = cwp.imageio.tonemap_srgb8(acc[:, :3] / np.float32(4))
    diff = np.abs(got[:, :3].astype(int) - want.astype(int))
    assert diff.max() <= 1 and (diff == 0).mean() >= 0.999 and np.all(got[:, 3] == 255)   # powf may differ by an ulp at a rounding edge
    for mode in (1, 2):
        cwp.display(d_acc.data_ptr(), out.data_ptr(), 64 * 48, 4, 1.0, mode); gpu.cuda.synchronize()
        m = out.cpu().numpy()[:, 0].astype(int); lin = acc[:, 0]
        o = np.argsort(lin)
        assert np.all(np.diff(m[o]) >= -1)


def test_l2_probe(gpu, cwp):
    """The on-chip bandwidth probe (the traversal roofline's denominator) reports more than HBM can deliver and less
    than an implausible figure."""
    g = cwp.measure_l2_read()
    assert 3000.0 < g < 200000.0
