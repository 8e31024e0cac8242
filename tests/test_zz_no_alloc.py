"""cwp_render_noalloc: the frame of cwp_renderer_render without any allocation, for callers that cannot call
cudaMalloc (a plugin whose host application owns the GPU memory budget, a serving loop that must not stall on
cudaMalloc / cudaFree, code that must not fail on an allocation mid-frame). Its scratch is a fixed array inside the
library. Checked through the C ABI against the allocating renderer on the same frame, on two calls in a row (the
array keeps the previous call's contents, so the second call shows that everything that must start at zero does).
This file is collected last so that a failure here stops a -x run only after every other test has run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(torch, cwp, variant, tri, w, h, bounces, spp, batch):
    mesh, bvh = cwp.scene("boxes12k", variant=variant, bins=32)
    p = cwp.frame_params(mesh, w, h, bounces=bounces)
    r = cwp.Renderer(); r.init(p, bvh, variant=variant, tri=tri, batch=batch, bounces=bounces)
    st = r.render(spp)
    want = r.read_accum()
    r.close()
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in (("nodes", bvh.nodes), ("tris", bvh.tris), ("woop", bvh.woop), ("albedo", bvh.albedo.astype(np.float32)))}
    ds = cwp.DeviceScene(dev["nodes"].data_ptr(), dev["tris"].data_ptr(), dev["woop"].data_ptr() if tri else None, None, dev["albedo"].data_ptr())
    o = cwp.RenderOptions(); o.variant, o.tri, o.batch, o.bounces, o.device = variant, tri, batch, bounces, torch.cuda.current_device()
    return p, ds, o, dev, st, want


def _call(cwp, p, ds, o, spp, s_base, clear, accum, rays, stream):
    rc = cwp.lib().cwp_render_noalloc(C.byref(p), C.byref(ds), C.byref(o), spp, s_base, clear, accum.data_ptr(), rays, stream)
    assert rc == cwp.OK, cwp.lib().cwp_last_error()


@pytest.mark.parametrize("variant,tri", [(8, 1), (8, 0), (4, 1), (4, 0), (2, 1), (2, 0)])
def test_noalloc_matches_renderer_twice(gpu, cwp, variant, tri):
    torch = gpu
    w, h, spp, batch, bounces = (128, 96, 8, 4, 4) if (variant, tri) == (8, 1) else (64, 48, 4, 4, 4)   # under the 262,144-path limit
    p, ds, o, dev, st, want = _setup(torch, cwp, variant, tri, w, h, bounces, spp, batch)
    accum = torch.full((w * h, 4), 7.0, dtype=torch.float32, device="cuda")   # garbage: clear = 1 must reset it
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        rays = (C.c_int64 * 2)()
        _call(cwp, p, ds, o, spp, 0, 1, accum, rays, stream)
        got = accum.cpu().numpy()
        assert np.allclose(got, want, rtol=1e-5, atol=1e-6), f"call {call}: max diff {np.abs(got - want).max()}"
        assert rays[0] == st.rays and rays[1] == st.shadow_rays, (call, rays[0], rays[1], st.rays, st.shadow_rays)


def test_noalloc_progressive_matches_one_call(gpu, cwp):
    """Samples [0, 4) with clear = 1, then [4, 8) with clear = 0 and s_base = 4, give the renderer's 8-sample frame."""
    torch = gpu
    p, ds, o, dev, st, want = _setup(torch, cwp, 8, 1, 64, 48, 4, 8, 4)
    accum = torch.zeros((64 * 48, 4), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    r1, r2 = (C.c_int64 * 2)(), (C.c_int64 * 2)()
    _call(cwp, p, ds, o, 4, 0, 1, accum, r1, stream)
    _call(cwp, p, ds, o, 4, 4, 0, accum, r2, stream)
    assert np.allclose(accum.cpu().numpy(), want, rtol=1e-5, atol=1e-6)
    assert r1[0] + r2[0] == st.rays and r1[1] + r2[1] == st.shadow_rays


def test_noalloc_rejects_sizes_beyond_its_limit(gpu, cwp):
    torch = gpu
    mesh, bvh = cwp.scene("boxes12k", variant=2, bins=16)
    p = cwp.frame_params(mesh, 512, 512)
    o = cwp.RenderOptions(); o.variant, o.tri, o.batch, o.bounces, o.device = 2, 1, 2, 4, torch.cuda.current_device()   # 524,288 paths > 262,144
    buf = torch.zeros((512 * 512, 4), dtype=torch.float32, device="cuda")
    ds = cwp.DeviceScene(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), None, buf.data_ptr())
    rc = cwp.lib().cwp_render_noalloc(C.byref(p), C.byref(ds), C.byref(o), 2, 0, 1, buf.data_ptr(), None, None)
    assert rc == cwp.ERR_INVALID and b"no-allocation limit" in cwp.lib().cwp_last_error()
    o.batch = 1; p.max_b = 4; o.bounces = 63                                         # 62 bounces at most
    rc = cwp.lib().cwp_render_noalloc(C.byref(p), C.byref(ds), C.byref(o), 1, 0, 1, buf.data_ptr(), None, None)
    assert rc == cwp.ERR_INVALID and b"bounces 63" in cwp.lib().cwp_last_error()


def test_noalloc_rejects_wrong_device_and_host_memory(gpu, cwp):
    torch = gpu
    mesh, bvh = cwp.scene("boxes12k", variant=2, bins=16)
    p = cwp.frame_params(mesh, 32, 32)
    buf = torch.zeros((32 * 32, 4), dtype=torch.float32, device="cuda")
    ds = cwp.DeviceScene(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), None, buf.data_ptr())
    o = cwp.RenderOptions(); o.variant, o.tri, o.batch, o.bounces = 2, 1, 1, 4
    o.device = torch.cuda.current_device() + 1                                       # not the current device
    rc = cwp.lib().cwp_render_noalloc(C.byref(p), C.byref(ds), C.byref(o), 1, 0, 1, buf.data_ptr(), None, None)
    assert rc == cwp.ERR_INVALID and b"not the current device" in cwp.lib().cwp_last_error()
    o.device = torch.cuda.current_device()
    host = np.zeros((32 * 32, 4), np.float32)                                        # pageable host memory as the accumulation buffer
    rc = cwp.lib().cwp_render_noalloc(C.byref(p), C.byref(ds), C.byref(o), 1, 0, 1, host.ctypes.data, None, None)
    assert rc == cwp.ERR_INVALID and b"accumulation buffer is not device memory" in cwp.lib().cwp_last_error()
    o.sort = 1
    rc = cwp.lib().cwp_render_noalloc(C.byref(p), C.byref(ds), C.byref(o), 1, 0, 1, buf.data_ptr(), None, None)
    assert rc == cwp.ERR_INVALID and b"sort 1" in cwp.lib().cwp_last_error()
