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


def test_noalloc_matches_renderer_twice(gpu, cwp):
    torch = gpu
    mesh, bvh = cwp.scene("boxes12k", variant=8, bins=32)
    w, h, spp, batch, bounces = 128, 96, 8, 4, 4          # 49,152 paths per pass, under the 262,144 limit
    p = cwp.frame_params(mesh, w, h, bounces=bounces)
    r = cwp.Renderer(); r.init(p, bvh, variant=8, tri=1, batch=batch, bounces=bounces)
    st = r.render(spp)
    want = r.read_accum()
    r.close()
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in (("nodes", bvh.nodes), ("tris", bvh.tris), ("woop", bvh.woop), ("albedo", bvh.albedo.astype(np.float32)))}
    ds = cwp.DeviceScene(dev["nodes"].data_ptr(), dev["tris"].data_ptr(), dev["woop"].data_ptr(), None, dev["albedo"].data_ptr())
    o = cwp.RenderOptions(); o.variant, o.tri, o.batch, o.bounces = 8, 1, batch, bounces
    accum = torch.full((w * h, 4), 7.0, dtype=torch.float32, device="cuda")   # garbage: clear = 1 must reset it
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        rays = (C.c_int64 * 2)()
        rc = cwp.lib().cwp_render_noalloc(C.byref(p), C.byref(ds), C.byref(o), spp, 0, 1, accum.data_ptr(), rays, stream)
        assert rc == cwp.OK, cwp.lib().cwp_last_error()
        got = accum.cpu().numpy()
        assert np.allclose(got, want, rtol=1e-5, atol=1e-6), f"call {call}: max diff {np.abs(got - want).max()}"
        assert rays[0] == st.rays and rays[1] == st.shadow_rays, (call, rays[0], rays[1], st.rays, st.shadow_rays)


def test_noalloc_rejects_sizes_beyond_its_limit(gpu, cwp):
    torch = gpu
    mesh, bvh = cwp.scene("boxes12k", variant=2, bins=16)
    p = cwp.frame_params(mesh, 512, 512)
    o = cwp.RenderOptions(); o.variant, o.tri, o.batch, o.bounces = 2, 1, 2, 4   # 524,288 paths > 262,144
    buf = torch.zeros((512 * 512, 4), dtype=torch.float32, device="cuda")
    ds = cwp.DeviceScene(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), None, buf.data_ptr())
    rc = cwp.lib().cwp_render_noalloc(C.byref(p), C.byref(ds), C.byref(o), 2, 0, 1, buf.data_ptr(), None, None)
    assert rc == cwp.ERR_INVALID and b"no-allocation limit" in cwp.lib().cwp_last_error()
