"""The benchmark frame (117,002-triangle box field, 512 x 512, 256 spp, depth 4) rendered by the reference's own CUDA
build (oracle/_ref/pt, compiled from its sources for sm_100 with its own flags) and by this library on the same B200:
images agree at >= 50 dB PSNR in tone-mapped sRGB, and both frame rates are recorded (printed, and written as JSON to
$CWP_RESULTS_DIR/vs_reference_cuda.json when that variable is set)."""
import json
import os
import subprocess

import pytest

from conftest import REF_DIR

pytestmark = pytest.mark.gpu


def run_ref_pt(cwp, mesh, p, tmp, w, h, spp, batch, variant, reps=2):
    pt = os.path.join(REF_DIR, "pt")
    args = cwp.reference_inputs(mesh, p, str(tmp), w, h, spp, batch, variant=variant)
    out = str(tmp / f"ref_{variant}")
    res = subprocess.run([pt] + args + ["--out", out, "--reps", str(reps)], check=True, capture_output=True, text=True, timeout=600)
    lines = [json.loads(l) for l in res.stdout.splitlines() if l.startswith("{")]
    return lines, cwp.imageio.read_pfm(out + ".pfm")


@pytest.mark.parametrize("w,h", [(512, 512)])
def test_benchmark_frame_vs_reference_cuda(gpu, cwp, tmp_path, w, h):
    if not os.path.exists(os.path.join(REF_DIR, "pt")):
        pytest.skip("oracle/_ref/pt not built")
    spp, batch = 256, 256
    mesh, bvh16 = cwp.scene("boxes117k", variant=2, bins=16)
    p = cwp.frame_params(mesh, w, h)
    record = {"scene": "boxes117k", "w": w, "h": h, "spp": spp, "batch": batch}
    ref_img = None
    for rv in ("bvh2", "bvh8"):
        lines, img = run_ref_pt(cwp, mesh, p, tmp_path, w, h, spp, batch, rv)
        ref_img = img if ref_img is None else ref_img
        best = min(lines, key=lambda l: l["t_frame_ms"])
        record[f"reference_{rv}"] = {k: best[k] for k in ("t_frame_ms", "rays_total", "rays_closest", "rays_shadow", "mrays_s_e2e", "gpu")}
    for variant, bins in ((2, 16), (8, 32), (2, 32)):
        _, bvh = cwp.scene("boxes117k", variant=variant, bins=bins)
        r = cwp.Renderer(); r.init(p, bvh, variant=variant, batch=batch, bounces=4)
        r.render(spp)   # warm-up (graph capture)
        times = []
        for _ in range(3):
            st = r.render(spp); times.append(st.frame_ms)
        img = cwp.imageio.accum_to_image(r.read_accum(), w, h, spp)
        db = cwp.imageio.psnr(img, ref_img)
        record[f"ours_v{variant}_b{bins}"] = {"t_frame_ms": min(times), "rays_total": st.rays + st.shadow_rays, "psnr_vs_reference_db": db,
                                               "grays_s": (st.rays + st.shadow_rays) / min(times) / 1e6}
        r.close()
        assert db >= 50.0, (variant, bins, db)
    ref_best = min(record["reference_bvh2"]["t_frame_ms"], record["reference_bvh8"]["t_frame_ms"])
    ours_best = min(v["t_frame_ms"] for k, v in record.items() if k.startswith("ours_"))
    record["speedup_vs_reference_best"] = ref_best / ours_best
    print(json.dumps(record))
    d = os.environ.get("CWP_RESULTS_DIR")
    if d:
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, "vs_reference_cuda.json"), "w") as f:
            json.dump(record, f, indent=1)
