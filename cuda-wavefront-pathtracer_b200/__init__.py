"""B200 wavefront path tracer - Python binding of the C ABI (include/cwp_b200.h, libcwpb200.so).

The classes mirror the reference's C++ interface: ``Mesh`` (scene/mesh.h, io/mesh_loader.h), ``Bvh`` (BVHBuilder +
BVH2Flat / BVH4Flat / CWBVH + packTriangles / packWoop), ``Accel`` (device scene + trav<V,ANY,TRI> over ray batches)
and ``Renderer`` (WavefrontRenderer). Errors raise ``CwpError`` carrying the library's status code and message.
There is no CPU fallback: every compute call goes through the CUDA library, and importing fails loudly when
libcwpb200.so has not been built.
"""
import ctypes as C
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("CWPB_LIB") or os.path.join(_HERE, "libcwpb200.so")   # CWPB_LIB: load another build of the library

OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_STATE, ERR_TRAVERSAL, ERR_IO = range(7)
LAYOUT_BVH2, LAYOUT_BVH4, LAYOUT_CWBVH = 2, 4, 8
TRI_MT, TRI_WOOP = 0, 1
FILTER_TABLE = 64


class CwpError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cwp error {code}: {msg}")
        self.code = code


class MeshView(C.Structure):
    _fields_ = [("verts", C.POINTER(C.c_float)), ("n_verts", C.c_int64), ("faces", C.POINTER(C.c_int32)), ("n_tris", C.c_int64),
                ("face_mat", C.POINTER(C.c_int32)), ("normals", C.POINTER(C.c_float)), ("albedo", C.POINTER(C.c_float)), ("n_albedo", C.c_int32)]


class BuildOptions(C.Structure):
    _fields_ = [("variant", C.c_int32), ("bins", C.c_int32), ("leaf", C.c_int32), ("collapse", C.c_int32), ("threads", C.c_int32), ("spatial", C.c_float),
                ("builder", C.c_int32), ("device", C.c_int32)]


class BvhData(C.Structure):
    _fields_ = [("nodes", C.POINTER(C.c_float)), ("n_node_float4", C.c_int64), ("node_stride", C.c_int32),
                ("order", C.POINTER(C.c_int32)), ("n_tris", C.c_int64), ("tris", C.POINTER(C.c_float)), ("nrm", C.POINTER(C.c_float)),
                ("woop", C.POINTER(C.c_float)), ("max_depth", C.c_int32), ("max_leaf_tris", C.c_int32), ("sah", C.c_double), ("build_ms", C.c_double),
                ("verts", C.POINTER(C.c_float))]


class SceneBuffers(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("n_node_float4", C.c_int64), ("node_stride", C.c_int32), ("tris", C.c_void_p), ("n_tris", C.c_int64),
                ("nrm", C.c_void_p), ("woop", C.c_void_p), ("albedo", C.c_void_p), ("n_albedo", C.c_int32), ("verts", C.c_void_p)]


class Camera(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("ax", C.c_float * 3), ("ay", C.c_float * 3), ("az", C.c_float * 3),
                ("fx", C.c_float), ("fy", C.c_float), ("px", C.c_float), ("py", C.c_float), ("w", C.c_int32), ("h", C.c_int32),
                ("lens_r", C.c_float), ("focus_d", C.c_float)]


class Params(C.Structure):
    _fields_ = [("cam", Camera), ("sun_to", C.c_float * 3), ("sun_e", C.c_float * 3), ("sky", C.c_float * 3), ("sun_cos", C.c_float),
                ("max_b", C.c_int32), ("seed", C.c_uint32), ("eps", C.c_float), ("near_clip", C.c_float), ("has_n", C.c_int32),
                ("filter_bh", C.c_int32), ("ftab", C.c_float * (FILTER_TABLE + 1))]


class RenderOptions(C.Structure):
    _fields_ = [("variant", C.c_int32), ("tri", C.c_int32), ("batch", C.c_int32), ("bounces", C.c_int32), ("graph", C.c_int32),
                ("block", C.c_int32), ("device", C.c_int32), ("profile", C.c_int32), ("traversal", C.c_int32),
                ("sort", C.c_int32), ("stage_levels", C.c_int32), ("reserved", C.c_int32)]


class DeviceScene(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("tris", C.c_void_p), ("woop", C.c_void_p), ("nrm", C.c_void_p), ("albedo", C.c_void_p)]


class FrameStats(C.Structure):
    _fields_ = [("rays", C.c_double), ("shadow_rays", C.c_double), ("trace_ms", C.c_double), ("frame_ms", C.c_double)]


class RendererInfo(C.Structure):
    _fields_ = [("vram_mb", C.c_double), ("tlas_ms", C.c_double), ("pt_blocks", C.c_int32), ("n_sm", C.c_int32), ("gpu_name", C.c_char * 256)]


class Instance(C.Structure):
    _fields_ = [("inv", C.c_float * 12), ("fwd", C.c_float * 12), ("root", C.c_int32), ("mesh", C.c_int32), ("det_sign", C.c_float), ("pad", C.c_int32)]


class InstanceDesc(C.Structure):
    _fields_ = [("mesh", C.c_int32), ("translate", C.c_float * 3), ("translate_per_frame", C.c_float * 3), ("axis", C.c_float * 3),
                ("angle_deg", C.c_float), ("angle_deg_per_frame", C.c_float), ("scale", C.c_float * 3), ("scale_per_frame", C.c_float * 3)]


class BatchOptions(C.Structure):
    _fields_ = [("device", C.c_int32), ("leaf", C.c_int32), ("widths", C.c_int32), ("builder", C.c_int32), ("spatial", C.c_float),
                ("tlas_width", C.c_int32), ("reserved", C.c_int32 * 2)]


class BatchTuning(C.Structure):
    _fields_ = [("block", C.c_int32), ("width", C.c_int32), ("fetch", C.c_int32), ("smem_stack", C.c_int32), ("ms", C.c_float), ("reserved", C.c_int32 * 3)]


class BatchInfo(C.Structure):
    _fields_ = [("n_blas", C.c_int32), ("n_scenes", C.c_int32), ("n_tris", C.c_int64), ("n_instances", C.c_int64), ("node_bytes", C.c_int64 * 3),
                ("blas_build_ms", C.c_double), ("tlas_build_ms", C.c_double), ("blas_hploc_launches", C.c_int32), ("pad", C.c_int32)]


class Material(C.Structure):
    _fields_ = [("base_color", C.c_float * 3), ("metallic", C.c_float), ("specular_color", C.c_float * 3), ("roughness", C.c_float),
                ("emission", C.c_float * 3), ("ior", C.c_float), ("specular_weight", C.c_float), ("transmission", C.c_float), ("pad0", C.c_float), ("pad1", C.c_float)]


class ServerOptions(C.Structure):
    _fields_ = [("max_paths", C.c_int64), ("max_requests", C.c_int32), ("gd_energy", C.c_int32), ("hbm_reserve", C.c_int64), ("device", C.c_int32),
                ("regroup", C.c_int32), ("policy", C.c_int32), ("overlap", C.c_int32), ("reserved", C.c_int32 * 2)]


class Request(C.Structure):
    _fields_ = [("scene", C.c_int32), ("frame", C.c_int32), ("cam", Camera), ("spp", C.c_int32), ("max_depth", C.c_int32), ("seed", C.c_uint32),
                ("sun_to", C.c_float * 3), ("sun_e", C.c_float * 3), ("sky", C.c_float * 3), ("sun_cos", C.c_float), ("eps", C.c_float),
                ("env", C.c_int32), ("env_rot_deg", C.c_float),
                ("light_mode", C.c_int32), ("rr", C.c_int32), ("rr_depth", C.c_int32), ("env_uniform", C.c_int32), ("bump_shadow", C.c_int32),
                ("near_clip", C.c_float), ("filter_bh", C.c_int32)]


LIGHT_MIS, LIGHT_NEE, LIGHT_BSDF = 0, 1, 2


class Texture(C.Structure):
    _fields_ = [("rgba", C.c_void_p), ("w", C.c_int32), ("h", C.c_int32), ("srgb", C.c_int32), ("nearest", C.c_int32)]


class MaterialTextures(C.Structure):
    _fields_ = [("base_color", C.c_int32), ("emission", C.c_int32), ("normal", C.c_int32), ("metallic", C.c_int32), ("roughness", C.c_int32),
                ("metallic_ch", C.c_int32), ("roughness_ch", C.c_int32), ("normal_scale", C.c_float)]


def textures_array(images, nearest=False):
    """(cwp_texture array, the uint8 arrays it points into) from a list of (rgba uint8 [h, w, 4], srgb); nearest: the
    nearest texel instead of bilinear filtering for every image (the reference's --tex_filter nearest)"""
    keep = [np.ascontiguousarray(img[0], np.uint8) for img in images]
    arr = (Texture * max(len(images), 1))()
    for i, (img, spec) in enumerate(zip(keep, images)):
        arr[i].rgba, arr[i].w, arr[i].h, arr[i].srgb = img.ctypes.data, img.shape[1], img.shape[0], 1 if spec[1] else 0
        arr[i].nearest = 1 if nearest else 0
    return arr, keep


def material_textures(bindings):
    """cwp_material_textures array from a list of dicts (keys base_color, emission, normal, metallic, roughness,
    metallic_ch, roughness_ch, normal_scale; missing ids = -1)"""
    arr = (MaterialTextures * max(len(bindings), 1))()
    for i, b in enumerate(bindings):
        for k in ("base_color", "emission", "normal", "metallic", "roughness"):
            setattr(arr[i], k, b.get(k, -1))
        arr[i].metallic_ch, arr[i].roughness_ch, arr[i].normal_scale = b.get("metallic_ch", 2), b.get("roughness_ch", 1), b.get("normal_scale", 1.0)
    return arr


def texture_sample_batch(images, ids, uv, nearest=False):
    """device lookups (texture id, (u, v)) -> rgba float32 [n, 4] with the textures bound as the server binds them"""
    arr, keep = textures_array(images, nearest)
    ids = np.ascontiguousarray(ids, np.int32); uv = np.ascontiguousarray(uv, np.float32); out = np.zeros((len(ids), 4), np.float32)
    _check(lib().cwp_texture_sample_batch(arr, len(images), _iptr(ids), uv.ctypes.data, out.ctypes.data, len(ids)))
    return out


class EnvMap(C.Structure):
    _fields_ = [("rgb", C.c_void_p), ("w", C.c_int32), ("h", C.c_int32), ("strength", C.c_float), ("pad", C.c_int32)]


class RequestStats(C.Structure):
    _fields_ = [("submit_ms", C.c_double), ("admit_ms", C.c_double), ("done_ms", C.c_double), ("rays", C.c_double), ("shadow_rays", C.c_double),
                ("w", C.c_int32), ("h", C.c_int32), ("spp", C.c_int32), ("pad", C.c_int32)]


class ServerInfo(C.Structure):
    _fields_ = [("steps", C.c_int64), ("rays", C.c_int64), ("shadow_rays", C.c_int64), ("admissions", C.c_int64), ("tlas_rebuilds", C.c_int64),
                ("closest_ms", C.c_double), ("shade_ms", C.c_double), ("shadow_ms", C.c_double), ("raygen_ms", C.c_double), ("tlas_ms", C.c_double),
                ("step_ms", C.c_double), ("admit_ms", C.c_double), ("tlas_device_ms", C.c_double),
                ("accum_ms", C.c_double)]


# every exported symbol of the C ABI with its ctypes signature (restype, argtypes)
SIGNATURES = {
    "cwp_last_error": (C.c_char_p, []),
    "cwp_version": (C.c_int32, []),
    "cwp_mesh_box_field": (C.c_int, [C.c_int32, C.c_uint64, C.POINTER(C.c_void_p)]),
    "cwp_mesh_load": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "cwp_mesh_sphere_grid": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "cwp_sphere_grid_c2w": (None, [C.POINTER(C.c_float)]),
    "cwp_mesh_from_view": (C.c_int, [C.POINTER(MeshView), C.POINTER(C.c_void_p)]),
    "cwp_mesh_view_of": (C.c_int, [C.c_void_p, C.POINTER(MeshView)]),
    "cwp_mesh_write_ply": (C.c_int, [C.c_void_p, C.c_char_p]),
    "cwp_mesh_free": (None, [C.c_void_p]),
    "cwp_bvh_build": (C.c_int, [C.c_void_p, C.POINTER(BuildOptions), C.POINTER(C.c_void_p)]),
    "cwp_bvh_data_of": (C.c_int, [C.c_void_p, C.POINTER(BvhData)]),
    "cwp_bvh_free": (None, [C.c_void_p]),
    "cwp_accel_create": (C.c_int, [C.POINTER(SceneBuffers), C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "cwp_accel_destroy": (None, [C.c_void_p]),
    "cwp_trace_closest": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "cwp_trace_any": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "cwp_trace_closest_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_float)]),
    "cwp_trace_any_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_float)]),
    "cwp_accel_status": (C.c_int, [C.c_void_p]),
    "cwp_accel_set_traversal": (C.c_int, [C.c_void_p, C.c_int32]),
    "cwp_accel_set_precision": (C.c_int, [C.c_void_p, C.c_int32]),
    "cwp_trace_fp64": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "cwp_renderer_create": (C.c_int, [C.POINTER(C.c_void_p)]),
    "cwp_renderer_init": (C.c_int, [C.c_void_p, C.POINTER(Params), C.POINTER(SceneBuffers), C.POINTER(RenderOptions)]),
    "cwp_renderer_render": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(FrameStats), C.c_int32, C.c_int32]),
    "cwp_renderer_read_accum": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cwp_renderer_accum_device": (C.c_void_p, [C.c_void_p]),
    "cwp_renderer_set_params": (C.c_int, [C.c_void_p, C.POINTER(Params)]),
    "cwp_renderer_set_materials": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "cwp_renderer_info_of": (C.c_int, [C.c_void_p, C.POINTER(RendererInfo)]),
    "cwp_renderer_depth_stats": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]),
    "cwp_renderer_destroy": (None, [C.c_void_p]),
    "cwp_render_noalloc": (C.c_int, [C.POINTER(Params), C.POINTER(DeviceScene), C.POINTER(RenderOptions), C.c_int32, C.c_int32, C.c_int32,
                                     C.c_void_p, C.c_void_p, C.c_void_p]),
    "cwp_xform_invert": (C.c_int, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "cwp_xform_animate": (C.c_int, [C.POINTER(InstanceDesc), C.c_int32, C.POINTER(C.c_float)]),
    "cwp_instance_from_xform": (C.c_int, [C.POINTER(C.c_float), C.c_int32, C.POINTER(Instance)]),
    "cwp_batch_create": (C.c_int, [C.POINTER(MeshView), C.c_int32, C.POINTER(BatchOptions), C.POINTER(C.c_void_p)]),
    "cwp_batch_destroy": (None, [C.c_void_p]),
    "cwp_batch_set_tlas_width": (C.c_int, [C.c_void_p, C.c_int32]),
    "cwp_server_set_envmaps": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "cwp_server_set_textures": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "cwp_texture_sample_batch": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.c_void_p, C.c_void_p, C.c_int64]),
    "cwp_hdr_load": (C.c_int, [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_void_p]),
    "cwp_envmap_build": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cwp_emissive_tables": (C.c_int, [C.POINTER(MeshView), C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]),
    "cwp_batch_reserve_scenes": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "cwp_batch_update_scenes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "cwp_batch_set_scenes": (C.c_int, [C.c_void_p, C.POINTER(Instance), C.c_int64, C.POINTER(C.c_int32), C.c_int32]),
    "cwp_batch_trace": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "cwp_batch_autotune": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(BatchTuning)]),
    "cwp_batch_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(BatchTuning)]),
    "cwp_batch_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(BatchTuning)]),
    "cwp_batch_info_of": (C.c_int, [C.c_void_p, C.POINTER(BatchInfo)]),
    "cwp_batch_download": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(C.c_int64), C.c_void_p, C.POINTER(C.c_int64)]),
    "cwp_batch_blas_root": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "cwp_batch_download_tlas": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int64), C.c_void_p, C.c_void_p]),
    "cwp_batch_status": (C.c_int, [C.c_void_p]),
    "cwp_server_create": (C.c_int, [C.c_void_p, C.POINTER(Material), C.c_int32, C.POINTER(C.c_int32), C.POINTER(ServerOptions), C.POINTER(C.c_void_p)]),
    "cwp_server_destroy": (None, [C.c_void_p]),
    "cwp_server_set_scenes": (C.c_int, [C.c_void_p, C.POINTER(InstanceDesc), C.c_int64, C.POINTER(C.c_int32), C.c_int32]),
    "cwp_server_set_instance_xforms": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]),
    "cwp_server_submit": (C.c_int, [C.c_void_p, C.POINTER(Request), C.POINTER(C.c_int64)]),
    "cwp_server_step": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "cwp_server_poll": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.c_int32, C.POINTER(C.c_int32)]),
    "cwp_server_result": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.POINTER(RequestStats)]),
    "cwp_server_clock_ms": (C.c_double, [C.c_void_p]),
    "cwp_server_info_of": (C.c_int, [C.c_void_p, C.POINTER(ServerInfo)]),
    "cwp_bsdf_eval_batch": (C.c_int, [C.POINTER(Material), C.c_int32] + [C.c_void_p] * 4 + [C.c_int32] + [C.c_void_p] * 3 + [C.c_int64, C.c_void_p]),
    "cwp_bsdf_sample_batch": (C.c_int, [C.POINTER(Material), C.c_int32] + [C.c_void_p] * 3 + [C.c_int32] + [C.c_void_p] * 6 + [C.c_int64, C.c_void_p]),
    "cwp_display": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_float, C.c_int32, C.c_void_p]),
    "cwp_measure_l2_read": (C.c_int, [C.c_int64, C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
    "cwp_camera_look_at": (C.c_int, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float, C.c_int32, C.c_int32, C.POINTER(Camera)]),
    "cwp_camera_from_c2w": (C.c_int, [C.POINTER(C.c_float), C.c_float, C.c_float, C.c_int32, C.c_int32, C.POINTER(Camera)]),
    "cwp_params_defaults": (C.c_int, [C.POINTER(Params)]),
    "cwp_params_finish": (C.c_int, [C.POINTER(Params), C.c_float, C.c_float, C.c_float]),
}

_lib = None


def lib():
    """The loaded CUDA library; raises if it has not been built (there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is not built: run `make -C {_HERE}` (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _lib = L
    return _lib


def _check(rc):
    if rc != OK:
        raise CwpError(rc, lib().cwp_last_error().decode(errors="replace"))


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


class Mesh:
    """Indexed triangle mesh owned by the library (vertices, faces, material ids, albedo table)."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)

    @classmethod
    def box_field(cls, n_boxes, seed=1):
        h = C.c_void_p()
        _check(lib().cwp_mesh_box_field(n_boxes, seed, C.byref(h)))
        return cls(h.value)

    @classmethod
    def sphere_grid(cls, grid, nu=200, nv=100, ground=200):
        """The reference's synthetic scene (scene/synthetic.cpp:6-48); the defaults are its CLI's (2.0 M tris at 7)."""
        h = C.c_void_p()
        _check(lib().cwp_mesh_sphere_grid(grid, nu, nv, ground, C.byref(h)))
        return cls(h.value)

    @classmethod
    def load(cls, path):
        h = C.c_void_p()
        _check(lib().cwp_mesh_load(str(path).encode(), C.byref(h)))
        return cls(h.value)

    @classmethod
    def from_arrays(cls, verts, faces, face_mat=None, albedo=None, normals=None):
        verts = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        faces = np.ascontiguousarray(faces, np.int32).reshape(-1, 3)
        v = MeshView()
        v.verts, v.n_verts, v.faces, v.n_tris = _fptr(verts), len(verts), _iptr(faces), len(faces)
        keep = [verts, faces]
        if face_mat is not None:
            fm = np.ascontiguousarray(face_mat, np.int32); keep.append(fm); v.face_mat = _iptr(fm)
        if normals is not None:
            nr = np.ascontiguousarray(normals, np.float32); keep.append(nr); v.normals = _fptr(nr)
        if albedo is not None:
            al = np.ascontiguousarray(albedo, np.float32).reshape(-1, 3); keep.append(al); v.albedo = _fptr(al); v.n_albedo = len(al)
        h = C.c_void_p()
        _check(lib().cwp_mesh_from_view(C.byref(v), C.byref(h)))
        return cls(h.value)

    def arrays(self):
        """(verts [n,3] float32, faces [m,3] int32, face_mat [m] int32, albedo [k,3] float32) copies."""
        v = MeshView()
        _check(lib().cwp_mesh_view_of(self._h, C.byref(v)))
        verts = np.ctypeslib.as_array(v.verts, (v.n_verts, 3)).copy()
        faces = np.ctypeslib.as_array(v.faces, (v.n_tris, 3)).copy()
        fm = np.ctypeslib.as_array(v.face_mat, (v.n_tris,)).copy() if v.face_mat else np.zeros(v.n_tris, np.int32)
        alb = np.ctypeslib.as_array(v.albedo, (v.n_albedo, 3)).copy()
        return verts, faces, fm, alb

    @property
    def n_tris(self):
        v = MeshView(); _check(lib().cwp_mesh_view_of(self._h, C.byref(v))); return v.n_tris

    def write_ply(self, path):
        _check(lib().cwp_mesh_write_ply(self._h, str(path).encode()))

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.cwp_mesh_free(self._h); self._h = C.c_void_p()


class Bvh:
    """Host BVH build result: GPU node array, leaf order, packed triangles and Woop rows (numpy copies)."""

    def __init__(self, mesh, variant=LAYOUT_BVH2, bins=16, leaf=4, collapse=0, threads=0, spatial=0.0, builder=0, device=0):
        """builder 0: host binned SAH (spatial splits when spatial > 0); 1: GPU H-PLOC with SAH leaf collapse (the
        reference's --builder hploc; build_ms is then the GPU build time)."""
        o = BuildOptions(variant, bins, leaf, collapse, threads, spatial, builder, device)
        h = C.c_void_p()
        _check(lib().cwp_bvh_build(mesh._h, C.byref(o), C.byref(h)))
        try:
            d = BvhData(); _check(lib().cwp_bvh_data_of(h, C.byref(d)))
            self.variant, self.stride = variant, d.node_stride
            self.nodes = np.ctypeslib.as_array(d.nodes, (d.n_node_float4, 4)).copy()
            self.order = np.ctypeslib.as_array(d.order, (d.n_tris,)).copy()
            self.tris = np.ctypeslib.as_array(d.tris, (d.n_tris * 3, 4)).copy()
            self.woop = np.ctypeslib.as_array(d.woop, (d.n_tris * 3, 4)).copy()
            self.verts = np.ctypeslib.as_array(d.verts, (d.n_tris * 3, 4)).copy()
            self.nrm = np.ctypeslib.as_array(d.nrm, (d.n_tris * 3, 4)).copy() if d.nrm else None
            self.max_depth, self.max_leaf_tris, self.sah, self.build_ms = d.max_depth, d.max_leaf_tris, d.sah, d.build_ms
        finally:
            lib().cwp_bvh_free(h)
        _, _, _, self.albedo = mesh.arrays()

    @property
    def n_nodes(self):
        return len(self.nodes) // self.stride

    def scene_buffers(self):
        """SceneBuffers pointing at this object's arrays (valid while it lives)."""
        s = SceneBuffers()
        s.nodes, s.n_node_float4, s.node_stride = self.nodes.ctypes.data, len(self.nodes), self.stride
        s.tris, s.n_tris = self.tris.ctypes.data, len(self.order)
        s.nrm = self.nrm.ctypes.data if self.nrm is not None else None
        s.woop = self.woop.ctypes.data
        s.verts = self.verts.ctypes.data
        self._alb = np.ascontiguousarray(self.albedo, np.float32)
        s.albedo, s.n_albedo = self._alb.ctypes.data, len(self._alb)
        return s


class Accel:
    """Device copy of a scene for ray batches (closest-hit and any-hit)."""

    def __init__(self, bvh, tri=TRI_WOOP, device=0):
        self._keep = bvh
        h = C.c_void_p()
        s = bvh.scene_buffers()
        _check(lib().cwp_accel_create(C.byref(s), tri, device, C.byref(h)))
        self._h = h

    def trace_closest(self, d_o, d_d, d_hits, n, stream=None):
        """Device pointers (ints, e.g. torch data_ptr()); stream = cudaStream_t as int or None."""
        _check(lib().cwp_trace_closest(self._h, d_o, d_d, d_hits, n, stream))

    def trace_any(self, d_o, d_d, d_occ, n, stream=None):
        _check(lib().cwp_trace_any(self._h, d_o, d_d, d_occ, n, stream))

    def trace_closest_host(self, o, d):
        o = np.ascontiguousarray(o, np.float32); d = np.ascontiguousarray(d, np.float32)
        hits = np.empty((len(o), 4), np.float32); ms = C.c_float()
        _check(lib().cwp_trace_closest_host(self._h, o.ctypes.data, d.ctypes.data, hits.ctypes.data, len(o), C.byref(ms)))
        return hits, ms.value

    def trace_any_host(self, o, d):
        o = np.ascontiguousarray(o, np.float32); d = np.ascontiguousarray(d, np.float32)
        occ = np.empty(len(o), np.int32); ms = C.c_float()
        _check(lib().cwp_trace_any_host(self._h, o.ctypes.data, d.ctypes.data, occ.ctypes.data, len(o), C.byref(ms)))
        return occ, ms.value

    def status(self):
        _check(lib().cwp_accel_status(self._h))

    def set_precision(self, mode):
        """0 plain path, 1 precision form (f16 conservative slabs + watertight FP32 triangles)"""
        _check(lib().cwp_accel_set_precision(self._h, mode))

    def trace_fp64(self, d_o, d_d, d_t, d_tri, n, any_hit=False, stream=None):
        _check(lib().cwp_trace_fp64(self._h, 1 if any_hit else 0, d_o, d_d, d_t, d_tri, n, stream))

    def set_traversal(self, mode):
        """0 auto (persistent refill for BVH2 / CWBVH), 1 refill, 2 one ray per thread"""
        _check(lib().cwp_accel_set_traversal(self._h, mode))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().cwp_accel_destroy(self._h); self._h = C.c_void_p()

    def __del__(self):
        if _lib is not None:
            self.close()


def sphere_grid_c2w():
    """Row-major camera-to-world matrix of the synthetic scene's default view (scene/synthetic.cpp:50)."""
    m = (C.c_float * 16)()
    lib().cwp_sphere_grid_c2w(m)
    return np.array(m[:], np.float32).reshape(4, 4)


def camera_look_at(pos, target, up, hfov_deg, w, h):
    c = Camera()
    f3 = C.c_float * 3
    _check(lib().cwp_camera_look_at(f3(*pos), f3(*target), f3(*up), hfov_deg, w, h, C.byref(c)))
    return c


def params_defaults():
    p = Params()
    _check(lib().cwp_params_defaults(C.byref(p)))
    return p


def params_finish(p, sun_angle_deg, eps_scale, extent):
    _check(lib().cwp_params_finish(C.byref(p), sun_angle_deg, eps_scale, extent))
    return p


class Renderer:
    """WavefrontRenderer: init(params, bvh, options) -> render(spp) -> accum sums (w*h float4)."""

    def __init__(self):
        h = C.c_void_p()
        _check(lib().cwp_renderer_create(C.byref(h)))
        self._h = h

    def init(self, params, bvh, variant, tri=TRI_WOOP, batch=16, bounces=4, graph=1, device=0, profile=0, traversal=0, sort=0, stage_levels=0):
        self._params, self._bvh = params, bvh
        o = RenderOptions(); o.variant, o.tri, o.batch, o.bounces, o.graph, o.device, o.profile = variant, tri, batch, bounces, graph, device, profile
        o.traversal, o.sort, o.stage_levels = traversal, sort, stage_levels
        self.depths = bounces + 2
        s = bvh.scene_buffers()
        _check(lib().cwp_renderer_init(self._h, C.byref(params), C.byref(s), C.byref(o)))
        self.w, self.h = params.cam.w, params.cam.h

    def render(self, spp, s_base=0, clear=True):
        st = FrameStats()
        _check(lib().cwp_renderer_render(self._h, spp, C.byref(st), s_base, 1 if clear else 0))
        return st

    def read_accum(self):
        a = np.empty((self.h * self.w, 4), np.float32)
        _check(lib().cwp_renderer_read_accum(self._h, a.ctypes.data))
        return a

    def accum_device(self):
        return lib().cwp_renderer_accum_device(self._h)

    def set_params(self, p):
        self._params = p
        _check(lib().cwp_renderer_set_params(self._h, C.byref(p)))

    def set_materials(self, albedo):
        a = np.ascontiguousarray(albedo, np.float32).reshape(-1, 3)
        _check(lib().cwp_renderer_set_materials(self._h, a.ctypes.data, len(a)))

    def depth_stats(self):
        """Per-depth (closest rays, shadow rays, trace+shade ms, shadow ms) of the last frame."""
        n = self.depths
        c = np.zeros(n, np.int64); s = np.zeros(n, np.int64); tm = np.zeros(n, np.float32); sm = np.zeros(n, np.float32)
        _check(lib().cwp_renderer_depth_stats(self._h, c.ctypes.data, s.ctypes.data, tm.ctypes.data, sm.ctypes.data, n))
        return c, s, tm, sm

    def info(self):
        i = RendererInfo(); _check(lib().cwp_renderer_info_of(self._h, C.byref(i))); return i

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().cwp_renderer_destroy(self._h); self._h = C.c_void_p()

    def __del__(self):
        if _lib is not None:
            self.close()


def xform_invert(m):
    """FP64 inverse of a 3x4 row-major affine map, rounded to float: (inv [12] float32, det sign)."""
    m = np.ascontiguousarray(m, np.float32).reshape(12)
    inv = np.zeros(12, np.float32); sg = C.c_float()
    _check(lib().cwp_xform_invert(_fptr(m), _fptr(inv), C.byref(sg)))
    return inv, sg.value


def xform_animate(mesh, frame=0, translate=(0, 0, 0), axis=(0, 0, 1), angle_deg=0.0, scale=(1, 1, 1),
                  translate_per_frame=(0, 0, 0), angle_deg_per_frame=0.0, scale_per_frame=(0, 0, 0)):
    """3x4 object -> world map of an animated instance at a frame (translate . rotate(axis, angle) . scale)."""
    d = InstanceDesc(mesh, (C.c_float * 3)(*translate), (C.c_float * 3)(*translate_per_frame), (C.c_float * 3)(*axis), angle_deg,
                     angle_deg_per_frame, (C.c_float * 3)(*scale), (C.c_float * 3)(*scale_per_frame))
    m = np.zeros(12, np.float32)
    _check(lib().cwp_xform_animate(C.byref(d), frame, _fptr(m)))
    return m


def scene_xforms(descs, scene_first, scene, frame):
    """3x4 maps and meshes of one scene's instances at a frame, as the server animates them: (xforms [n, 12], mesh [n])"""
    i0, i1 = int(scene_first[scene]), int(scene_first[scene + 1])
    xf = np.zeros((i1 - i0, 12), np.float32); im = np.zeros(i1 - i0, np.int32)
    for k in range(i0, i1):
        _check(lib().cwp_xform_animate(C.byref(descs[k]), frame, _fptr(xf[k - i0])))
        im[k - i0] = descs[k].mesh
    return xf, im


def instances(xforms, meshes):
    """Array of cwp_instance records (numpy structured bytes, 112 B each) from 3x4 maps and mesh indices."""
    xforms = np.ascontiguousarray(xforms, np.float32).reshape(-1, 12)
    out = (Instance * len(xforms))()
    for i, (m, k) in enumerate(zip(xforms, meshes)):
        _check(lib().cwp_instance_from_xform(_fptr(np.ascontiguousarray(m)), int(k), C.byref(out[i])))
    return out


class Batch:
    """Batched form: many meshes built on the GPU at once (segmented H-PLOC, BVH2 / BVH4 / CWBVH encodings), many
    two-level scenes, one persistent launch over a scene-tagged ray queue, and the launch-shape autotuner."""

    def __init__(self, meshes, device=0, leaf=4, widths=0, builder=0, spatial=0.0, tlas_width=4, normals=None):
        """normals: per mesh, vertex normals [n_verts, 3] or None (the serving integrator's shading normals)"""
        arrs, views = [], (MeshView * len(meshes))()
        for i, m in enumerate(meshes):
            v, f, fm, _ = m.arrays() if isinstance(m, Mesh) else m
            v = np.ascontiguousarray(v, np.float32); f = np.ascontiguousarray(f, np.int32)
            fm = np.ascontiguousarray(fm if fm is not None else np.zeros(len(f)), np.int32)
            arrs += [v, f, fm]
            views[i].verts, views[i].n_verts, views[i].faces, views[i].n_tris, views[i].face_mat = _fptr(v), len(v), _iptr(f), len(f), _iptr(fm)
            if normals is not None and normals[i] is not None:
                nv = np.ascontiguousarray(normals[i], np.float32).reshape(len(v), 3); arrs.append(nv)
                views[i].normals = _fptr(nv)
        o = BatchOptions(device, leaf, widths, builder, spatial, tlas_width)
        h = C.c_void_p()
        _check(lib().cwp_batch_create(views, len(meshes), C.byref(o), C.byref(h)))
        self._h = h; self.tlas_width = tlas_width

    def set_scenes(self, inst, scene_first):
        first = np.ascontiguousarray(scene_first, np.int32)
        _check(lib().cwp_batch_set_scenes(self._h, inst, len(inst), _iptr(first), len(first) - 1))

    def reserve_scenes(self, n_scenes, cap):
        """n_scenes empty scenes with room for cap instances each (the incremental form)"""
        _check(lib().cwp_batch_reserve_scenes(self._h, n_scenes, cap))

    def update_scenes(self, scenes, inst, counts):
        """replace the instances of the listed scenes (inst: their instances in order, counts per scene) and rebuild only
        their TLAS"""
        sc = np.ascontiguousarray(scenes, np.int32); ct = np.ascontiguousarray(counts, np.int32)
        _check(lib().cwp_batch_update_scenes(self._h, _iptr(sc), len(sc), inst if inst is not None and len(inst) else None, _iptr(ct)))

    def trace(self, d_o, d_d, d_scene, d_hits, d_inst, n, any_hit=False, stream=None):
        _check(lib().cwp_batch_trace(self._h, 1 if any_hit else 0, d_o, d_d, d_scene, d_hits, d_inst, n, stream))

    def autotune(self, d_o, d_d, d_scene, d_hits, d_inst, n):
        t = BatchTuning()
        _check(lib().cwp_batch_autotune(self._h, d_o, d_d, d_scene, d_hits, d_inst, n, C.byref(t)))
        return t

    def set_tuning(self, block=128, width=8, fetch=12, smem_stack=0):
        t = BatchTuning(block, width, fetch, smem_stack, 0.0)
        _check(lib().cwp_batch_set_tuning(self._h, C.byref(t)))

    def tuning(self):
        t = BatchTuning(); _check(lib().cwp_batch_get_tuning(self._h, C.byref(t))); return t

    def info(self):
        i = BatchInfo(); _check(lib().cwp_batch_info_of(self._h, C.byref(i))); return i

    def status(self):
        _check(lib().cwp_batch_status(self._h))

    def download(self, width):
        """(nodes [k,4] float32, tris [3n,4] float32) of one layout"""
        nn, nt = C.c_int64(), C.c_int64()
        _check(lib().cwp_batch_download(self._h, width, None, C.byref(nn), None, C.byref(nt)))
        nodes = np.zeros((nn.value, 4), np.float32); tris = np.zeros((nt.value, 4), np.float32)
        _check(lib().cwp_batch_download(self._h, width, nodes.ctypes.data, C.byref(nn), tris.ctypes.data, C.byref(nt)))
        return nodes, tris

    def set_tlas_width(self, width):
        """TLAS form the traversal reads (and download_tlas returns): 2 or 4"""
        _check(lib().cwp_batch_set_tlas_width(self._h, width)); self.tlas_width = width

    def download_tlas(self, n_scenes, n_inst):
        """(tlas nodes [4 n_inst, 4] for width 2 or [8 n_inst, 4] for width 4, scene roots [n_scenes], instances as
        float32 [n_inst, 28])"""
        nn = C.c_int64()
        nodes = np.zeros((8 * max(n_inst, 1), 4), np.float32); roots = np.zeros(n_scenes, np.int32); inst = np.zeros((max(n_inst, 1), 28), np.float32)
        _check(lib().cwp_batch_download_tlas(self._h, nodes.ctypes.data, C.byref(nn), roots.ctypes.data, inst.ctypes.data))
        return nodes[:nn.value], roots, inst[:n_inst]

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.cwp_batch_destroy(self._h); self._h = C.c_void_p()


def display(d_accum, d_rgba, n, spp, exposure_ev=0.0, mode=0, stream=None):
    """Device tone mapping of an accumulation buffer into RGBA8 (mode 0: the PNG transform)."""
    _check(lib().cwp_display(d_accum, d_rgba, n, spp, exposure_ev, mode, stream))


def measure_l2_read(nbytes=32 << 20, reps=50, device=0):
    """On-chip (L2) read bandwidth of the device in GB/s: the denominator of the traversal kernels' roofline."""
    g = C.c_double(); _check(lib().cwp_measure_l2_read(nbytes, reps, device, C.byref(g))); return g.value


def materials_array(m):
    """(Material * n) from a float32 [n, 16] array in the cwp_material layout"""
    m = np.ascontiguousarray(m, np.float32).reshape(-1, 16)
    arr = (Material * len(m))()
    C.memmove(arr, m.ctypes.data, m.nbytes)
    return arr


def bsdf_eval_batch(mats, mat, wo, wi, eta, gd, ux, nr=None):
    """Device BSDF values for (material index, wo, wi) triples in local frames: (f [n, 3], pdf [n]); nr: unperturbed
    normals [n, 3] for the bump-terminator term, or None"""
    M = materials_array(mats); n = len(mat)
    a = [np.ascontiguousarray(x, t) for x, t in ((mat, np.int32), (wo, np.float32), (wi, np.float32), (eta, np.float32), (ux, np.float32))]
    nr = np.ascontiguousarray(nr, np.float32) if nr is not None else None
    f = np.zeros((n, 3), np.float32); pdf = np.zeros(n, np.float32)
    _check(lib().cwp_bsdf_eval_batch(M, len(M), a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, a[3].ctypes.data, gd, a[4].ctypes.data,
                                     f.ctypes.data, pdf.ctypes.data, n, nr.ctypes.data if nr is not None else None))
    return f, pdf


def bsdf_sample_batch(mats, mat, wo, eta, gd, ux, uvw, nr=None):
    """Device BSDF samples: (wi [n, 3], weight [n, 3], pdf [n], ok [n])."""
    M = materials_array(mats); n = len(mat)
    a = [np.ascontiguousarray(x, t) for x, t in ((mat, np.int32), (wo, np.float32), (eta, np.float32), (ux, np.float32), (uvw, np.float32))]
    nr = np.ascontiguousarray(nr, np.float32) if nr is not None else None
    wi = np.zeros((n, 3), np.float32); w = np.zeros((n, 3), np.float32); pdf = np.zeros(n, np.float32); ok = np.zeros(n, np.int32)
    _check(lib().cwp_bsdf_sample_batch(M, len(M), a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, gd, a[3].ctypes.data, a[4].ctypes.data,
                                       wi.ctypes.data, w.ctypes.data, pdf.ctypes.data, ok.ctypes.data, n, nr.ctypes.data if nr is not None else None))
    return wi, w, pdf, ok


def hdr_load(path):
    """Radiance .hdr file -> float32 [h, w, 3] linear radiance, row 0 = top"""
    w, h = C.c_int32(), C.c_int32()
    _check(lib().cwp_hdr_load(str(path).encode(), C.byref(w), C.byref(h), None))
    rgb = np.zeros((h.value, w.value, 3), np.float32)
    _check(lib().cwp_hdr_load(str(path).encode(), C.byref(w), C.byref(h), rgb.ctypes.data))
    return rgb


def envmap_build(rgb, strength=1.0):
    """Importance-sampling tables of an equirectangular map: (texels [h, w, 4], marg [h + 1], cond [h, w + 1])"""
    rgb = np.ascontiguousarray(rgb, np.float32); h, w = rgb.shape[:2]
    tex = np.zeros((h, w, 4), np.float32); marg = np.zeros(h + 1, np.float32); cond = np.zeros((h, w + 1), np.float32)
    _check(lib().cwp_envmap_build(rgb.ctypes.data, w, h, strength, tex.ctypes.data, marg.ctypes.data, cond.ctypes.data))
    return tex, marg, cond


def make_request(scene, cam, spp, frame=0, max_depth=8, seed=1, sun_to=None, sun_e=None, sky=None, sun_angle_rad=None, eps=1e-3, env=-1, env_rot_deg=0.0,
                 light_mode=LIGHT_MIS, rr=0, rr_depth=3, env_uniform=0, bump_shadow=0, near_clip=0.0, filter_bh=0):
    """A serving request; lighting defaults to the benchmark's sun and sky (env = -1) or names one of the server's
    environment maps; emissive materials of the scene are light-sampled too (light_mode, as the reference's
    --light_sampling mis / nee / bsdf); rr / rr_depth: Russian roulette (--rr, --rr_depth)."""
    from . import workloads as W
    sun_to = W.SUN_TO if sun_to is None else sun_to; sun_e = (W.SUN_E,) * 3 if sun_e is None else sun_e
    sky = W.SKY if sky is None else sky; sun_angle_rad = W.SUN_ANGLE_RAD if sun_angle_rad is None else sun_angle_rad
    r = Request()
    r.scene, r.frame, r.cam, r.spp, r.max_depth, r.seed = scene, frame, cam, spp, max_depth, seed
    s = np.array(sun_to, np.float64); s /= np.linalg.norm(s)
    r.sun_to[:] = tuple(float(x) for x in s); r.sun_e[:] = tuple(sun_e); r.sky[:] = tuple(sky)
    r.sun_cos = float(np.float32(math.cos(sun_angle_rad / 2.0))); r.eps = eps
    r.env, r.env_rot_deg = env, env_rot_deg
    r.light_mode, r.rr, r.rr_depth, r.env_uniform, r.bump_shadow = light_mode, rr, rr_depth, env_uniform, bump_shadow
    r.near_clip, r.filter_bh = near_clip, filter_bh
    return r


def emissive_tables(meshes, mesh_mat_base, materials, xforms, inst_mesh):
    """Light tables of the emissive triangles of an instanced scene at one frame (what the server builds at admission):
    (em_tris [n, 12] float32 = world (w0, global id bits), (w1 - w0, material bits), (w2 - w0, 0); em_cdf [n + 1];
    mat_pdf [n_mats]). meshes: (verts, faces, face_mat, _) tuples or Mesh; xforms: [n_inst, 12] 3x4 rows."""
    arrs, views = [], (MeshView * len(meshes))()
    for i, m in enumerate(meshes):
        v, f, fm, _ = m.arrays() if isinstance(m, Mesh) else m
        v = np.ascontiguousarray(v, np.float32); f = np.ascontiguousarray(f, np.int32)
        fm = np.ascontiguousarray(fm if fm is not None else np.zeros(len(f)), np.int32)
        arrs += [v, f, fm]
        views[i].verts, views[i].n_verts, views[i].faces, views[i].n_tris, views[i].face_mat = _fptr(v), len(v), _iptr(f), len(f), _iptr(fm)
    M = materials_array(materials); base = np.ascontiguousarray(mesh_mat_base, np.int32)
    xf = np.ascontiguousarray(xforms, np.float32).reshape(-1, 12); im = np.ascontiguousarray(inst_mesh, np.int32)
    n = C.c_int64()
    args = (views, len(meshes), base.ctypes.data, C.cast(M, C.c_void_p), len(M), xf.ctypes.data, im.ctypes.data, len(im))
    _check(lib().cwp_emissive_tables(*args, None, None, None, C.byref(n)))
    t = np.zeros((n.value, 12), np.float32); c = np.zeros(n.value + 1, np.float32); p = np.zeros(len(M), np.float32)
    _check(lib().cwp_emissive_tables(*args, t.ctypes.data, c.ctypes.data, p.ctypes.data, C.byref(n)))
    return t, (c if n.value else np.zeros(0, np.float32)), p


class Server:
    """Serving form: requests over the resident scenes of a Batch, continuous batching (max_requests > 1) or the plain
    form (max_requests = 1)."""

    def __init__(self, batch, materials, mesh_mat_base, max_paths=8 << 20, max_requests=64, gd_energy=1, hbm_reserve=1 << 30, device=0,
                 regroup=True, policy=0, overlap=True):
        self._batch = batch
        M = materials_array(materials); base = np.ascontiguousarray(mesh_mat_base, np.int32)
        o = ServerOptions(max_paths, max_requests, gd_energy, hbm_reserve, device, 1 if regroup else -1, policy, 1 if overlap else -1)
        h = C.c_void_p()
        _check(lib().cwp_server_create(batch._h, M, len(M), _iptr(base), C.byref(o), C.byref(h)))
        self._h = h

    def set_textures(self, images, bindings, uvs, tans=None, nearest=False):
        """images: list of (rgba uint8 [h, w, 4], srgb); bindings: cwp_material_textures array (material_textures);
        uvs: float32 [n_tris, 8] over all batch meshes in mesh order; tans: float32 [n_tris, 12] or None; nearest: the
        nearest texel instead of bilinear filtering"""
        arr, keep = textures_array(images, nearest)
        uvs = np.ascontiguousarray(uvs, np.float32)
        tans = np.ascontiguousarray(tans, np.float32) if tans is not None else None
        _check(lib().cwp_server_set_textures(self._h, arr, len(images), bindings, len(bindings), uvs.ctypes.data,
                                             tans.ctypes.data if tans is not None else None))

    def set_envmaps(self, maps):
        """maps: list of (rgb float32 [h, w, 3], strength); requests name them by index (Request.env)"""
        keep = [np.ascontiguousarray(rgb, np.float32) for rgb, _ in maps]
        arr = (EnvMap * max(len(maps), 1))()
        for i, (rgb, (_, strength)) in enumerate(zip(keep, maps)):
            arr[i].rgb, arr[i].w, arr[i].h, arr[i].strength = rgb.ctypes.data, rgb.shape[1], rgb.shape[0], strength
        _check(lib().cwp_server_set_envmaps(self._h, arr, len(maps)))

    def set_scenes(self, descs, scene_first):
        first = np.ascontiguousarray(scene_first, np.int32)
        _check(lib().cwp_server_set_scenes(self._h, descs, len(descs), _iptr(first), len(first) - 1))

    def set_instance_xforms(self, per_desc):
        """per descriptor: a [k, 12] array of 3x4 matrices by frame (the last held), or None for its animation
        parameters; None clears them"""
        if per_desc is None:
            _check(lib().cwp_server_set_instance_xforms(self._h, None, None, None, 0)); return
        first, count, rows = [], [], []
        for x in per_desc:
            x = np.zeros((0, 12), np.float32) if x is None else np.asarray(x, np.float32).reshape(-1, 12)
            first.append(sum(len(r) for r in rows)); count.append(len(x)); rows.append(x)
        xf = np.ascontiguousarray(np.concatenate(rows) if rows else np.zeros((0, 12), np.float32))
        f = np.array(first, np.int32); c = np.array(count, np.int32)
        _check(lib().cwp_server_set_instance_xforms(self._h, xf.ctypes.data if len(xf) else None, f.ctypes.data, c.ctypes.data, len(per_desc)))

    def submit(self, req):
        i = C.c_int64(); _check(lib().cwp_server_submit(self._h, C.byref(req), C.byref(i))); return i.value

    def step(self):
        a, p = C.c_int32(), C.c_int32()
        _check(lib().cwp_server_step(self._h, C.byref(a), C.byref(p)))
        return a.value, p.value

    def poll(self, cap=1024):
        ids = (C.c_int64 * cap)(); n = C.c_int32()
        _check(lib().cwp_server_poll(self._h, ids, cap, C.byref(n)))
        return list(ids[:n.value])

    def result(self, rid, w=None, h=None):
        """(accum [w h, 4] radiance sums or None when w is None, RequestStats); releases the request"""
        st = RequestStats()
        acc = np.zeros((w * h, 4), np.float32) if w else None
        _check(lib().cwp_server_result(self._h, rid, acc.ctypes.data if acc is not None else None, C.byref(st)))
        return acc, st

    def clock_ms(self):
        return lib().cwp_server_clock_ms(self._h)

    def info(self):
        i = ServerInfo(); _check(lib().cwp_server_info_of(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in ServerInfo._fields_}

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value and _lib is not None:
            _lib.cwp_server_destroy(self._h); self._h = C.c_void_p()


from . import imageio  # noqa: E402,F401
from .workloads import *  # noqa: E402,F401,F403  (scene / camera / lighting presets of the benchmark configs)
