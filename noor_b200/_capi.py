"""ctypes mirror of include/noor_b200.h (structs and entry points).

The struct field order and types follow the header exactly; the tests check
the sizes against the C compiler's (sizeof) through the library.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
# the in-tree build; NOOR_B200_LIB names another build of the same sources
# (e.g. one compiled with different launch bounds)
LIB_PATH = Path(os.environ.get("NOOR_B200_LIB", str(_HERE / "libnoor_b200.so")))

f32 = C.c_float
u32 = C.c_uint32
i32 = C.c_int32
u64 = C.c_uint64
pf = C.POINTER(C.c_float)
pu = C.POINTER(C.c_uint32)

NOOR_OK = 0
ERRORS = {1: "INVALID", 2: "CUDA", 3: "NO_CONTEXT", 4: "UNSUPPORTED", 5: "OOM", 6: "DEVICE", 7: "CAPACITY"}

NOOR_DIFFUSE = 1 << 0
NOOR_TRANSLUCENT = 1 << 2
NOOR_GLOSSY = 1 << 3
NOOR_MIRROR = 1 << 4
NOOR_GLASS = 1 << 5
NOOR_ROUGHGLASS = 1 << 6
NOOR_METAL = 1 << 7
NOOR_SUBSTRATE = 1 << 8
NOOR_EMITTER = 1 << 9
NOOR_CLEARCOAT = 1 << 10
NOOR_SHADOWCATCHER = 1 << 11
NOOR_ALPHA = 1 << 12
NOOR_BUMP = 1 << 13
NOOR_MESHLIGHT = 1 << 14
NOOR_FILTER_POINT, NOOR_FILTER_LINEAR = 0, 1
NOOR_ADDRESS_WRAP, NOOR_ADDRESS_CLAMP = 0, 1
(NOOR_MAP_DIFFUSE, NOOR_MAP_ROUGHNESS, NOOR_MAP_METALNESS, NOOR_MAP_SPECULAR, NOOR_MAP_EMITTANCE, NOOR_MAP_ALPHA,
 NOOR_MAP_BUMP) = range(7)
NOOR_SKY_HDR, NOOR_SKY_PHYSICAL, NOOR_SKY_CONSTANT = 0, 1, 2
NOOR_LIGHT_SKY_MASK = 0x20
NOOR_ISECT_WATERTIGHT, NOOR_ISECT_REF_WALD = 0, 1
NOOR_FILM_KAHAN, NOOR_FILM_REF_LERP = 0, 1
NOOR_ENV_FP64, NOOR_ENV_REFERENCE = 0, 1
NOOR_SHAPE_QUAD, NOOR_SHAPE_SPHERE, NOOR_SHAPE_DISK = 0, 1, 2
NOOR_CAMERA_PERSP, NOOR_CAMERA_ORTHO, NOOR_CAMERA_ENV = 0, 1, 2
NOOR_TONEMAP_NONE, NOOR_TONEMAP_GAMMA, NOOR_TONEMAP_REINHARD, NOOR_TONEMAP_FILMIC, NOOR_TONEMAP_UNCHARTED2 = -1, 0, 1, 2, 3
NOOR_DEV_STACK_OVERFLOW, NOOR_DEV_QUEUE_OVERFLOW, NOOR_DEV_WAIT_TIMEOUT, NOOR_DEV_BAD_INDEX = 1, 2, 4, 8

TRI_LEAF_MASK = 0x80000000
MESH_LEAF_MASK = 0x40000000
MESH_INSTANCE_MASK = 0x20000000
MESH_INNER_MASK = 0x10000000
LIGHT_NODE_MASK = 0x08000000
NOOR_TRAVERSAL_AUTO, NOOR_TRAVERSAL_BINARY, NOOR_TRAVERSAL_WIDE, NOOR_TRAVERSAL_WIDE_SHADOW = 0, 1, 2, 3


class Shape(C.Structure):
    _fields_ = [("center", f32 * 3), ("u", f32 * 3), ("v", f32 * 3), ("n", f32 * 3), ("area", f32),
                ("radius", f32), ("radius2", f32), ("light_idx", i32), ("type", i32)]


class AreaLight(C.Structure):
    _fields_ = [("shape", Shape), ("ke", f32 * 3), ("two_sided", i32)]


class PointLight(C.Structure):
    _fields_ = [("ke", f32 * 3), ("position", f32 * 3)]


class SpotLight(C.Structure):
    _fields_ = [("ke", f32 * 3), ("position", f32 * 3), ("direction", f32 * 3), ("cos_inner", f32),
                ("cos_outer", f32)]


class DistantLight(C.Structure):
    _fields_ = [("ke", f32 * 3), ("direction", f32 * 3)]


class Texture(C.Structure):
    _fields_ = [("width", i32), ("height", i32), ("rgba", pf), ("filter", i32), ("address", i32)]


class Image(C.Structure):
    _fields_ = [("width", i32), ("height", i32), ("rgba", pf)]


class Material(C.Structure):
    _fields_ = [("diffuse_uvscale", f32 * 2), ("specular_uvscale", f32 * 2), ("transparency_uvscale", f32 * 2),
                ("emittance_uvscale", f32 * 2), ("bump_uvscale", f32 * 2), ("roughness_uvscale", f32 * 2),
                ("metalness_uvscale", f32 * 2), ("diffuse_tex_idx", u32), ("specular_tex_idx", u32),
                ("transmission_tex_idx", u32), ("emittance_tex_idx", u32), ("bump_tex_idx", u32),
                ("transparency_tex_idx", u32), ("ior_tex_idx", u32), ("k_tex_idx", u32), ("roughness_tex_idx", u32),
                ("metalness_tex_idx", u32), ("bumpfactor", f32), ("emitter_scale", f32), ("coat_weight", f32),
                ("coat_roughness", f32), ("coat_thickness", f32), ("coat_sigma", f32), ("coat_ior", f32),
                ("type", u32), ("distribution", u32)]


class Payload(C.Structure):
    _fields_ = [("num_triangles", u32), ("attribute_indices", pu), ("vertices", pf), ("normals", pf), ("uvs", pf),
                ("num_vertices", u32), ("normal_row", pf * 3), ("world_to_object_row", pf * 3),
                ("object_to_world_row", pf * 3), ("num_instances", u32), ("wald_ax_nu_nv_nd", pu),
                ("wald_bnu_bnv_au_av", pu), ("wald_cnu_cnv_deg_mat", pu), ("bvh_root_node", u32),
                ("bvh_min_right_start", pu), ("bvh_max_axis_count", pu), ("num_bvh_nodes", u32),
                ("textures", C.POINTER(Texture)), ("num_textures", u32), ("area_lights", C.POINTER(AreaLight)),
                ("num_area_lights", i32), ("point_lights", C.POINTER(PointLight)), ("num_point_lights", i32),
                ("spot_lights", C.POINTER(SpotLight)), ("num_spot_lights", i32),
                ("distant_lights", C.POINTER(DistantLight)), ("num_distant_lights", i32),
                ("num_infinite_lights", i32), ("materials", C.POINTER(Material)), ("num_materials", u32)]


class Camera(C.Structure):
    _fields_ = [("camera_to_world", (f32 * 4) * 3), ("raster_to_camera", (f32 * 4) * 3),
                ("world_to_raster", (f32 * 4) * 3), ("dx_camera", f32 * 3), ("dy_camera", f32 * 3),
                ("lens_radius", f32), ("focal_length", f32), ("image_area", f32), ("w", u32), ("h", u32),
                ("center", u32), ("type", i32)]


class HosekState(C.Structure):
    _fields_ = [("configs", (f32 * 9) * 3), ("radiances", f32 * 3), ("turbidity", f32), ("solar_radius", f32),
                ("emission_correction_factor_sky", f32 * 3), ("emission_correction_factor_sun", f32 * 3),
                ("albedo", f32), ("elevation", f32)]


class HosekSky(C.Structure):
    _fields_ = [("state", HosekState * 3), ("solar_dir", f32 * 3), ("ground_albedo", f32 * 3),
                ("solar_scale", f32), ("solar_radius", f32)]


class Spec(C.Structure):
    _fields_ = [("reflection_bias", f32), ("shadow_bias", f32), ("world_radius", f32), ("wr2", f32),
                ("bvh_root_node", u32), ("lighting_type", u32), ("bounces", u32), ("rr", u32), ("bvh_height", u32),
                ("num_gpus", u32), ("skydome_type", i32), ("debug_sky", u32), ("mis", u32), ("intersector", u32),
                ("film_mode", u32), ("env_sampling", u32)]


class Ray(C.Structure):
    _fields_ = [("org", f32 * 3), ("tmax", f32), ("dir", f32 * 3), ("pad", f32)]


class Hit(C.Structure):
    _fields_ = [("t", f32), ("tri_idx", u32), ("ins_idx", u32), ("material_type", u32), ("u", f32), ("v", f32),
                ("hit", u32), ("pad", u32)]


class BvhSpec(C.Structure):
    _fields_ = [("num_bins", u32), ("max_height", u32), ("Ci", f32), ("Ct", f32), ("min_leaf_tris", u32),
                ("max_leaf_tris", u32)]


class Mesh(C.Structure):
    _fields_ = [("tri_start", u32), ("tri_count", u32), ("to_global", f32 * 16), ("instance", i32),
                ("light_idx", i32)]


class MaterialDesc(C.Structure):
    _fields_ = [("diffuse", f32 * 3), ("specular", f32 * 3), ("transmission", f32 * 3), ("emittance", f32 * 3),
                ("transparency", f32 * 3), ("ior", f32 * 3), ("k", f32 * 3), ("roughness", f32 * 2),
                ("coat_weight", f32), ("coat_roughness", f32), ("coat_thickness", f32), ("coat_sigma", f32),
                ("coat_ior", f32), ("emitter_scale", f32), ("type", u32), ("distribution", u32),
                ("map", i32 * 7), ("map_uvscale", (f32 * 2) * 7), ("bumpfactor", f32)]


class SceneDesc(C.Structure):
    _fields_ = [("vertices", pf), ("num_vertices", u32), ("normals", pf), ("num_normals", u32), ("uvs", pf),
                ("num_uvs", u32), ("vindices", pu), ("nindices", pu), ("uvindices", pu), ("material_indices", pu),
                ("num_triangles", u32), ("meshes", C.POINTER(Mesh)), ("num_meshes", u32),
                ("materials", C.POINTER(MaterialDesc)), ("num_materials", u32),
                ("area_lights", C.POINTER(AreaLight)), ("num_area_lights", u32),
                ("point_lights", C.POINTER(PointLight)), ("num_point_lights", u32),
                ("spot_lights", C.POINTER(SpotLight)), ("num_spot_lights", u32),
                ("distant_lights", C.POINTER(DistantLight)), ("num_distant_lights", u32), ("skydome_type", i32),
                ("env_width", i32), ("env_height", i32), ("env_rgba", pf), ("bvh", BvhSpec),
                ("images", C.POINTER(Image)), ("num_images", u32)]


class BuildStat(C.Structure):
    _fields_ = [("height", u32), ("num_inner_nodes", u32), ("num_leaf_nodes", u32), ("max_leaf_tris", u32),
                ("scene_min", f32 * 3), ("scene_max", f32 * 3), ("scene_radius", f32), ("build_seconds", C.c_double),
                ("box_seconds", C.c_double), ("tree_seconds", C.c_double), ("tree_device_ms", C.c_double),
                ("tail_seconds", C.c_double), ("tail_device_ms", C.c_double)]


class WfFrame(C.Structure):
    _fields_ = [("scene_id", u32), ("width", u32), ("height", u32), ("spp", u32), ("first_frame", u32),
                ("bounces", u32), ("camera", Camera), ("d_film", pf)]


class WfParams(C.Structure):
    _fields_ = [("block_size", u32), ("queue_capacity", u32), ("sort_granularity", u32), ("use_graph", u32),
                ("max_iterations", u32), ("traversal", u32), ("shade_regs", u32)]


class WfProfile(C.Structure):
    _fields_ = [("ms", f32 * 7), ("launches", u32 * 7), ("iterations", u32)]


class AdjointDesc(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("spp", u32), ("first_frame", u32), ("bounces", u32),
                ("d_albedo", pf), ("d_roughness", pf), ("d_env", pf)]


# name -> (restype, argtypes)
PROTOTYPES = {
    "load_cuda_data": (C.c_int, [C.POINTER(Payload), C.POINTER(HosekSky), C.POINTER(Camera), C.POINTER(Spec),
                                 C.c_void_p]),
    "update_cuda_camera": (C.c_int, []),
    "update_cuda_hosek": (C.c_int, []),
    "update_cuda_spec": (C.c_int, []),
    "cuda_path_tracer": (C.c_int, [C.POINTER(C.c_uint)]),
    "debug_skydome": (C.c_int, [C.POINTER(C.c_uint), C.c_int, C.c_int]),
    "device_free_memory": (C.c_int, []),
    "get_lookAt": (C.c_int, [pf]),
    "noor_last_error": (C.c_char_p, []),
    "noor_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "noor_abi_sizes": (C.c_int, [pu, C.c_int]),
    "noor_build_payload_gpu": (C.c_int, [C.POINTER(SceneDesc), C.POINTER(C.c_void_p), C.POINTER(BuildStat)]),
    "noor_tonemap_device": (C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.c_float, C.c_void_p]),
    "noor_save_image": (C.c_int, [C.c_char_p, C.c_int, C.c_float]),
    "noor_render_frames": (C.c_int, [C.POINTER(C.c_uint), C.c_uint]),
    "noor_get_framebuffer": (C.c_int, [pf, C.c_size_t]),
    "noor_get_framebuffer_device": (C.c_int, [C.c_void_p, C.c_size_t]),
    "noor_reset_film": (C.c_int, []),
    "noor_ray_counters": (C.c_int, [C.POINTER(u64), C.c_int]),
    "noor_device_status": (C.c_int, [pu, C.c_int]),
    "noor_stream": (C.c_void_p, []),
    "noor_event_record": (C.c_int, [C.c_int]),
    "noor_event_elapsed": (C.c_int, [C.c_int, C.c_int, pf]),
    "noor_launch_count": (C.c_int, [C.POINTER(u64)]),
    "noor_trace_closest": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "noor_trace_any": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "noor_camera_rays": (C.c_int, [C.c_uint, C.c_void_p]),
    "noor_eval_bsdf": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_size_t]),
    "noor_eval_routines": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_size_t]),
    "noor_eval_sky": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "noor_eval_env_sample": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t]),
    "noor_get_reference_distribution": (C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int), pf, pf]),
    "noor_get_env_distribution": (C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int), pf, pf, pf, pf,
                                            C.POINTER(C.c_double)]),
    "noor_build_payload": (C.c_int, [C.POINTER(SceneDesc), C.POINTER(C.c_void_p), C.POINTER(BuildStat)]),
    "noor_payload_view": (C.c_int, [C.c_void_p, C.POINTER(Payload)]),
    "noor_payload_triangle_order": (C.c_int, [C.c_void_p, pu, C.c_size_t]),
    "noor_payload_default_spec": (C.c_int, [C.c_void_p, u32, u32, C.POINTER(Spec)]),
    "noor_free_payload": (None, [C.c_void_p]),
    "noor_wide_tree_info": (C.c_int, [C.POINTER(Payload), u32, pu, pu, pu, pu]),
    "noor_camera_lookat": (C.c_int, [pf, pf, pf, f32, u32, u32, C.POINTER(Camera)]),
    "noor_hosek_fit": (C.c_int, [pf, f32, pf, f32, f32, f32, f32, C.POINTER(HosekSky)]),
    "noor_scene_upload": (C.c_int, [C.POINTER(Payload), C.POINTER(HosekSky), C.POINTER(Spec), pu]),
    "noor_wavefront_render": (C.c_int, [C.POINTER(WfFrame), u32, C.POINTER(WfParams)]),
    "noor_wavefront_autotune": (C.c_int, [C.POINTER(WfFrame), u32, C.POINTER(WfParams), pf]),
    "noor_wavefront_render_timed": (C.c_int, [C.POINTER(WfFrame), u32, C.POINTER(WfParams), pf]),
    "noor_wavefront_counters": (C.c_int, [C.POINTER(u64), C.c_int]),
    "noor_wavefront_profile": (C.c_int, [C.POINTER(WfFrame), u32, C.POINTER(WfParams), C.POINTER(WfProfile)]),
    "noor_megakernel_batch": (C.c_int, [C.POINTER(WfFrame), u32, pf]),
    "noor_megakernel_frame_noalloc": (C.c_int, [C.POINTER(WfFrame)]),
    "noor_context_current": (C.c_void_p, []),
    "noor_context_bind": (C.c_int, [C.c_void_p]),
    "noor_adjoint_forward": (C.c_int, [C.POINTER(AdjointDesc), C.c_void_p]),
    "noor_adjoint_backward": (C.c_int, [C.POINTER(AdjointDesc), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
}


ABI_STRUCTS = [Shape, AreaLight, Texture, Material, Payload, Camera, HosekState, HosekSky, Spec, Ray, Hit, BvhSpec,
               Mesh, MaterialDesc, SceneDesc, BuildStat, WfFrame, WfParams, AdjointDesc, WfProfile, PointLight,
               SpotLight, DistantLight]


class NoorError(RuntimeError):
    def __init__(self, fn: str, code: int, msg: str):
        super().__init__(f"{fn} failed: {ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    """Load libnoor_b200.so (built in-tree); raise if it is missing."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run `python noor_b200/build.py` (nvcc, sm_100a)")
        L = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | C.RTLD_GLOBAL)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def call(name: str, *args) -> None:
    """Call an int-returning entry point and raise NoorError on failure."""
    rc = getattr(lib(), name)(*args)
    if rc != NOOR_OK:
        msg = lib().noor_last_error()
        raise NoorError(name, rc, msg.decode() if msg else "")
