"""ctypes mirror of include/ftb200.h (the C ABI of the forward light tracer).

The structures here must stay byte-identical to the header; tests/test_abi.py checks the
sizes and field offsets against the compiled library.
"""
import ctypes as C

FTB_OK = 0
LAMBDA_SPD = 0
LAMBDA_UNIFORM_380_780 = 1
BUILD_SAH, BUILD_DEVICE = 0, 1
(OK, ERR_INVALID, ERR_NO_DEVICE, ERR_UNSUPPORTED, ERR_CUDA, ERR_OOM, ERR_DEVICE_LIMIT, ERR_TOO_LARGE,
 ERR_TIMEOUT) = range(9)

STATUS_NAMES = {
    0: "FTB_OK", 1: "FTB_ERR_INVALID", 2: "FTB_ERR_NO_DEVICE", 3: "FTB_ERR_UNSUPPORTED",
    4: "FTB_ERR_CUDA", 5: "FTB_ERR_OOM", 6: "FTB_ERR_DEVICE_LIMIT", 7: "FTB_ERR_TOO_LARGE",
    8: "FTB_ERR_TIMEOUT",
}

SPEC_CONST, SPEC_TABLE, SPEC_CAUCHY, SPEC_SELLMEIER, SPEC_BLACKBODY = 0, 1, 2, 3, 4

MAT_DIFFUSE = 0
MAT_DIELECTRIC = 1
MAT_MIRROR = 2
MAT_HALF_MIRROR = 3
MAT_GLOSSY = 4
MAT_DIFFUSE_TRANSMIT = 11
MAT_FILTER = 12

EMIT_QUAD, EMIT_SPHERE = 0, 1
BOUND_NONE, BOUND_BOX, BOUND_SPHERE = 0, 1, 2
PRIORITY_UNSET = -(2 ** 31)

FATE_ABSORBED, FATE_ESCAPED, FATE_RESIDUAL, FATE_SENSOR, FATE_DROPPED = 0, 1, 2, 3, 4

D3 = C.c_double * 3


class Spectrum(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n", C.c_int32), ("offset", C.c_int64),
                ("p", C.c_double * 6)]


class Material(C.Structure):
    _fields_ = [("type", C.c_int32), ("priority", C.c_int32), ("reflect", C.c_int32),
                ("ior", C.c_int32), ("absorb", C.c_int32), ("transmit", C.c_int32),
                ("roughness", C.c_double)]


class Emitter(C.Structure):
    _fields_ = [("shape", C.c_int32), ("collimated", C.c_int32), ("cdf_n", C.c_int32),
                ("spd", C.c_int32), ("cdf_offset", C.c_int64), ("step", C.c_double),
                ("power", C.c_double), ("origin", D3), ("u", D3), ("v", D3),
                ("normal", D3), ("area", C.c_double), ("radius", C.c_double),
                ("beam", D3)]


class Medium(C.Structure):
    _fields_ = [("sigma_a", C.c_int32), ("sigma_s", C.c_int32), ("bound", C.c_int32),
                ("pad0", C.c_int32), ("g", C.c_double), ("bmin", D3), ("bmax", D3),
                ("center", D3), ("radius", C.c_double)]


_PD = C.POINTER(C.c_double)
_PI32 = C.POINTER(C.c_int32)


class BlasDesc(C.Structure):
    _fields_ = [("n_tris", C.c_int64), ("tri_v", _PD), ("tri_n", _PD), ("tri_mat", _PI32),
                ("handle", C.c_void_p)]


class Instance(C.Structure):
    _fields_ = [("blas", C.c_int32), ("mat_override", C.c_int32), ("to_world", C.c_double * 12)]


class SceneDesc(C.Structure):
    _fields_ = [("n_tris", C.c_int64), ("tri_v", _PD), ("tri_n", _PD), ("tri_mat", _PI32),
                ("n_spheres", C.c_int64), ("sph", _PD), ("sph_mat", _PI32),
                ("n_curves", C.c_int64), ("curve", _PD), ("curve_mat", _PI32),
                ("n_mats", C.c_int32), ("n_spectra", C.c_int32),
                ("mats", C.POINTER(Material)), ("spectra", C.POINTER(Spectrum)),
                ("n_table", C.c_int64), ("table_w", _PD), ("table_v", _PD),
                ("n_emitters", C.c_int32), ("n_media", C.c_int32),
                ("emitters", C.POINTER(Emitter)), ("emitter_cdf", _PD),
                ("media", C.POINTER(Medium)), ("n_blas", C.c_int32), ("build", C.c_int32),
                ("blas", C.POINTER(BlasDesc)), ("n_instances", C.c_int64),
                ("instances", C.POINTER(Instance))]


class Camera(C.Structure):
    _fields_ = [("eye", D3), ("u", D3), ("v", D3), ("w", D3), ("tan_half_x", C.c_double),
                ("tan_half_y", C.c_double), ("res_x", C.c_int32), ("res_y", C.c_int32)]


class RenderParams(C.Structure):
    _fields_ = [("n_photons", C.c_int64), ("seed_base", C.c_uint64),
                ("max_bounce", C.c_int32), ("frac_bits", C.c_int32), ("hero_c", C.c_int32),
                ("lambda_mode", C.c_int32)]


class Energy(C.Structure):
    _fields_ = [("emitted", C.c_double), ("absorbed", C.c_double), ("sensor", C.c_double),
                ("escaped", C.c_double), ("residual", C.c_double), ("fx", C.c_int64 * 5)]

    def as_list(self):
        return [self.emitted, self.absorbed, self.sensor, self.escaped, self.residual]


class FilmInfo(C.Structure):
    _fields_ = [("frac_bits", C.c_int32), ("pad0", C.c_int32), ("scale", C.c_double),
                ("power_ref", C.c_double)]


class Footprint(C.Structure):
    _fields_ = [("scene_bytes", C.c_uint64), ("film_bytes", C.c_uint64),
                ("wave_bytes", C.c_uint64), ("total_bytes", C.c_uint64)]


class PhotonLog(C.Structure):
    _fields_ = [("n_hits", C.c_int32), ("fate", C.c_int32), ("prim_hash", C.c_uint64),
                ("beta", C.c_double), ("prims", C.c_int32 * 8)]


class Job(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("cam", Camera), ("d_film", C.c_void_p), ("n_photons", C.c_int64),
                ("seed_base", C.c_uint64), ("max_bounce", C.c_int32), ("frac_bits", C.c_int32),
                ("hero_c", C.c_int32), ("lambda_mode", C.c_int32)]


class KernelProfile(C.Structure):
    _fields_ = [("ms", C.c_double * 4), ("launches", C.c_int64 * 4), ("counters", C.c_uint64 * 8)]


class Tuning(C.Structure):
    _fields_ = [("wave_slots", C.c_int32), ("grid_mult", C.c_int32), ("use_graphs", C.c_int32),
                ("sort_rays", C.c_int32), ("regenerate", C.c_int32)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_active", C.c_int32), ("film_budget", C.c_uint64),
                ("wave_slots", C.c_int32), ("hero_max", C.c_int32), ("hbm_budget", C.c_uint64)]


class Request(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("cam", Camera), ("n_photons", C.c_int64),
                ("seed_base", C.c_uint64), ("max_bounce", C.c_int32), ("frac_bits", C.c_int32),
                ("hero_c", C.c_int32), ("lambda_mode", C.c_int32), ("host_film", C.POINTER(C.c_int64))]


class JobResult(C.Structure):
    _fields_ = [("status", C.c_int), ("pad", C.c_int32), ("info", FilmInfo), ("energy", Energy),
                ("submit_s", C.c_double), ("admit_s", C.c_double), ("finish_s", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
                ("queued", C.c_int64), ("active", C.c_int64), ("photons_done", C.c_int64),
                ("waves", C.c_int64), ("busy_s", C.c_double), ("film_bytes", C.c_uint64),
                ("scene_bytes", C.c_uint64), ("wave_bytes", C.c_uint64), ("evictions", C.c_int64),
                ("restores", C.c_int64)]


STRUCTS = {
    "ftb_spectrum": Spectrum, "ftb_material": Material, "ftb_emitter": Emitter,
    "ftb_medium": Medium, "ftb_scene_desc": SceneDesc, "ftb_camera": Camera,
    "ftb_render_params": RenderParams, "ftb_energy": Energy, "ftb_film_info": FilmInfo,
    "ftb_footprint": Footprint, "ftb_photon_log": PhotonLog,
    "ftb_kernel_profile": KernelProfile, "ftb_job": Job, "ftb_blas_desc": BlasDesc,
    "ftb_instance": Instance, "ftb_server_config": ServerConfig, "ftb_request": Request,
    "ftb_job_result": JobResult, "ftb_server_stats": ServerStats, "ftb_tuning": Tuning,
}

# every entry point declared in include/ftb200.h
EXPORTS = [
    "ftb_last_error", "ftb_abi_version", "ftb_available", "ftb_device_name", "ftb_mem_info",
    "ftb_forward_supported", "ftb_camera_look_at", "ftb_emission_cdf", "ftb_scene_create",
    "ftb_scene_destroy", "ftb_scene_footprint", "ftb_scene_evict", "ftb_scene_restore",
    "ftb_scene_resident", "ftb_scene_power", "ftb_render_forward",
    "ftb_render_forward_device", "ftb_session_begin", "ftb_session_batch",
    "ftb_session_hits0", "ftb_session_download", "ftb_session_end", "ftb_trace_log",
    "ftb_scene_set_profiling", "ftb_scene_profile", "ftb_render_forward_noalloc",
    "ftb_render_batch", "ftb_blas_create", "ftb_blas_destroy", "ftb_scene_set_instance_transforms",
    "ftb_scene_clone_instances", "ftb_server_create", "ftb_server_submit", "ftb_server_wait",
    "ftb_server_get_stats", "ftb_server_destroy", "ftb_get_tuning", "ftb_set_tuning", "ftb_autotune",
]
NOALLOC_MAX_PHOTONS = 32768
NOALLOC_SCRATCH_BYTES = 21062912
