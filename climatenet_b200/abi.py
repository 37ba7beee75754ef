"""ctypes mirror of include/pdf.h (structs and enums only).

The layout here must match include/pdf.h field for field; tests check the
struct sizes against the C compiler's view through ``pdf_abi_sizes``.
"""
import ctypes as C

PDF_OK = 0
PDF_INVALID_ARG = 1
PDF_CUDA_ERROR = 2
PDF_NOT_SPD = 3
PDF_CAPACITY_EXCEEDED = 4
PDF_DEVICE_TIMEOUT = 5
PDF_NAN_DETECTED = 6
PDF_IO_ERROR = 7
PDF_NO_DEVICE = 8

STATUS_NAMES = {
    0: "PDF_OK", 1: "PDF_INVALID_ARG", 2: "PDF_CUDA_ERROR", 3: "PDF_NOT_SPD",
    4: "PDF_CAPACITY_EXCEEDED", 5: "PDF_DEVICE_TIMEOUT", 6: "PDF_NAN_DETECTED",
    7: "PDF_IO_ERROR", 8: "PDF_NO_DEVICE",
}

PDF_OBSTACLE_SPHERE = 0
PDF_OBSTACLE_ROTATING_SPHERE = 1
PDF_OBSTACLE_PLANE = 2
PDF_OBSTACLE_MESH = 3
PDF_OBSTACLE_BOX = 4
PDF_OBSTACLE_MOVING_MESH = 5

PDF_FP64 = 0
PDF_FP32_REFINE = 1
PDF_WARM_NONE = 0
PDF_WARM_MLP = 1

MLP_IN, MLP_HIDDEN, MLP_OUT = 10, 64, 3
MLP_PARAMS = MLP_HIDDEN * MLP_IN + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN + MLP_OUT * MLP_HIDDEN + MLP_OUT

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class pdf_obstacle(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("material", C.c_int32),
        ("center", C.c_double * 3), ("radius", C.c_double),
        ("axis", C.c_double * 3), ("angular_speed", C.c_double),
        ("rotation_start_time", C.c_double),
        ("point", C.c_double * 3), ("normal", C.c_double * 3),
        ("n_vertices", C.c_int32), ("n_triangles", C.c_int32),
        ("vertices", _dp), ("triangles", _ip), ("threshold", C.c_double),
        ("mesh", C.c_int32), ("size", C.c_double * 3),
        ("n_frames", C.c_int32), ("frame_interval", C.c_double),
    ]


class pdf_mesh_desc(C.Structure):
    _fields_ = [
        ("vertex_offset", C.c_int32), ("n_vertices", C.c_int32),
        ("triangle_offset", C.c_int32), ("n_triangles", C.c_int32),
        ("area_density", C.c_double), ("bending", C.c_double),
        ("stretching", C.c_double), ("material", C.c_int32),
    ]


class pdf_scene_desc(C.Structure):
    _fields_ = [
        ("n_vertices", C.c_int32),
        ("rest_positions", _dp), ("positions", _dp), ("velocities", _dp),
        ("n_triangles", C.c_int32), ("triangles", _ip),
        ("n_meshes", C.c_int32), ("meshes", C.POINTER(pdf_mesh_desc)),
        ("n_pins", C.c_int32), ("pin_vertices", _ip), ("pin_positions", _dp),
        ("pin_weights", _dp),
        ("n_obstacles", C.c_int32), ("obstacles", C.POINTER(pdf_obstacle)),
        ("n_materials", C.c_int32), ("friction", _dp),
    ]


class pdf_params(C.Structure):
    _fields_ = [
        ("time_step", C.c_double), ("local_global_iterations", C.c_int32),
        ("self_collision", C.c_int32), ("self_collision_tolerance", C.c_double),
        ("gravity", C.c_double * 3), ("air_damping", C.c_double),
        ("precision", C.c_int32), ("residual_tolerance", C.c_double),
        ("warm_start", C.c_int32), ("refine_max", C.c_int32),
        ("refine_tolerance", C.c_double), ("device", C.c_int32),
        ("contact_capacity", C.c_int32), ("use_graph", C.c_int32),
        ("mlp_weights", C.c_char * 256),
        ("trace_alart_curnier", C.c_int32),
    ]


PDF_LOG_POSITION = 0
PDF_LOG_VELOCITY = 1


class pdf_log_entry(C.Structure):
    _fields_ = [("kind", C.c_int32), ("n_vertices", C.c_int32), ("vertices", _ip)]


class pdf_step_report(C.Structure):
    _fields_ = [
        ("n_contacts", C.c_int32), ("n_self_contacts", C.c_int32),
        ("n_levels", C.c_int32), ("iterations", C.c_int32),
        ("residual", C.c_double), ("residual_max", C.c_double),
        ("normal_residual", C.c_double), ("tangential_residual", C.c_double),
        ("time", C.c_double), ("refine_sweeps", C.c_int32),
        ("solve_residual", C.c_double), ("device_ms", C.c_double),
    ]


class pdf_stats(C.Structure):
    _fields_ = [
        ("detection_ms", C.c_double), ("self_detection_ms", C.c_double),
        ("ordering_ms", C.c_double), ("rhs_ms", C.c_double),
        ("friction_ms", C.c_double), ("self_friction_ms", C.c_double),
        ("solve_ms", C.c_double), ("step_ms", C.c_double),
        ("steps", C.c_int64), ("iterations", C.c_int64),
        ("setup_ms", C.c_double), ("factor_ms", C.c_double),
        ("factor_nnz", C.c_int64), ("n_supernodes", C.c_int32),
        ("n_levels", C.c_int32), ("lhs_nnz", C.c_int64),
        ("n_constraint_rows", C.c_int32), ("kernel_launches", C.c_int64),
        ("factor_nnz_true", C.c_int64), ("sweep_chunk", C.c_int32),
        ("sweep_chunk_ms", C.c_double * 3),
        ("sweep_cut_level", C.c_int32), ("sweep_blocks", C.c_int32),
        ("sweep_block_elems", C.c_int64), ("sweep_upper_elems", C.c_int64),
        ("sweep_cut_ms", C.c_double * 8),
        ("sweep_upper_mode", C.c_int32), ("sweep_upper_levels", C.c_int32),
        ("sweep_cut_level_ms", C.c_double * 8),
        ("sweep_block_shape", C.c_int32), ("sweep_block_warps", C.c_int32),
        ("sweep_block_ctas", C.c_int32), ("sweep_ring_stages", C.c_int32 * 2),
        ("sweep_shape_ms", C.c_double * 5),
    ]


class pdf_contact(C.Structure):
    _fields_ = [
        ("vertex", C.c_int32), ("partner", C.c_int32), ("face", C.c_int32 * 3),
        ("normal", C.c_double * 3), ("speed", C.c_double * 3),
        ("mu", C.c_double), ("force", C.c_double * 3), ("ac", C.c_double),
    ]


def params(time_step=5e-3, iterations=20, self_collision=False, self_tol=0.0,
           gravity=(0.0, 0.0, -9.81), air_damping=0.0, precision=PDF_FP64,
           residual_tolerance=0.0, warm_start=PDF_WARM_NONE, refine_max=4,
           refine_tolerance=1e-10, device=0, contact_capacity=0, use_graph=1, mlp_weights="",
           trace_alart_curnier=0):
    """Build a pdf_params with the reference's meaning for each field."""
    p = pdf_params()
    p.time_step = time_step
    p.local_global_iterations = iterations
    p.self_collision = 1 if self_collision else 0
    p.self_collision_tolerance = self_tol
    for i in range(3):
        p.gravity[i] = gravity[i]
    p.air_damping = air_damping
    p.precision = precision
    p.residual_tolerance = residual_tolerance
    p.warm_start = warm_start
    p.refine_max = refine_max
    p.refine_tolerance = refine_tolerance
    p.device = device
    p.contact_capacity = contact_capacity
    p.use_graph = use_graph
    p.mlp_weights = mlp_weights.encode() if isinstance(mlp_weights, str) else bytes(mlp_weights)
    p.trace_alart_curnier = trace_alart_curnier
    return p


def contacts_to_numpy(arr, n):
    """Convert n pdf_contact records to a dict of numpy arrays."""
    import numpy as np
    out = {
        "vertex": np.array([arr[i].vertex for i in range(n)], dtype=np.int64),
        "partner": np.array([arr[i].partner for i in range(n)], dtype=np.int64),
        "face": np.array([list(arr[i].face) for i in range(n)], dtype=np.int64).reshape(n, 3),
        "normal": np.array([list(arr[i].normal) for i in range(n)]).reshape(n, 3),
        "speed": np.array([list(arr[i].speed) for i in range(n)]).reshape(n, 3),
        "mu": np.array([arr[i].mu for i in range(n)]),
        "force": np.array([list(arr[i].force) for i in range(n)]).reshape(n, 3),
        "ac": np.array([arr[i].ac for i in range(n)]),
    }
    return out
