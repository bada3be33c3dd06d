"""ctypes binding of libins2d.so (include/ins2d.h).

Loading fails loudly: there is no CPU fallback for the hot path.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# INS2D_LIBRARY selects another build of the library (launch-shape variants)
LIB_PATH = os.environ.get("INS2D_LIBRARY") or os.path.join(HERE, "libins2d.so")

OK, EINVAL, ENOTCONV, EBREAKDOWN, ENONFINITE, ETIMEOUT, ECUDA, ENOMEM = range(8)
STATUS_NAMES = {0: "OK", 1: "EINVAL", 2: "ENOTCONV", 3: "EBREAKDOWN", 4: "ENONFINITE",
                5: "ETIMEOUT", 6: "ECUDA", 7: "ENOMEM"}
BC_CODES = {"dir": 0, "pres": 1, "per": 2, "sym": 3}
MEM_HOST, MEM_DEVICE = 0, 1
PREC_FP64, PREC_FP32_STENCIL = 0, 1
PRECOND_CODES = {"default": 0, "jacobi": 1, "mg": 2, "fdm": 3}
MAX_STAGES = 8

# every symbol include/ins2d.h declares
EXPORTED = [
    "ins2d_ctx_create", "ins2d_ctx_destroy", "ins2d_last_error", "ins2d_get_sizes",
    "ins2d_set_stream", "ins2d_wait_stream", "ins2d_set_poll_limit", "ins2d_set_bc_values", "ins2d_set_bc_sampler", "ins2d_F",
    "ins2d_divergence", "ins2d_laplacian", "ins2d_pressure_poisson",
    "ins2d_pressure_additional_solve", "ins2d_erk_step", "ins2d_erk_run", "ins2d_conservation", "ins2d_initial_projection",
    "ins2d_profile", "ins2d_profile_read", "ins2d_fft_poisson_noalloc",
    "ins2d_ens_create", "ins2d_ens_destroy", "ins2d_ens_last_error", "ins2d_ens_size", "ins2d_ens_member",
    "ins2d_ens_set_stream", "ins2d_ens_wait_stream", "ins2d_ens_set_state", "ins2d_ens_get_state", "ins2d_ens_state_ptr", "ins2d_ens_set_member_dt",
    "ins2d_ens_erk_run", "ins2d_ens_set_solver", "ins2d_ens_solve_shape",
    "ins2d_cnn_create", "ins2d_cnn_destroy", "ins2d_cnn_last_error", "ins2d_cnn_set_stream", "ins2d_cnn_set_path",
    "ins2d_cnn_get_params", "ins2d_cnn_set_params", "ins2d_cnn_get_activations", "ins2d_cnn_forward", "ins2d_cnn_loss_grad",
    "ins2d_cnn_train_step", "ins2d_cnn_loss_grad_residual", "ins2d_cnn_train_step_residual", "ins2d_cnn_prepare_pairs", "ins2d_set_learned_guess", "ins2d_set_learned_mode", "ins2d_record_pairs",
    "ins2d_recorded_pairs", "ins2d_learned_train",
    "ins2d_slab_fft_create", "ins2d_slab_fft_destroy", "ins2d_slab_fft_last_error", "ins2d_slab_fft_rows_forward",
    "ins2d_slab_fft_columns", "ins2d_slab_fft_rows_inverse",
]
CNN_NPARAM = 37440
CNN_PATH_TCGEN05, CNN_PATH_MMA_SYNC = 0, 1
PROF_FAMILIES = ["stage", "div", "poisson", "project", "residual", "other"]

c_double_p = ctypes.POINTER(ctypes.c_double)


class GridDesc(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int32), ("Ny", ctypes.c_int32), ("x", c_double_p), ("y", c_double_p)]


class BcDesc(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("u_left", "u_right", "u_low", "u_up", "v_left", "v_right",
                                               "v_low", "v_up", "bc_unsteady")]


class Opts(ctypes.Structure):
    _fields_ = [("Re", ctypes.c_double), ("poisson", ctypes.c_int32), ("CG_acc", ctypes.c_double),
                ("CG_maxit", ctypes.c_int32), ("p_add_solve", ctypes.c_int32), ("rk_stages", ctypes.c_int32),
                ("rk_A", ctypes.c_double * (MAX_STAGES * MAX_STAGES)), ("rk_b", ctypes.c_double * MAX_STAGES),
                ("rk_c", ctypes.c_double * MAX_STAGES), ("precision", ctypes.c_int32), ("device", ctypes.c_int32),
                ("precond", ctypes.c_int32)]


BC_VALUE_FIELDS = ("uLo", "uUp", "uLo_i", "uUp_i", "uLe_i", "uRi_i", "vLe", "vRi", "vLo_i", "vUp_i",
                   "vLe_i", "vRi_i", "pLe", "pRi", "pLo", "pUp", "dudtLe_i", "dudtRi_i", "dvdtLo_i", "dvdtUp_i")


class BcValues(ctypes.Structure):
    _fields_ = [(n, c_double_p) for n in BC_VALUE_FIELDS]


class Sizes(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("Nx", "Ny", "Nux_in", "Nuy_in", "Nvx_in", "Nvy_in", "Npx", "Npy",
                                               "Nu", "Nv", "NV", "Np")]


class SolveStats(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int32), ("norm1", ctypes.c_double), ("norm2", ctypes.c_double)]


class StepStats(ctypes.Structure):
    _fields_ = [("n_solves", ctypes.c_int32), ("iters_total", ctypes.c_int32), ("iters_max", ctypes.c_int32),
                ("norm1_max", ctypes.c_double)]


SAMPLER_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p)

_LIB = None


def load():
    """Loads libins2d.so, building it first when the sources are newer."""
    global _LIB
    if _LIB is not None:
        return _LIB
    from . import build as _build
    try:
        if not os.environ.get("INS2D_LIBRARY"):
            _build.build()
    except Exception as e:  # no nvcc: use an existing library if present
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libins2d.so is missing and could not be built: {e}") from e
    lib = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    P = ctypes.POINTER
    sig = {
        "ins2d_ctx_create": (ctypes.c_int, [P(GridDesc), P(BcDesc), P(Opts), P(vp)]),
        "ins2d_ctx_destroy": (ctypes.c_int, [vp]),
        "ins2d_last_error": (ctypes.c_char_p, [vp]),
        "ins2d_get_sizes": (ctypes.c_int, [vp, P(Sizes)]),
        "ins2d_set_stream": (ctypes.c_int, [vp, vp]),
        "ins2d_wait_stream": (ctypes.c_int, [vp, vp]),
        "ins2d_set_poll_limit": (ctypes.c_int, [vp, ctypes.c_int64]),
        "ins2d_set_bc_values": (ctypes.c_int, [vp, ctypes.c_double, P(BcValues)]),
        "ins2d_set_bc_sampler": (ctypes.c_int, [vp, SAMPLER_FN, vp]),
        "ins2d_F": (ctypes.c_int, [vp, vp, vp, vp, ctypes.c_double, ctypes.c_int, vp, P(ctypes.c_double),
                                   ctypes.c_int]),
        "ins2d_divergence": (ctypes.c_int, [vp, vp, vp, P(ctypes.c_double), ctypes.c_int]),
        "ins2d_laplacian": (ctypes.c_int, [vp, vp, vp, ctypes.c_int]),
        "ins2d_pressure_poisson": (ctypes.c_int, [vp, vp, vp, P(SolveStats), ctypes.c_int]),
        "ins2d_pressure_additional_solve": (ctypes.c_int, [vp, vp, vp, ctypes.c_double, P(SolveStats),
                                                           ctypes.c_int]),
        "ins2d_erk_step": (ctypes.c_int, [vp, vp, vp, ctypes.c_double, ctypes.c_double, P(StepStats),
                                          ctypes.c_int]),
        "ins2d_erk_run": (ctypes.c_int, [vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                         P(StepStats), ctypes.c_int]),
        "ins2d_conservation": (ctypes.c_int, [vp, vp, ctypes.c_double, P(ctypes.c_double), ctypes.c_int]),
        "ins2d_initial_projection": (ctypes.c_int, [vp, vp, ctypes.c_double, P(ctypes.c_double), ctypes.c_int]),
        "ins2d_profile": (ctypes.c_int, [vp, ctypes.c_int]),
        "ins2d_profile_read": (ctypes.c_int, [vp, P(ctypes.c_double), P(ctypes.c_int64)]),
        "ins2d_fft_poisson_noalloc": (ctypes.c_int, [vp, vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                                     ctypes.c_double, vp]),
        "ins2d_ens_create": (ctypes.c_int, [ctypes.c_int32, P(GridDesc), P(BcDesc), P(Opts), P(vp)]),
        "ins2d_ens_destroy": (ctypes.c_int, [vp]),
        "ins2d_ens_last_error": (ctypes.c_char_p, [vp]),
        "ins2d_ens_size": (ctypes.c_int32, [vp]),
        "ins2d_ens_member": (vp, [vp, ctypes.c_int32]),
        "ins2d_ens_set_stream": (ctypes.c_int, [vp, vp]),
        "ins2d_slab_fft_create": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                                 ctypes.c_int32, P(vp)]),
        "ins2d_slab_fft_destroy": (ctypes.c_int, [vp]),
        "ins2d_slab_fft_last_error": (ctypes.c_char_p, [vp]),
        "ins2d_slab_fft_rows_forward": (ctypes.c_int, [vp, vp, ctypes.c_int32, vp, vp]),
        "ins2d_slab_fft_columns": (ctypes.c_int, [vp, vp, ctypes.c_int32, ctypes.c_int32, P(ctypes.c_double), vp]),
        "ins2d_slab_fft_rows_inverse": (ctypes.c_int, [vp, vp, ctypes.c_int32, ctypes.c_double, vp, vp]),
        "ins2d_ens_wait_stream": (ctypes.c_int, [vp, vp]),
        "ins2d_ens_set_state": (ctypes.c_int, [vp, ctypes.c_int32, vp, vp, ctypes.c_int]),
        "ins2d_ens_get_state": (ctypes.c_int, [vp, ctypes.c_int32, vp, vp, ctypes.c_int]),
        "ins2d_ens_state_ptr": (ctypes.c_int, [vp, ctypes.c_int32, P(vp), P(vp)]),
        "ins2d_ens_set_member_dt": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_double]),
        "ins2d_ens_erk_run": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int32, P(StepStats)]),
        "ins2d_ens_set_solver": (ctypes.c_int, [vp, ctypes.c_int32]),
        "ins2d_ens_solve_shape": (ctypes.c_int, [vp, P(ctypes.c_int32), P(ctypes.c_int32), P(ctypes.c_double)]),
        "ins2d_cnn_create": (ctypes.c_int, [ctypes.c_int32, ctypes.c_uint64, P(vp)]),
        "ins2d_cnn_destroy": (ctypes.c_int, [vp]),
        "ins2d_cnn_last_error": (ctypes.c_char_p, [vp]),
        "ins2d_cnn_set_stream": (ctypes.c_int, [vp, vp]),
        "ins2d_cnn_set_path": (ctypes.c_int, [vp, ctypes.c_int32]),
        "ins2d_cnn_get_params": (ctypes.c_int, [vp, vp, P(ctypes.c_float)]),
        "ins2d_cnn_set_params": (ctypes.c_int, [vp, vp, ctypes.c_float]),
        "ins2d_cnn_get_activations": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int64, vp]),
        "ins2d_cnn_forward": (ctypes.c_int, [vp, vp, vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
        "ins2d_cnn_loss_grad": (ctypes.c_int, [vp, vp, vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                               P(ctypes.c_double), vp]),
        "ins2d_cnn_train_step": (ctypes.c_int, [vp, vp, vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                ctypes.c_float, P(ctypes.c_double)]),
        "ins2d_cnn_loss_grad_residual": (ctypes.c_int, [vp, vp, vp, ctypes.c_int32, P(ctypes.c_double), vp]),
        "ins2d_cnn_train_step_residual": (ctypes.c_int, [vp, vp, vp, ctypes.c_int32, ctypes.c_float,
                                                         P(ctypes.c_double)]),
        "ins2d_cnn_prepare_pairs": (ctypes.c_int, [vp, vp, vp, ctypes.c_int32, ctypes.c_int32, vp, vp]),
        "ins2d_set_learned_guess": (ctypes.c_int, [vp, vp]),
        "ins2d_set_learned_mode": (ctypes.c_int, [vp, ctypes.c_int32]),
        "ins2d_record_pairs": (ctypes.c_int, [vp, vp, vp, ctypes.c_int32]),
        "ins2d_recorded_pairs": (ctypes.c_int32, [vp]),
        "ins2d_learned_train": (ctypes.c_int, [vp, vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                               ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_float,
                                               ctypes.c_int32, ctypes.c_uint64, ctypes.c_int, P(ctypes.c_double),
                                               P(ctypes.c_double)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib
