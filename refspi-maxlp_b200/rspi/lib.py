"""ctypes binding of librspi.so (the C ABI declared in include/rspi.h).

The library is the only compute path: if it is missing or fails to load,
``load()`` raises.  There is no CPU fallback.
"""
import ctypes
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'librspi.so')

P = ctypes.c_void_p
L = ctypes.c_longlong
I = ctypes.c_int
D = ctypes.c_double
F = ctypes.c_float

# name: (restype, argtypes) -- mirrors include/rspi.h
SIGNATURES = {
    'rspi_version': (ctypes.c_char_p, []),
    'rspi_status_string': (ctypes.c_char_p, [I]),
    'rspi_photon_offsets': (I, [P, P, P, L, P, P, P, P, P, P, I, P, P]),
    'rspi_powder': (I, [P, L, P, P, L, L, L, P, P, P]),
    'rspi_ll_entry_rows': (I, [P, P, P, P, P, P, P, P, L, L, P, P, P, P]),
    'rspi_scan_rows': (I, [P, L, P, P]),
    'rspi_ll_entry_fill': (I, [P, P, P, P, P, P, P, P, L, L, P, P, P, P]),
    'rspi_holo_slices': (I, [P, P, P, P, L, L, P, P, L, P, P, P]),
    'rspi_vscale_init': (I, [P, L, P, P, L, P, P, P]),
    'rspi_rot_log_slices': (I, [P, L, L, P, L, P, P, L, L, L, L, P, I, P, P]),
    'rspi_holo_pairs': (I, [P, L, L, P, P]),
    'rspi_rot_log_slices_pairs': (I, [P, L, L, P, L, P, P, L, L, L, L, P, I, P, P]),
    'rspi_loglike': (I, [P, I, L, L, P, P, P, P, P, L, L, L, P, I, L, I, I, I, P]),
    'rspi_loglike_max_tile': (I, [L, I]),
    'rspi_frame_reduce': (I, [P, I, L, L, P, P, P, P]),
    'rspi_maxlp_frame_params': (I, [P, L, L, L, P, P, P, P, P]),
    'rspi_maxlp_histogram': (I, [P, P, P, P, P, P, P, L, P, P, P, L, P, L, L, P, P, P]),
    'rspi_maxlp_pixel_map': (I, [P, L, L, P, P, P, P, P]),
    'rspi_maxlp_histogram_map': (I, [P, P, P, P, P, P, P, L, P, P, L, L, P, P, L, P, P, P]),
    'rspi_maxlp_pattern': (I, [P, P, P, L, P, L, P, L, P, L, I, P, I, P, P]),
    'rspi_maxlp_pattern_screened': (I, [P, P, P, L, P, L, P, L, P, L, I, P, I, P, P, P]),
    'rspi_log2_error_max': (I, [F, F, P, P]),
    'rspi_maxlp_pixel_frames': (I, [I, L, P, L] + [P] * 7 + [L, P, P, P, P, P, P]),
    'rspi_maxlp_pixel_values': (I, [P, L, P, P, L, I, D, P, P, P]),
    'rspi_sets_entries_check': (I, [P, L, I, P, P]),
    'rspi_sim_views': (I, [P, P, I, L, L, P, P, P, P, D, D, D, I, P, P, P]),
    'rspi_sim_counts': (I, [P, L, L, P, P, I, ctypes.c_ulonglong, P, P, P, P]),
    'rspi_sim_poisson': (I, [P, L, ctypes.c_ulonglong, ctypes.c_ulonglong, P, P, P]),
    'rspi_sim_sparse_counts': (I, [P, L, L, P, P, P]),
    'rspi_sim_sparse_fill': (I, [P, L, L, P, P, P, P, P, P]),
    'rspi_maxlp_fcalc': (I, [L, D, D, D, P, P, P, P]),
    'rspi_sphere_ramp': (I, [L, D, D, D, P, P, P]),
    'rspi_quad4_entry_groups': (I, [P, P, L, I, I, I, P, P]),
    'rspi_quad4_entry_fill': (I, [P, P, L, I, I, I, P, P, L, L, P, P]),
    'rspi_quad4_part_sums_floats': (L, [L, I]),
    'rspi_screen_loglike7': (I, [P, L, L, P, P, P, P, P, L, I, I, L, L, P, L, P, I, I, I, P]),
    'rspi_mean': (I, [P, L, P, P]),
    'rspi_ll16_entry_rows': (I, [P] * 8 + [L, L, I, P, P, P]),
    'rspi_ll16_entry_fill': (I, [P] * 8 + [L, L, I, P, P, P]),
    'rspi_screen_candidates': (I, [P, L, L, P, P, P, P, P, D, P, P, P, P, P, L, P, P, P, P]),
    'rspi_rescore': (I, [P, P, P, L, L, L, P, L, P, L, P, P, L, L, P, P, P, P, P, P, P, P, P,
                         P, P, P, P, P, P, L, P]),
    'rspi_screen_candidates_noalloc': (I, [P, L, L, P, P, P, P, P, D, P, P, P, P, L, P, P, P,
                                           P]),
    'rspi_nll': (I, [I, I] + [P] * 7 + [L, P, L, P, L] + [P] * 18),
    'rspi_entries16_check': (I, [P, L, P, P]),
    'rspi_emc_nll': (I, [I, I, P, L, P, P, L, P, P, P, P, P, P, P, P, L, P, P, P, P, P, D, P,
                         P, P, P, P, P, P, P, P]),
    'rspi_cdft2': (I, [P, P, P, L, I, P]),
    'rspi_phase_support': (I, [P, L, D, D, D, I, D, P, P, P]),
    'rspi_phase_proj_fourier': (I, [P, P, P, P, L, P]),
    'rspi_phase_proj_real': (I, [P, P, P, P, L, P]),
    'rspi_phase_refine': (I, [P, P, P, P, P, L, I, I, P]),
    'rspi_sets_counts': (I, [P, P, L, I, I, I, P, P]),
    'rspi_sets_group': (I, [P, P, L, I, I, P, P, P]),
    'rspi_sets_steps': (I, [P, P, L, I, P, P, P]),
    'rspi_sets_fill': (I, [P, P, I, I, I, P, P, L, P, P, P, P]),
    'rspi_holo_quads32': (I, [P, L, L, P, P]),
    'rspi_rot_log_slices_sets': (I, [P, P, L, L, P, L, P, P, L, I, I, L, L, P, P, P]),
    'rspi_sets_part_sums_floats': (L, [L, I]),
    'rspi_screen_loglike_sets': (I, [P, L, P, P, P, P, P, P, L, I, I, L, L, P, L, P, I, P, I,
                                     I, P, P]),
    'rspi_frame_max_finalize': (I, [P, P, L, P, P, P]),
    'rspi_screen_candidates_cols': (I, [P, L, L, P, L, P, P, P, P, P, D, P, P, P, P, P, L, P, P,
                                        P, P, P]),
    'rspi_rescore_cols': (I, [P, P, P, L, L, L, P, L, P, L, P, P, L, L, P, P, P, P, P, P, P, P,
                              P, L, P, P, P, P, P, P, P, L, P]),
    'rspi_loglike_stream': (I, [I, P, L, L, P, P, P, P, L, L, L, P, L, I, I, I, P]),
    'rspi_posterior_pairs': (I, [P, L, L, P, D, P, P, P, L, P, P, P, P, P]),
    'rspi_merge_coverage': (I, [L, P, L, P, P]),
    'rspi_merge': (I, [P, P, P, P, L, P, D, P, P, P, P, P, P, P, P, L, L, P, L, P, P, P, P, P, P]),
    'rspi_dense_frames': (I, [P, L, L, P, L, L, P, P, P, P]),
    'rspi_rot_log_split': (I, [P, L, L, P, L, P, P, L, L, L, L, P, P, P, P]),
    'rspi_dense_loglike': (I, [P, P, P, P, L, L, L, L, L, L, P, P, P, L, P, P]),
    'rspi_maxlp_grid': (I, [P, P, P, L, P, L, P, P, L, P, L, I, I, P, P, P, P]),
    'rspi_dense_frames_u8': (I, [P, L, L, P, L, L, P, P, P]),
    'rspi_rot_log_fixed': (I, [P, L, L, P, L, P, P, L, L, L, L, L, P, P, P]),
    'rspi_dense_loglike_i8': (I, [P, P, L, L, L, L, L, L, P, P, P, L, P, P]),
}

_lib = None


class RspiError(RuntimeError):
    pass


def load():
    """Load and type the library once; raise if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RspiError('librspi.so is not built (%s); run __graft_entry__.build() or '
                        'python refspi-maxlp_b200/csrc/build.py' % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def status_string(code):
    return load().rspi_status_string(int(code)).decode()


def check(code, what):
    if code != 0:
        raise RspiError('%s failed: %s (%d)' % (what, status_string(code), code))


# kernels each entry point launches (memsets are not counted)
KERNELS_PER_CALL = {
    'rspi_photon_offsets': 4, 'rspi_powder': 2, 'rspi_ll_entry_rows': 1, 'rspi_scan_rows': 1,
    'rspi_ll_entry_fill': 1, 'rspi_holo_slices': 1, 'rspi_vscale_init': 1,
    'rspi_rot_log_slices': 1, 'rspi_holo_pairs': 1, 'rspi_rot_log_slices_pairs': 1,
    'rspi_loglike': 1, 'rspi_frame_reduce': 1,
    'rspi_maxlp_frame_params': 1, 'rspi_maxlp_histogram': 1, 'rspi_maxlp_pixel_map': 3,
    'rspi_maxlp_histogram_map': 1, 'rspi_maxlp_pattern': 1,
    'rspi_maxlp_pattern_screened': 1, 'rspi_log2_error_max': 1,
    'rspi_maxlp_pixel_frames': 1, 'rspi_maxlp_pixel_values': 1, 'rspi_maxlp_fcalc': 1,
    'rspi_sphere_ramp': 1, 'rspi_quad4_entry_groups': 1, 'rspi_quad4_entry_fill': 2,
    'rspi_screen_loglike7': 1, 'rspi_quad4_part_sums_floats': 0,
    'rspi_mean': 1, 'rspi_ll16_entry_rows': 1, 'rspi_ll16_entry_fill': 1, 'rspi_screen_candidates': 3, 'rspi_rescore': 5,
    'rspi_loglike_stream': 1, 'rspi_posterior_pairs': 3,
    'rspi_entries16_check': 1, 'rspi_emc_nll': 2, 'rspi_cdft2': 2, 'rspi_phase_support': 5,
    'rspi_phase_proj_fourier': 1, 'rspi_phase_proj_real': 4, 'rspi_sets_counts': 1, 'rspi_sets_group': 1, 'rspi_sets_steps': 1,
    'rspi_sets_fill': 1, 'rspi_rot_log_slices_sets': 1, 'rspi_holo_quads32': 1, 'rspi_sets_part_sums_floats': 0,
    'rspi_screen_loglike_sets': 1, 'rspi_frame_max_finalize': 1,
    'rspi_screen_candidates_cols': 4, 'rspi_rescore_cols': 5, 'rspi_nll': 2, 'rspi_screen_candidates_noalloc': 3, 'rspi_merge_coverage': 1, 'rspi_merge': 2,
    'rspi_dense_frames': 1, 'rspi_rot_log_split': 1, 'rspi_dense_loglike': 1,
    'rspi_maxlp_grid': 2, 'rspi_dense_frames_u8': 1, 'rspi_rot_log_fixed': 1,
    'rspi_dense_loglike_i8': 1, 'rspi_sets_entries_check': 1, 'rspi_sim_views': 1, 'rspi_sim_counts': 1,
    'rspi_sim_poisson': 1, 'rspi_sim_sparse_counts': 1, 'rspi_sim_sparse_fill': 1,
}
launch_count = 0


def call(name, *args):
    """Call entry point ``name``, raise on a non-zero status, count launches."""
    global launch_count
    check(getattr(load(), name)(*args), name)
    launch_count += KERNELS_PER_CALL.get(name, 0)
