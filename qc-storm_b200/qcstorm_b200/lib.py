"""ctypes binding of lib/libqcstorm_b200.so (include/qcstorm_b200.h).

Thin: every call goes to the C ABI.  There is no CPU fallback; if the
library or a CUDA device is missing the calls raise.
"""
import ctypes as C
import os

import numpy as np

from .abi import LIB_PATH, LocPara

_lib = None

# name -> (restype, argtypes) of every exported function of the header
_SIGS = {
    "qcs_loc_para_default": (None, [C.POINTER(LocPara)]),
    "qcs_last_error": (C.c_char_p, []),
    "qcs_device_available": (C.c_int, []),
    "qcs_loc_init": (C.c_int, [C.POINTER(LocPara), C.POINTER(C.c_void_p)]),
    "qcs_loc_init_capacity": (C.c_int, [C.POINTER(LocPara), C.c_int, C.POINTER(C.c_void_p)]),
    "qcs_loc_deinit": (C.c_int, [C.c_void_p]),
    "qcs_loc_capacity": (C.c_int, [C.c_void_p]),
    "qcs_loc_bfgs_mle_localization": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(LocPara), C.c_int,
                                                C.c_void_p]),
    "qcs_loc_read_rows": (C.c_int, [C.c_void_p, C.POINTER(LocPara), C.c_void_p]),
    "qcs_loc_h_loc_arry": (C.c_void_p, [C.c_void_p]),
    "qcs_loc_valid_num": (C.c_int, [C.c_void_p]),
    "qcs_loc_fit_ratios": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qcs_loc_localize_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(LocPara), C.c_int,
                                          C.c_void_p]),
    "qcs_loc_localize_device_n": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(LocPara), C.c_void_p,
                                            C.c_int, C.c_void_p]),
    "qcs_loc_localize_mixed_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                                C.c_void_p]),
    "qcs_loc_device_rows": (C.c_void_p, [C.c_void_p]),
    "qcs_loc_device_valid_num": (C.c_void_p, [C.c_void_p]),
    "qcs_loc_device_roi_buffer": (C.c_void_p, [C.c_void_p]),
    "qcs_loc_device_wle_buffer": (C.c_void_p, [C.c_void_p]),
    "qcs_wle_estimate": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(LocPara), C.c_void_p]),
    "qcs_wle_estimate_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(LocPara), C.c_void_p,
                                          C.c_void_p]),
    "qcs_fit_single_device": (C.c_int, [C.c_int, C.POINTER(LocPara), C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                        C.c_void_p]),
    "qcs_crlb_device": (C.c_int, [C.POINTER(LocPara), C.c_void_p, C.c_int, C.c_void_p]),
    "qcs_loc_set_model_selection": (C.c_int, [C.c_void_p, C.c_int, C.c_float]),
    "qcs_loc_model_selection": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    "qcs_crlb_fisher_fp64": (C.c_int, [C.POINTER(LocPara), C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                       C.c_void_p]),
    "qcs_fit_single_group_device": (C.c_int, [C.c_int, C.POINTER(LocPara), C.c_void_p, C.c_void_p, C.c_int,
                                              C.c_void_p, C.c_int, C.c_void_p]),
    "qcs_measure_mufu_rate": (C.c_int, [C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_double)]),
    "qcs_localize_noalloc": (C.c_int, [C.POINTER(LocPara), C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
    "qcs_zero_init": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "qcs_zero_deinit": (C.c_int, [C.c_void_p]),
    "qcs_zero_remove": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "qcs_zero_h_loc_arry": (C.c_void_p, [C.c_void_p]),
    "qcs_zero_valid_num": (C.c_int, [C.c_void_p]),
    "qcs_zero_remove_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                         C.c_void_p, C.c_void_p, C.c_void_p]),
    "qcs_learned_param_count": (C.c_int, []),
    "qcs_learned_create": (C.c_int, [C.c_int, C.c_ulonglong, C.POINTER(C.c_void_p)]),
    "qcs_learned_destroy": (C.c_int, [C.c_void_p]),
    "qcs_learned_get_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qcs_learned_set_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qcs_learned_features_device": (C.c_int, [C.POINTER(LocPara), C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                              C.c_void_p]),
    "qcs_learned_targets_device": (C.c_int, [C.POINTER(LocPara), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                             C.c_void_p, C.c_void_p, C.c_void_p]),
    "qcs_learned_forward_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "qcs_learned_gradient_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                              C.POINTER(C.c_float), C.c_void_p]),
    "qcs_learned_get_grads": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qcs_learned_train_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                           C.c_float, C.c_ulonglong, C.c_void_p, C.c_void_p]),
    "qcs_learned_start_device": (C.c_int, [C.c_void_p, C.POINTER(LocPara), C.c_void_p, C.c_int, C.c_void_p,
                                           C.c_void_p, C.c_void_p]),
    "qcs_learned_work_bytes": (C.c_size_t, [C.c_int]),
    "qcs_learned_localize_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(LocPara),
                                              C.c_int, C.c_int, C.c_int, C.c_float, C.c_void_p]),
    "qcs_learned_refit_num": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "qcs_learned_set_inference": (C.c_int, [C.c_void_p, C.c_int]),
    "qcs_loc_localize_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(LocPara), C.c_int, C.c_void_p]),
    "qcs_learned_localize_async": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(LocPara),
                                             C.c_int, C.c_int, C.c_int, C.c_float, C.c_void_p]),
    "qcs_loc_finish": (C.c_int, [C.c_void_p, C.POINTER(LocPara)]),
    "qcs_locfile_open": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "qcs_locfile_write": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "qcs_locfile_write_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "qcs_locfile_flush": (C.c_int, [C.c_void_p]),
    "qcs_locfile_rows": (C.c_longlong, [C.c_void_p]),
    "qcs_locfile_close": (C.c_int, [C.c_void_p]),
    "qcs_render_init": (C.c_int, [C.POINTER(LocPara), C.c_int, C.POINTER(C.c_void_p)]),
    "qcs_render_deinit": (C.c_int, [C.c_void_p]),
    "qcs_render_reset": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qcs_render_reset_max": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qcs_render_rows": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(LocPara), C.c_int, C.c_float, C.c_int,
                                  C.c_void_p]),
    "qcs_render_rows_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(LocPara), C.c_int,
                                         C.c_float, C.c_void_p]),
    "qcs_render_d_image": (C.c_void_p, [C.c_void_p]),
    "qcs_render_d_colormap": (C.c_void_p, [C.c_void_p]),
    "qcs_render_read": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "qcs_learned_fused_status": (C.c_int, [C.c_void_p]),
    "qcs_fit_from_start_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(LocPara), C.c_int,
                                            C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_void_p]),
    "qcs_extract_max_batched_num": (C.c_int, [C.c_int, C.c_int]),
    "qcs_extract_init": (C.c_int, [C.POINTER(LocPara), C.POINTER(C.c_void_p)]),
    "qcs_extract_init_ex": (C.c_int, [C.POINTER(LocPara), C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "qcs_extract_deinit": (C.c_int, [C.c_void_p]),
    "qcs_extract_molecules": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(LocPara), C.c_int, C.c_int,
                                        C.c_void_p]),
    "qcs_extract_accumulated_roi_num": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "qcs_extract_reset_roi_num": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qcs_extract_h_image_roi": (C.c_void_p, [C.c_void_p]),
    "qcs_extract_h_wle_para": (C.c_void_p, [C.c_void_p]),
    "qcs_extract_d_image_roi": (C.c_void_p, [C.c_void_p]),
    "qcs_extract_d_wle_para": (C.c_void_p, [C.c_void_p]),
    "qcs_extract_device_roi_num": (C.c_void_p, [C.c_void_p]),
    "qcs_extract_frame_range": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "qcs_extract_dropped_num": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "qcs_learned_gradient_counts_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                     C.c_int, C.POINTER(C.c_float), C.c_void_p]),
    "qcs_learned_train_counts_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                  C.c_int, C.c_int, C.c_float, C.c_ulonglong, C.c_void_p,
                                                  C.c_void_p]),
    "qcs_loc_count_labels_device": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "qcs_learned_set_count_threshold": (C.c_int, [C.c_void_p, C.c_float]),
    "qcs_learned_set_two_emitter": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int]),
    "qcs_learned_set_direct_two_emitter": (C.c_int, [C.c_void_p, C.c_int]),
    "qcs_learned_set_single_refits": (C.c_int, [C.c_void_p, C.c_int]),
    "qcs_learned_refit_2e_num": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "qcs_learned_set_three_emitter": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float]),
    "qcs_learned_refit_3e_num": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "qcs_loc_set_three_emitter_capture": (C.c_int, [C.c_void_p, C.c_int]),
    "qcs_loc_device_three_emitter_params": (C.c_void_p, [C.c_void_p]),
    "qcs_loc_three_emitter_targets_device": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(LocPara), C.c_int,
                                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "qcs_loc_two_emitter_targets_device": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(LocPara), C.c_int, C.c_void_p,
                                                     C.c_void_p, C.c_void_p, C.c_void_p]),
    "qcs_consec_init": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "qcs_consec_deinit": (C.c_int, [C.c_void_p]),
    "qcs_consec_fit": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(LocPara), C.c_void_p]),
    "qcs_consec_fit_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(LocPara), C.c_void_p]),
    "qcs_consec_out_num": (C.c_int, [C.c_void_p]),
    "qcs_consec_h_out_loc_arry": (C.c_void_p, [C.c_void_p]),
    "qcs_consec_d_out_loc_arry": (C.c_void_p, [C.c_void_p]),
    "qcs_consec_ontime_ratio": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qcs_consec_read_rows": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qcs_loc_autotune": (C.c_int, [C.c_void_p, C.POINTER(LocPara), C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "qcs_loc_tuning": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "qcs_loc_set_tuning": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "qcs_loc_tuning_multi": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "qcs_loc_set_tuning_multi": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "qcs_loc_save_tuning": (C.c_int, [C.c_void_p, C.c_char_p]),
    "qcs_learned_autotune": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(LocPara), C.c_int,
                                       C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p]),
    "qcs_loc_load_tuning": (C.c_int, [C.c_void_p, C.c_char_p]),
    "qcs_stat_init": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "qcs_stat_deinit": (C.c_int, [C.c_void_p]),
    "qcs_stat_reset_all": (C.c_int, [C.c_void_p]),
    "qcs_stat_get_statistical_inf": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(LocPara), C.c_void_p]),
    "qcs_stat_get_statistical_inf_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(LocPara),
                                                      C.c_void_p]),
    "qcs_stat_histograms": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qcs_stat_means": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qcs_stat_series": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "qcs_stat_update_ontime_ratio": (C.c_int, [C.c_void_p, C.c_void_p]),
    "qcs_stat_ontime": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.c_void_p]),
    "qcs_learned_create_for": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.POINTER(C.c_void_p)]),
    "qcs_learned_create_arch": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.POINTER(C.c_void_p)]),
    "qcs_learned_arch": (C.c_int, [C.c_void_p]),
    "qcs_learned_shape": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "qcs_learned_localize_device_n": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(LocPara),
                                                C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_void_p]),
    "qcs_learned_count_threshold": (C.c_float, [C.c_void_p]),
    "qcs_learned_classes_device": (C.c_int, [C.c_void_p, C.POINTER(LocPara), C.c_void_p, C.c_int, C.c_void_p,
                                             C.c_void_p, C.c_void_p]),
    "qcs_fit_from_start_classes_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(LocPara), C.c_int,
                                                    C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float,
                                                    C.c_void_p]),
}


class QcsError(RuntimeError):
    def __init__(self, code, what):
        super().__init__("qcstorm_b200 error %d: %s" % (code, what))
        self.code = code


def load(path=LIB_PATH):
    """Load the library (once) and attach signatures."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError("qcstorm_b200 library not built: %s (run qc-storm_b200/build.py)" % path)
        lib = C.CDLL(path)
        for name, (res, args) in _SIGS.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def check(code):
    if code != 0:
        raise QcsError(code, load().qcs_last_error().decode())


def _host(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    return a, C.c_void_p(a.ctypes.data)


def localize_mixed_device(entries, stream=0):
    """qcs_loc_localize_mixed_device: entries = [(LocContext, d_rois, n, d_wle or 0, para or None), ...] of
    different ROI sizes; their single-emitter fits run in one persistent launch, rows stay in each context."""
    lib = load()
    k = len(entries)
    ctx = (C.c_void_p * k)(*[e[0].h for e in entries])
    rois = (C.c_void_p * k)(*[e[1] for e in entries])
    wle = (C.c_void_p * k)(*[(e[3] if len(e) > 3 and e[3] else None) for e in entries])
    para = (LocPara * k)(*[(e[4] if len(e) > 4 and e[4] is not None else e[0].para) for e in entries])
    n = (C.c_int * k)(*[int(e[2]) for e in entries])
    check(lib.qcs_loc_localize_mixed_device(C.cast(ctx, C.c_void_p), C.cast(rois, C.c_void_p), C.cast(wle, C.c_void_p),
                                            C.cast(para, C.c_void_p), C.cast(n, C.c_void_p), k,
                                            C.c_void_p(stream) if stream else None))


class LocContext:
    """LDLocData_TypeDef: buffers for records of one ROI size."""

    def __init__(self, para, capacity=0):
        self.lib = load()
        self.para = para
        h = C.c_void_p()
        check(self.lib.qcs_loc_init_capacity(C.byref(para), int(capacity), C.byref(h)))
        self.h = h
        self.capacity = self.lib.qcs_loc_capacity(h)

    def close(self):
        if self.h:
            self.lib.qcs_loc_deinit(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def localize(self, rois, wle=None, para=None, stream=0, copy=True):
        """BFGS_MLELocalization on host arrays; returns (rows[n_valid, 12], ratios[7]); copy=False returns a view
        of the context's pinned row buffer (h_LocArry), valid until the next call."""
        para = para or self.para
        rois, pr = _host(rois, np.uint16)
        n = rois.shape[0]
        pw = None
        if wle is not None:
            wle, pw = _host(wle, np.float32)
        check(self.lib.qcs_loc_bfgs_mle_localization(self.h, pr, pw, C.byref(para), n,
                                                     C.c_void_p(stream) if stream else None))
        nv = self.lib.qcs_loc_valid_num(self.h)
        ptr = self.lib.qcs_loc_h_loc_arry(self.h)
        rows = np.ctypeslib.as_array((C.c_float * (12 * nv)).from_address(ptr)).reshape(nv, 12) if nv else \
            np.zeros((0, 12), np.float32)
        ratios = np.zeros(7, np.float32)
        check(self.lib.qcs_loc_fit_ratios(self.h, C.c_void_p(ratios.ctypes.data)))
        return (rows.copy() if copy and nv else rows), ratios

    def wle(self, rois, para=None):
        """WLEParameterEstimate on host records; returns wle[n, 6]."""
        para = para or self.para
        rois, pr = _host(rois, np.uint16)
        out = np.zeros((rois.shape[0], 6), np.float32)
        check(self.lib.qcs_wle_estimate(self.h, pr, rois.shape[0], C.byref(para), C.c_void_p(out.ctypes.data)))
        return out

    def set_model_selection(self, mode="lr", threshold=0.0):
        """Multi-emitter model selection: "cascade" (the reference's, default)
        or "lr" (FP64 likelihood-ratio test over 1, 2, 3 emitter fits)."""
        if mode not in ("cascade", "lr"):
            raise ValueError("mode: 'cascade' or 'lr'")
        check(self.lib.qcs_loc_set_model_selection(self.h, 1 if mode == "lr" else 0, C.c_float(threshold)))

    def model_selection(self):
        m, t = C.c_int(0), C.c_float(0)
        check(self.lib.qcs_loc_model_selection(self.h, C.byref(m), C.byref(t)))
        return ("lr" if m.value == 1 else "cascade"), t.value

    def localize_async(self, h_rois_ptr, n, h_wle_ptr=0, stream=0, para=None, net=None, iters=2, dev_th=0.0,
                       bisections=0):
        """qcs_loc_localize_async (or, with net, qcs_learned_localize_async) on host
        memory given by address (pinned for overlap); finish() publishes the rows."""
        para = para or self.para
        self._async_para = para
        wle = C.c_void_p(h_wle_ptr) if h_wle_ptr else None
        st = C.c_void_p(stream) if stream else None
        if net is None:
            check(self.lib.qcs_loc_localize_async(self.h, C.c_void_p(h_rois_ptr), wle, C.byref(para), int(n), st))
        else:
            check(self.lib.qcs_learned_localize_async(self.h, net.h, C.c_void_p(h_rois_ptr), wle, C.byref(para),
                                                      int(n), int(iters), int(bisections), C.c_float(dev_th), st))

    def finish(self, copy=True):
        """qcs_loc_finish: (rows[n_valid, 12], ratios[7]); copy=False returns a view of
        the context's pinned row buffer, valid until the next call."""
        check(self.lib.qcs_loc_finish(self.h, C.byref(getattr(self, "_async_para", None) or self.para)))
        nv = self.lib.qcs_loc_valid_num(self.h)
        ptr = self.lib.qcs_loc_h_loc_arry(self.h)
        rows = np.ctypeslib.as_array((C.c_float * (12 * nv)).from_address(ptr)).reshape(nv, 12) if nv else \
            np.zeros((0, 12), np.float32)
        ratios = np.zeros(7, np.float32)
        check(self.lib.qcs_loc_fit_ratios(self.h, C.c_void_p(ratios.ctypes.data)))
        return (rows.copy() if copy else rows), ratios

    # device-pointer forms (integers from torch.Tensor.data_ptr(), stream handles)
    def localize_device(self, d_rois, n, d_wle=0, stream=0, para=None):
        para = para or self.para
        check(self.lib.qcs_loc_localize_device(self.h, C.c_void_p(d_rois), C.c_void_p(d_wle) if d_wle else None,
                                               C.byref(para), int(n), C.c_void_p(stream) if stream else None))

    def localize_device_n(self, d_rois, d_wle, d_n, max_n, stream=0, para=None):
        """Localization of *d_n device records (count read on the device)."""
        para = para or self.para
        check(self.lib.qcs_loc_localize_device_n(self.h, C.c_void_p(d_rois), C.c_void_p(d_wle), C.byref(para),
                                                 C.c_void_p(d_n), int(max_n), C.c_void_p(stream) if stream else None))

    def autotune(self, d_rois, d_wle, n, para=None, stream=0):
        """qcs_loc_autotune: lanes per ROI by batch size; returns the table [(largest batch, lanes)]."""
        para = para or self.para
        check(self.lib.qcs_loc_autotune(self.h, C.byref(para), C.c_void_p(d_rois), C.c_void_p(d_wle), int(n),
                                        C.c_void_p(stream) if stream else None))
        return self.tuning()

    def tuning(self):
        sizes = np.zeros(8, np.int32)
        lanes = np.zeros(8, np.int32)
        k = self.lib.qcs_loc_tuning(self.h, C.c_void_p(sizes.ctypes.data), C.c_void_p(lanes.ctypes.data), 8)
        return [(int(sizes[i]), int(lanes[i])) for i in range(k)]

    def set_tuning(self, table):
        sizes = np.array([t[0] for t in table] or [0], np.int32)
        lanes = np.array([t[1] for t in table] or [1], np.int32)
        check(self.lib.qcs_loc_set_tuning(self.h, C.c_void_p(sizes.ctypes.data), C.c_void_p(lanes.ctypes.data),
                                          len(table)))

    def tuning_multi(self):
        """(2E limit, 3E limit) of the multi-emitter stages' lane-group kernels."""
        a, b = C.c_int(0), C.c_int(0)
        check(self.lib.qcs_loc_tuning_multi(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_tuning_multi(self, limit_2e, limit_3e):
        check(self.lib.qcs_loc_set_tuning_multi(self.h, int(limit_2e), int(limit_3e)))

    def save_tuning(self, path):
        check(self.lib.qcs_loc_save_tuning(self.h, str(path).encode()))

    def load_tuning(self, path):
        check(self.lib.qcs_loc_load_tuning(self.h, str(path).encode()))

    def read_rows(self, stream=0, para=None):
        """Rows of the last device call, on the host: (rows[n_valid, 12], ratios[7])."""
        para = para or self.para
        check(self.lib.qcs_loc_read_rows(self.h, C.byref(para), C.c_void_p(stream) if stream else None))
        nv = self.lib.qcs_loc_valid_num(self.h)
        ptr = self.lib.qcs_loc_h_loc_arry(self.h)
        rows = np.ctypeslib.as_array((C.c_float * (12 * nv)).from_address(ptr)).reshape(nv, 12).copy() if nv else \
            np.zeros((0, 12), np.float32)
        ratios = np.zeros(7, np.float32)
        check(self.lib.qcs_loc_fit_ratios(self.h, C.c_void_p(ratios.ctypes.data)))
        return rows, ratios

    def device_rows(self):
        return self.lib.qcs_loc_device_rows(self.h)

    def device_valid_num(self):
        return self.lib.qcs_loc_device_valid_num(self.h)


def fit_single_device(loc_type, para, d_rois, d_wle, n, d_loc, stream=0):
    check(load().qcs_fit_single_device(int(loc_type), C.byref(para), C.c_void_p(d_rois), C.c_void_p(d_wle), int(n),
                                       C.c_void_p(d_loc), C.c_void_p(stream) if stream else None))


def fit_single_group_device(loc_type, para, d_rois, d_wle, n, d_loc, lanes=8, stream=0):
    """qcs_fit_single_group_device: the single-emitter fit with `lanes` lanes per ROI."""
    check(load().qcs_fit_single_group_device(int(loc_type), C.byref(para), C.c_void_p(d_rois), C.c_void_p(d_wle),
                                             int(n), C.c_void_p(d_loc), int(lanes),
                                             C.c_void_p(stream) if stream else None))


def crlb_device(para, d_loc, n, stream=0):
    check(load().qcs_crlb_device(C.byref(para), C.c_void_p(d_loc), int(n), C.c_void_p(stream) if stream else None))


FISHER_COLS = 8  # x nm, y nm, z nm, photons, background, sigma_x px, sigma_y px, status
FISHER_NAMES = ["x_nm", "y_nm", "z_nm", "photons", "background", "sigma_x_px", "sigma_y_px", "status"]


def crlb_fisher_device(para, d_rows, n, d_out, d_rois=0, n_rois=0, stream=0):
    """qcs_crlb_fisher_fp64: the FP64 Fisher-matrix CRLB of n device rows into
    d_out (n x FISHER_COLS floats); d_rois / n_rois place the first n_rois
    rows' emitters at their fitted positions in their records."""
    check(load().qcs_crlb_fisher_fp64(C.byref(para), C.c_void_p(d_rows), int(n),
                                      C.c_void_p(d_rois) if d_rois else None, int(n_rois), C.c_void_p(d_out),
                                      C.c_void_p(stream) if stream else None))


def crlb_fisher(para, rows, rois=None):
    """The same from host rows (and records), through device copies."""
    import torch
    rows = np.ascontiguousarray(rows, np.float32)
    n = rows.shape[0]
    d_rows = torch.from_numpy(rows).cuda()
    d_out = torch.zeros((max(n, 1), FISHER_COLS), dtype=torch.float32, device="cuda")
    d_rois = None
    if rois is not None:
        d_rois = torch.from_numpy(np.ascontiguousarray(rois, np.uint16).view(np.int16)).cuda()
    s = torch.cuda.current_stream()
    crlb_fisher_device(para, d_rows.data_ptr(), n, d_out.data_ptr(), d_rois.data_ptr() if d_rois is not None else 0,
                       rois.shape[0] if rois is not None else 0, s.cuda_stream)
    s.synchronize()
    return d_out.cpu().numpy()[:n]


def mufu_rate(iters=4000):
    """Measured MUFU operations per second of the current device."""
    ms = C.c_float(0)
    ops = C.c_double(0)
    check(load().qcs_measure_mufu_rate(int(iters), C.byref(ms), C.byref(ops)))
    return ops.value / (ms.value * 1e-3)


IMAGE_SOURCE = {"gpu": 0, "pinned": 1, "normal": 2}


class ExtractContext:
    """LDROIExtractData_TypeDef: detection and ROI cutting on batches of frames.

    Records and WLE rows accumulate on the device across extract() calls until
    reset(), like the reference's TotalROINumber."""

    def __init__(self, para, max_batched_num=0, capacity=0):
        self.lib = load()
        self.para = para
        h = C.c_void_p()
        check(self.lib.qcs_extract_init_ex(C.byref(para), int(max_batched_num), int(capacity), C.byref(h)))
        self.h = h
        self.whole = para.ROISize * (para.ROISize + 1)

    def close(self):
        if self.h:
            self.lib.qcs_extract_deinit(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def extract(self, frames, start_frame=0, para=None, stream=0):
        """ExtractMolecules on a host array of stacked frames (n, H, W) uint16."""
        para = para or self.para
        frames, pf = _host(frames, np.uint16)
        nb = frames.shape[0] if frames.ndim == 3 else 1
        check(self.lib.qcs_extract_molecules(self.h, pf, IMAGE_SOURCE["normal"], C.byref(para), int(start_frame), nb,
                                             C.c_void_p(stream) if stream else None))

    def extract_device(self, d_frames, batched_num, start_frame=0, para=None, stream=0, source="gpu"):
        """ExtractMolecules on frames at a device (or pinned host) address."""
        para = para or self.para
        check(self.lib.qcs_extract_molecules(self.h, C.c_void_p(d_frames), IMAGE_SOURCE[source], C.byref(para),
                                             int(start_frame), int(batched_num),
                                             C.c_void_p(stream) if stream else None))

    def accumulated(self):
        n = C.c_int(0)
        check(self.lib.qcs_extract_accumulated_roi_num(self.h, C.byref(n)))
        return n.value

    def reset(self, stream=0):
        check(self.lib.qcs_extract_reset_roi_num(self.h, C.c_void_p(stream) if stream else None))

    def records(self):
        """Host copies of the accumulated (records[n, R(R+1)] uint16, wle[n, 6] float32)."""
        n = self.accumulated()
        pr = self.lib.qcs_extract_h_image_roi(self.h)
        pw = self.lib.qcs_extract_h_wle_para(self.h)
        if not pr or not pw:
            raise QcsError(4, self.lib.qcs_last_error().decode())
        if n == 0:
            return np.zeros((0, self.whole), np.uint16), np.zeros((0, 6), np.float32)
        rois = np.ctypeslib.as_array((C.c_uint16 * (self.whole * n)).from_address(pr)).reshape(n, self.whole).copy()
        wle = np.ctypeslib.as_array((C.c_float * (6 * n)).from_address(pw)).reshape(n, 6).copy()
        return rois, wle

    def frame_range(self):
        a, b = C.c_int(0), C.c_int(0)
        check(self.lib.qcs_extract_frame_range(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def dropped(self):
        n = C.c_int(0)
        check(self.lib.qcs_extract_dropped_num(self.h, C.byref(n)))
        return n.value

    def device_records(self):
        """(device address of the records, of the WLE rows, of the int count)."""
        return (self.lib.qcs_extract_d_image_roi(self.h), self.lib.qcs_extract_d_wle_para(self.h),
                self.lib.qcs_extract_device_roi_num(self.h))


class ZeroRemover:
    """ZeroLocalizationsRemovel_TypeDef: drop rejected rows, optionally order by frame."""

    def __init__(self, capacity=0):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.qcs_zero_init(int(capacity), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.lib.qcs_zero_deinit(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def remove(self, rows, sort_frame=False, first_frame=0, end_frame=0, stream=0):
        rows, pr = _host(rows, np.float32)
        n = rows.shape[0]
        check(self.lib.qcs_zero_remove(self.h, pr, n, int(bool(sort_frame)), int(first_frame), int(end_frame),
                                       C.c_void_p(stream) if stream else None))
        k = self.lib.qcs_zero_valid_num(self.h)
        ptr = self.lib.qcs_zero_h_loc_arry(self.h)
        if k == 0:
            return np.zeros((0, 12), np.float32)
        return np.ctypeslib.as_array((C.c_float * (12 * k)).from_address(ptr)).reshape(k, 12).copy()

    def remove_device(self, d_rows, n, d_out, d_n=0, d_nvalid=0, sort_frame=False, first_frame=0, end_frame=0,
                      stream=0):
        check(self.lib.qcs_zero_remove_device(self.h, C.c_void_p(d_rows), int(n), C.c_void_p(d_n) if d_n else None,
                                              int(bool(sort_frame)), int(first_frame), int(end_frame),
                                              C.c_void_p(d_out), C.c_void_p(d_nvalid) if d_nvalid else None,
                                              C.c_void_p(stream) if stream else None))


def learned_in_width(roi_size):
    """Network input width for an R x R ROI (R*R pixels + 2 scale features, padded)."""
    return 64 if roi_size * roi_size + 2 <= 64 else 128


def learned_start_width(loc_type):
    """Start-point floats per record: GS2D 5, AS3D 6, two-emitter GS2D 8, three-emitter GS2D 11."""
    return 11 if loc_type == LEARNED_GS2D_3E else (8 if loc_type == LEARNED_GS2D_2E else (6 if loc_type == 1 else 5))


def learned_out_width(loc_type):
    """Network outputs per record: 8, or 16 for the three-emitter kind."""
    return 16 if loc_type == LEARNED_GS2D_3E else 8


LEARNED_ARCH = {"mlp": 0, "conv": 1}  # QCS_LEARNED_ARCH_MLP, QCS_LEARNED_ARCH_CONV


class LearnedNet:
    """Learned start points (qcs_learned_*) for one localization type and ROI
    size (GS2D or AS3D; 7, 9 or 11): device tensors are torch CUDA tensors.
    arch: "mlp" (the default network) or "conv" (the convolutional one)."""

    def __init__(self, batch=4096, seed=1, loc_type=0, roi_size=7, arch="mlp"):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.qcs_learned_create_arch(LEARNED_ARCH[arch], int(loc_type), int(roi_size), int(batch), int(seed),
                                               C.byref(h)))
        self.h = h
        self.arch = arch
        lt, rs, npar = C.c_int(0), C.c_int(0), C.c_int(0)
        check(self.lib.qcs_learned_shape(h, C.byref(lt), C.byref(rs), C.byref(npar)))
        self.loc_type, self.roi_size, self.n_params = lt.value, rs.value, npar.value

    def close(self):
        """Frees the network.  A two-emitter network still attached to a GS2D
        network is refused (QcsError, QCS_ERR_STATE) and stays usable."""
        if self.h:
            check(self.lib.qcs_learned_destroy(self.h))
            self.h = None
            self._two = None
            self._three = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        out = np.zeros(self.n_params, np.float32)
        check(self.lib.qcs_learned_get_params(self.h, C.c_void_p(out.ctypes.data)))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        check(self.lib.qcs_learned_set_params(self.h, C.c_void_p(p.ctypes.data)))

    def grads(self):
        out = np.zeros(self.n_params, np.float32)
        check(self.lib.qcs_learned_get_grads(self.h, C.c_void_p(out.ctypes.data)))
        return out

    @staticmethod
    def features(para, d_rois, n, stream=0):
        import torch
        feat = torch.empty((n, learned_in_width(para.ROISize)), dtype=torch.float32, device="cuda")
        scale = torch.empty((n, 2), dtype=torch.float32, device="cuda")
        check(load().qcs_learned_features_device(C.byref(para), C.c_void_p(d_rois), int(n), C.c_void_p(feat.data_ptr()),
                                                 C.c_void_p(scale.data_ptr()), C.c_void_p(stream) if stream else None))
        return feat, scale

    @staticmethod
    def targets(para, d_rois, d_rows, scale, n, stream=0):
        import torch
        t = torch.empty((n, 6 if para.LocType == 1 else 5), dtype=torch.float32, device="cuda")
        v = torch.empty((n,), dtype=torch.float32, device="cuda")
        check(load().qcs_learned_targets_device(C.byref(para), C.c_void_p(d_rois), C.c_void_p(d_rows),
                                                C.c_void_p(scale.data_ptr()), int(n), C.c_void_p(t.data_ptr()),
                                                C.c_void_p(v.data_ptr()), C.c_void_p(stream) if stream else None))
        return t, v

    def forward(self, feat, stream=0):
        import torch
        n = feat.shape[0]
        out = torch.empty((n, learned_out_width(self.loc_type)), dtype=torch.float32, device="cuda")
        check(self.lib.qcs_learned_forward_device(self.h, C.c_void_p(feat.data_ptr()), int(n),
                                                  C.c_void_p(out.data_ptr()), C.c_void_p(stream) if stream else None))
        return out

    def gradient(self, feat, tgt, valid, stream=0, classes=None):
        """Loss and gradient of one batch; classes: emitter-count labels (float, -1 = none) or None."""
        loss = C.c_float(0)
        check(self.lib.qcs_learned_gradient_counts_device(
            self.h, C.c_void_p(feat.data_ptr()), C.c_void_p(tgt.data_ptr()), C.c_void_p(valid.data_ptr()),
            C.c_void_p(classes.data_ptr()) if classes is not None else None, int(feat.shape[0]), C.byref(loss),
            C.c_void_p(stream) if stream else None))
        return loss.value

    def train(self, feat, tgt, valid, epochs, lr=1e-3, seed=7, stream=0, classes=None):
        losses = np.zeros(epochs, np.float32)
        check(self.lib.qcs_learned_train_counts_device(
            self.h, C.c_void_p(feat.data_ptr()), C.c_void_p(tgt.data_ptr()), C.c_void_p(valid.data_ptr()),
            C.c_void_p(classes.data_ptr()) if classes is not None else None, int(feat.shape[0]), int(epochs),
            C.c_float(lr), int(seed), C.c_void_p(losses.ctypes.data), C.c_void_p(stream) if stream else None))
        return losses

    def set_count_threshold(self, th):
        """Emitter-count routing threshold (0: route by the WLE classes alone)."""
        check(self.lib.qcs_learned_set_count_threshold(self.h, C.c_float(th)))

    def set_two_emitter(self, two, iters=3, bisections=6, dev_th=0.0, fallback="3e"):
        """Start the two-emitter fits of learned multi-emitter calls from the
        LEARNED_GS2D_2E network `two` (None detaches); poor fits go on to the
        three-emitter fit (fallback "3e"), are refitted plainly ("plain"), or keep
        their own result ("none")."""
        modes = {"3e": 0, "plain": 1, "none": 2}  # QCS_TWO_FALLBACK_3E, _PLAIN, _NONE
        if fallback not in modes:
            raise ValueError("fallback: '3e', 'plain' or 'none'")
        check(self.lib.qcs_learned_set_two_emitter(self.h, two.h if two is not None else None, int(iters),
                                                   int(bisections), C.c_float(dev_th), modes[fallback]))
        self._two = two

    def autotune(self, ctx, d_rois, n, d_wle=0, para=None, stream=0):
        """qcs_learned_autotune: (iterations, line-search steps) of the fastest schedule whose acceptance is
        within 0.5 points of the best."""
        para = para or ctx.para
        it, nb = C.c_int(0), C.c_int(0)
        check(self.lib.qcs_learned_autotune(ctx.h, self.h, C.c_void_p(d_rois), C.c_void_p(d_wle) if d_wle else None,
                                            C.byref(para), int(n), C.byref(it), C.byref(nb),
                                            C.c_void_p(stream) if stream else None))
        return it.value, nb.value

    def set_three_emitter(self, three, iters=4, bisections=6, dev_th=0.0):
        """Start the three-emitter fits of learned multi-emitter calls from the
        LEARNED_GS2D_3E network `three` (None detaches); poor fits are refitted
        plainly (dev_th < 0: no refits, the learned fits' results stand)."""
        check(self.lib.qcs_learned_set_three_emitter(self.h, three.h if three is not None else None, int(iters),
                                                     int(bisections), C.c_float(dev_th)))
        self._three = three

    def refits_3e(self, ctx):
        k = C.c_int(0)
        check(self.lib.qcs_learned_refit_3e_num(ctx.h, C.byref(k)))
        return k.value

    def set_single_refits(self, on=True):
        """Single-emitter learned calls: plain refits of the rejected or poor fits (off: their results stand)."""
        check(self.lib.qcs_learned_set_single_refits(self.h, 1 if on else 0))

    def set_direct_two_emitter(self, on=True):
        """Multi-emitter calls: poor bright single fits straight to the two-emitter fit."""
        check(self.lib.qcs_learned_set_direct_two_emitter(self.h, 1 if on else 0))

    def refits_2e(self, ctx):
        k = C.c_int(0)
        check(self.lib.qcs_learned_refit_2e_num(ctx.h, C.byref(k)))
        return k.value

    def count_threshold(self):
        return float(self.lib.qcs_learned_count_threshold(self.h))

    def classes(self, para, d_rois, n, stream=0):
        """Start points (n x 5) and emitter-count classes (n, uint8) of n device records."""
        import torch
        st = torch.empty((n, 5), dtype=torch.float32, device="cuda")
        cls = torch.empty((n,), dtype=torch.uint8, device="cuda")
        check(self.lib.qcs_learned_classes_device(self.h, C.byref(para), C.c_void_p(d_rois), int(n),
                                                  C.c_void_p(st.data_ptr()), C.c_void_p(cls.data_ptr()),
                                                  C.c_void_p(stream) if stream else None))
        return st, cls

    def start(self, para, d_rois, n, stream=0):
        import torch
        st = torch.empty((n, learned_start_width(self.loc_type)), dtype=torch.float32, device="cuda")
        work = torch.empty((int(self.lib.qcs_learned_work_bytes(int(n))) // 4 + 1,), dtype=torch.float32,
                           device="cuda")
        check(self.lib.qcs_learned_start_device(self.h, C.byref(para), C.c_void_p(d_rois), int(n),
                                                C.c_void_p(st.data_ptr()), C.c_void_p(work.data_ptr()),
                                                C.c_void_p(stream) if stream else None))
        return st

    def localize(self, ctx, d_rois, n, d_wle=0, iters=3, dev_th=0.0, para=None, stream=0, bisections=0):
        """qcs_learned_localize_device on a LocContext; rows stay in the context."""
        para = para or ctx.para
        check(self.lib.qcs_learned_localize_device(ctx.h, self.h, C.c_void_p(d_rois), C.c_void_p(d_wle) if d_wle else None,
                                                   C.byref(para), int(n), int(iters), int(bisections),
                                                   C.c_float(dev_th),
                                                   C.c_void_p(stream) if stream else None))

    def localize_n(self, ctx, d_rois, d_wle, d_n, max_n, iters=2, dev_th=0.0, para=None, stream=0, bisections=0):
        """qcs_learned_localize_device_n: record count on the device (multi-emitter fitting)."""
        para = para or ctx.para
        check(self.lib.qcs_learned_localize_device_n(ctx.h, self.h, C.c_void_p(d_rois), C.c_void_p(d_wle),
                                                     C.byref(para), C.c_void_p(d_n), int(max_n), int(iters),
                                                     int(bisections), C.c_float(dev_th),
                                                     C.c_void_p(stream) if stream else None))

    def set_fused(self, fused=True):
        check(self.lib.qcs_learned_set_inference(self.h, int(bool(fused))))

    def fused_status(self):
        check(self.lib.qcs_learned_fused_status(self.h))

    def refits(self, ctx):
        k = C.c_int(0)
        check(self.lib.qcs_learned_refit_num(ctx.h, C.byref(k)))
        return k.value


def fit_from_start(ctx, d_rois, n, d_start, d_wle=0, iters=3, dev_th=0.0, para=None, stream=0, bisections=0,
                   d_classes=0):
    """qcs_fit_from_start_classes_device: GS2D 7x7 fits from given start points (and, with
    multi-emitter fitting on, optional emitter-count classes); rows stay in the context."""
    para = para or ctx.para
    check(load().qcs_fit_from_start_classes_device(ctx.h, C.c_void_p(d_rois), C.c_void_p(d_wle) if d_wle else None,
                                                   C.byref(para), int(n), C.c_void_p(d_start),
                                                   C.c_void_p(d_classes) if d_classes else None, int(iters),
                                                   int(bisections), C.c_float(dev_th),
                                                   C.c_void_p(stream) if stream else None))


LEARNED_GS2D_2E = 16  # network kind of the two-emitter start points
LEARNED_GS2D_3E = 17  # network kind of the three-emitter start points


def set_three_emitter_capture(ctx, on=True):
    """Keep the plain three-emitter fits' parameters of the following calls on ctx."""
    check(load().qcs_loc_set_three_emitter_capture(ctx.h, 1 if on else 0))


def three_emitter_params(ctx):
    """Device pointer of the captured three-emitter parameters (11 floats per 3E-queue slot)."""
    return load().qcs_loc_device_three_emitter_params(ctx.h)


def three_emitter_targets(ctx, para, d_rois, scale, n, stream=0):
    """Targets (n x 11) and valid flags of a LEARNED_GS2D_3E network from the
    plain multi-emitter call just made, with capture on, on ctx over the same n records."""
    import torch
    t = torch.empty((n, 11), dtype=torch.float32, device="cuda")
    v = torch.empty((n,), dtype=torch.float32, device="cuda")
    check(load().qcs_loc_three_emitter_targets_device(ctx.h, C.c_void_p(d_rois), C.byref(para), int(n),
                                                      C.c_void_p(scale.data_ptr()), C.c_void_p(t.data_ptr()),
                                                      C.c_void_p(v.data_ptr()), C.c_void_p(stream) if stream else None))
    return t, v


def two_emitter_targets(ctx, para, d_rois, scale, n, stream=0):
    """Targets (n x 8) and valid flags of a LEARNED_GS2D_2E network from the
    plain multi-emitter call just made on ctx over the same n records."""
    import torch
    t = torch.empty((n, 8), dtype=torch.float32, device="cuda")
    v = torch.empty((n,), dtype=torch.float32, device="cuda")
    check(load().qcs_loc_two_emitter_targets_device(ctx.h, C.c_void_p(d_rois), C.byref(para), int(n),
                                                    C.c_void_p(scale.data_ptr()), C.c_void_p(t.data_ptr()),
                                                    C.c_void_p(v.data_ptr()), C.c_void_p(stream) if stream else None))
    return t, v


def count_labels(ctx, n, stream=0):
    """Emitter-count labels (float, n) of the last multi-emitter call's records on ctx."""
    import torch
    out = torch.empty((n,), dtype=torch.float32, device="cuda")
    check(load().qcs_loc_count_labels_device(ctx.h, int(n), C.c_void_p(out.data_ptr()),
                                             C.c_void_p(stream) if stream else None))
    return out


class ConsecFit:
    """ConsecutiveFit_TypeDef (qcs_consec_*): merges localizations of one
    molecule over consecutive frames, one group of frame-sorted rows per call."""

    def __init__(self, capacity=0):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.qcs_consec_init(int(capacity), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.lib.qcs_consec_deinit(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def fit(self, rows, para, is_end=False, stream=0):
        """One group of host rows; returns (output rows, on-time ratios[10])."""
        rows, pr = _host(rows, np.float32)
        check(self.lib.qcs_consec_fit(self.h, pr, rows.shape[0] if rows.ndim == 2 else 0, int(bool(is_end)),
                                      C.byref(para), C.c_void_p(stream) if stream else None))
        return self._result()

    def fit_device(self, d_rows, n, para, is_end=False, stream=0):
        check(self.lib.qcs_consec_fit_device(self.h, C.c_void_p(d_rows), int(n), int(bool(is_end)), C.byref(para),
                                             C.c_void_p(stream) if stream else None))
        return self.lib.qcs_consec_out_num(self.h)

    def _result(self):
        n = self.lib.qcs_consec_out_num(self.h)
        ptr = self.lib.qcs_consec_h_out_loc_arry(self.h)
        rows = np.ctypeslib.as_array((C.c_float * (12 * n)).from_address(ptr)).reshape(n, 12).copy() if n else \
            np.zeros((0, 12), np.float32)
        return rows, self.ontime_ratio()

    def ontime_ratio(self):
        """The last call's 10 on-time ratios (input of Statistics.update_ontime)."""
        on = np.zeros(10, np.float32)
        check(self.lib.qcs_consec_ontime_ratio(self.h, C.c_void_p(on.ctypes.data)))
        return on

    def device_rows(self):
        return self.lib.qcs_consec_d_out_loc_arry(self.h)

    def read_rows(self):
        """The last call's output rows copied from the device."""
        n = self.lib.qcs_consec_out_num(self.h)
        out = np.zeros((n, 12), np.float32)
        if n:
            check(self.lib.qcs_consec_read_rows(self.h, C.c_void_p(out.ctypes.data)))
        return out


# qcs_stat_series indices (QCS_STAT_SERIES_* in qcstorm_b200.h)
STAT_SERIES_PHOTON, STAT_SERIES_PREC, STAT_SERIES_SNR, STAT_SERIES_BKG = 0, 1, 2, 3
STAT_SERIES_PSF, STAT_SERIES_PSF_CTL, STAT_SERIES_DENSITY = 4, 5, 6
STAT_SERIES_ONTIME_F1 = 7  # .. 10: ratios of on times of 1, 2, 3 and >= 4 frames
STAT_SERIES = 11


class Statistics:
    """FluoStatisticData_TypeDef (qcs_stat_*): histograms, means, activation
    density and their time series over the localization rows of each call."""

    def __init__(self, capacity=0):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.qcs_stat_init(int(capacity), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.lib.qcs_stat_deinit(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self):
        check(self.lib.qcs_stat_reset_all(self.h))

    def update(self, rows, para, stream=0):
        rows, pr = _host(rows, np.float32)
        check(self.lib.qcs_stat_get_statistical_inf(self.h, pr, rows.shape[0], C.byref(para),
                                                    C.c_void_p(stream) if stream else None))
        return self.result()

    def update_device(self, d_rows, n, para, stream=0):
        check(self.lib.qcs_stat_get_statistical_inf_device(self.h, C.c_void_p(d_rows), int(n), C.byref(para),
                                                           C.c_void_p(stream) if stream else None))
        return self.result()

    def result(self):
        """(histograms [4, 1600], means [10])."""
        hist = np.zeros((4, 1600), np.int32)
        means = np.zeros(10, np.float32)
        check(self.lib.qcs_stat_histograms(self.h, C.c_void_p(hist.ctypes.data)))
        check(self.lib.qcs_stat_means(self.h, C.c_void_p(means.ctypes.data)))
        return hist, means

    def update_ontime(self, ratios):
        """UpdateOntimeRatio on the 10 on-time ratios of a consecutive-frame
        merge (ConsecFit.fit's second result): (mean on time in frames, the 10
        ratios as shown, entries 0..3 folded and clamped)."""
        r = np.ascontiguousarray(ratios, np.float32).reshape(-1)
        if r.size != 10:
            raise ValueError("UpdateOntimeRatio takes 10 on-time ratios")
        check(self.lib.qcs_stat_update_ontime_ratio(self.h, C.c_void_p(r.ctypes.data)))
        return self.ontime()

    def ontime(self):
        m = C.c_float()
        out = np.zeros(10, np.float32)
        check(self.lib.qcs_stat_ontime(self.h, C.byref(m), C.c_void_p(out.ctypes.data)))
        return m.value, out

    def series(self, which):
        n = self.lib.qcs_stat_series(self.h, int(which), None, 0)
        out = np.zeros(max(n, 0), np.float32)
        if n > 0:
            self.lib.qcs_stat_series(self.h, int(which), C.c_void_p(out.ctypes.data), n)
        return out


class RenderContext:
    """Super-resolution render (qcs_render_*): SR image, colour map (3D), display maximum and histogram."""

    def __init__(self, para, capacity=0):
        self.lib = load()
        self.para = para
        h = C.c_void_p()
        check(self.lib.qcs_render_init(C.byref(para), int(capacity), C.byref(h)))
        self.h = h.value

    def close(self):
        if self.h:
            self.lib.qcs_render_deinit(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self, stream=0, display=True):
        """Images to zero (and, with display, the maximum and histogram)."""
        st = C.c_void_p(stream) if stream else None
        check(self.lib.qcs_render_reset(self.h, st))
        if display:
            check(self.lib.qcs_render_reset_max(self.h, st))

    def render(self, rows, mode=0, fixed_prec=0.0, para=None, stream=0):
        """qcs_render_rows on host rows (n x 12)."""
        para = para or self.para
        rows, pr = _host(rows, np.float32)
        check(self.lib.qcs_render_rows(self.h, pr, C.byref(para), int(mode), C.c_float(fixed_prec), rows.shape[0],
                                       C.c_void_p(stream) if stream else None))

    def render_device(self, d_rows, d_n, max_n, mode=0, fixed_prec=0.0, para=None, stream=0):
        """qcs_render_rows_device: rows and (optionally) their count in device memory."""
        para = para or self.para
        check(self.lib.qcs_render_rows_device(self.h, C.c_void_p(d_rows), C.c_void_p(d_n) if d_n else None,
                                              int(max_n), C.byref(para), int(mode), C.c_float(fixed_prec),
                                              C.c_void_p(stream) if stream else None))

    def read(self, stream=0):
        """(image, colormap or None, max, hist) on the host."""
        shape = (self.para.SRImageHigh, self.para.SRImageWidth)
        img = np.zeros(shape, np.float32)
        is3d = self.para.LocType != 0
        cmap = np.zeros(shape, np.float32) if is3d else None
        mx = C.c_int(0)
        hist = np.zeros(400, np.int32)
        check(self.lib.qcs_render_read(self.h, C.c_void_p(img.ctypes.data),
                                       C.c_void_p(cmap.ctypes.data) if is3d else None, C.byref(mx),
                                       C.c_void_p(hist.ctypes.data), C.c_void_p(stream) if stream else None))
        return img, cmap, mx.value, hist


class LocFile:
    """Localization file: 12 float32 per row (qcs_locfile_*)."""

    def __init__(self, path, append=False, capacity=0):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.qcs_locfile_open(os.fsencode(path), int(bool(append)), int(capacity), C.byref(h)))
        self.h = h.value

    def write(self, rows):
        rows, pr = _host(rows, np.float32)
        check(self.lib.qcs_locfile_write(self.h, pr, int(rows.shape[0])))

    def write_device(self, d_rows, d_n, max_n, stream=0):
        check(self.lib.qcs_locfile_write_device(self.h, C.c_void_p(d_rows), C.c_void_p(d_n) if d_n else None,
                                                int(max_n), C.c_void_p(stream) if stream else None))

    def flush(self):
        check(self.lib.qcs_locfile_flush(self.h))

    def rows(self):
        return int(self.lib.qcs_locfile_rows(self.h))

    def close(self):
        if self.h:
            h, self.h = self.h, None
            check(self.lib.qcs_locfile_close(h))
