"""ctypes binding of libtomotopy_b200.so (the C ABI in include/tomotopy_b200.h).

The library is the product path: if it is missing and cannot be built here,
importing this module raises -- there is no CPU fallback.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtomotopy_b200.so")

TMT_OK = 0
STATUS_NAMES = {
    0: "TMT_OK", -1: "TMT_ERR_INVALID_ARGUMENT", -2: "TMT_ERR_CUDA", -3: "TMT_ERR_OUT_OF_MEMORY",
    -4: "TMT_ERR_STATE", -5: "TMT_ERR_UNSUPPORTED", -6: "TMT_ERR_CANCELLED", -7: "TMT_ERR_TIMEOUT",
    -8: "TMT_ERR_INTERNAL",
}
SAMPLER_AUTO, SAMPLER_DENSE, SAMPLER_SPARSE = 0, 1, 2
LEN_POISSON, LEN_LOGNORMAL = 0, 1


class TmtConfig(C.Structure):
    _fields_ = [("K", C.c_uint32), ("V", C.c_uint32), ("alpha", C.POINTER(C.c_float)),
                ("alpha_scalar", C.c_float), ("eta", C.c_float), ("seed", C.c_uint64),
                ("optim_interval", C.c_uint32), ("burn_in", C.c_uint32), ("device", C.c_int32),
                ("sampler", C.c_int32), ("hbm_budget", C.c_uint64), ("sweep_groups", C.c_uint32)]


class TmtInfo(C.Structure):
    _fields_ = [("D", C.c_uint64), ("N_all", C.c_uint64), ("N", C.c_uint64), ("global_step", C.c_uint64),
                ("device_bytes", C.c_uint64), ("K", C.c_uint32), ("V", C.c_uint32), ("sampler", C.c_int32),
                ("last_sweep_ms", C.c_float), ("kernel_launches", C.c_uint64),
                ("sweep_kernel_ms", C.c_double), ("sweeps_timed", C.c_uint32), ("sweep_groups", C.c_uint32),
                ("train_ms", C.c_double), ("rank", C.c_uint32), ("world", C.c_uint32)]


class TmtServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_slots", C.c_uint32), ("token_budget", C.c_uint64),
                ("step_token_sweeps", C.c_uint32), ("max_doc_len", C.c_uint32)]


ALLREDUCE_FN = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32, C.c_void_p)
TMT_I32, TMT_F64 = 0, 1


class TmtShard(C.Structure):
    _fields_ = [("rank", C.c_uint32), ("world", C.c_uint32), ("D_global", C.c_uint64), ("doc_begin", C.c_uint64),
                ("doc_len_global", C.c_void_p), ("allreduce", ALLREDUCE_FN), ("user", C.c_void_p)]


class TmtServerStats(C.Structure):
    _fields_ = [("steps", C.c_uint64), ("completed", C.c_uint64), ("queued", C.c_uint64),
                ("mean_active", C.c_double), ("tokens_in_flight_max", C.c_uint64),
                ("token_sweeps", C.c_uint64), ("alg_bytes", C.c_double), ("kernel_ms", C.c_double),
                ("busy_ms", C.c_double)]


class TmtModelArgs(C.Structure):
    _fields_ = [("K", C.c_uint32), ("alpha", C.POINTER(C.c_float)), ("n_alpha", C.c_uint32), ("eta", C.c_float),
                ("seed", C.c_uint64), ("min_cf", C.c_uint64), ("min_df", C.c_uint64), ("rm_top", C.c_uint64),
                ("device", C.c_int32), ("sweep_groups", C.c_uint32), ("tw", C.c_int32)]


class TmtModelInfo(C.Structure):
    _fields_ = [("K", C.c_uint32), ("V", C.c_uint32), ("n_vocab", C.c_uint32), ("n_docs", C.c_uint64),
                ("N", C.c_uint64), ("global_step", C.c_uint64), ("prepared", C.c_int32), ("alpha", C.c_float),
                ("eta", C.c_float), ("optim_interval", C.c_uint32), ("burn_in", C.c_uint32), ("seed", C.c_uint64),
                ("min_cf", C.c_uint64), ("min_df", C.c_uint64), ("rm_top", C.c_uint64), ("tw", C.c_int32),
                ("weighted_n", C.c_double)]


class TmtSynthSpec(C.Structure):
    _fields_ = [("V", C.c_uint32), ("T", C.c_uint32), ("D", C.c_uint64), ("len_kind", C.c_int32),
                ("len_a", C.c_double), ("len_b", C.c_double), ("len_min", C.c_uint32), ("len_max", C.c_uint32),
                ("doc_alpha", C.c_double), ("topic_beta", C.c_double), ("zipf_s", C.c_double),
                ("seed", C.c_uint64), ("threads", C.c_uint32), ("doc_offset", C.c_uint64)]


_P = C.c_void_p
_H = C.c_void_p
SIGNATURES = {
    "tmt_create": (C.c_int, [C.POINTER(TmtConfig), C.POINTER(_H)]),
    "tmt_upload_corpus": (C.c_int, [_H, _P, _P, C.c_uint64, _P]),
    "tmt_upload_corpus_weighted": (C.c_int, [_H, _P, _P, C.c_uint64, _P, _P]),
    "tmt_download_counts_f32": (C.c_int, [_H, _P, _P, _P, _P]),
    "tmt_train": (C.c_int, [_H, C.c_uint32, C.c_uint32, _P]),
    "tmt_ll": (C.c_int, [_H, _P, _P]),
    "tmt_set_counts": (C.c_int, [_H, _P, _P]),
    "tmt_set_counts_f32": (C.c_int, [_H, _P, _P]),
    "tmt_set_word_priors": (C.c_int, [_H, C.c_uint32, _P, _P]),
    "tmt_set_doc_topic_mask": (C.c_int, [_H, _P]),
    "tmt_set_doc_alpha": (C.c_int, [_H, C.c_uint32, _P, _P]),
    "tmt_set_alpha": (C.c_int, [_H, _P]),
    "tmt_corpus_counts": (C.c_int, [C.c_uint64, _P, _P, C.c_uint32, _P, _P]),
    "tmt_prepare_corpus_counted": (C.c_int, [C.c_uint64, _P, _P, C.c_uint32, _P, _P, C.c_uint64, C.c_uint64,
                                             C.c_uint64, _P, _P, _P, C.POINTER(C.c_uint32)]),
    "tmt_plan_shard": (C.c_int, [_P, C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint64, _P, _P, _P, _P]),
    "tmt_upload_shard": (C.c_int, [_H, _P, _P, C.c_uint64, _P, C.POINTER(TmtShard)]),
    "tmt_set_global_step": (C.c_int, [_H, C.c_uint64]),
    "tmt_set_seed": (C.c_int, [_H, C.c_uint64]),
    "tmt_set_graphs": (C.c_int, [_H, C.c_int32]),
    "tmt_set_doc_rows": (C.c_int, [_H, C.c_uint64, _P]),
    "tmt_set_doc_split": (C.c_int, [_H, C.c_uint64, C.c_uint32]),
    "tmt_get_doc_split": (C.c_int, [_H, _P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "tmt_get_sweep_variants": (C.c_int, [_H, _P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "tmt_get_sweep_timings": (C.c_int, [_H, _P, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "tmt_set_optim": (C.c_int, [_H, C.c_uint32, C.c_uint32]),
    "tmt_infer_batch": (C.c_int, [_H, _P, _P, C.c_uint64, C.c_uint32, C.c_uint64, _P, _P, _P]),
    "tmt_infer_batch_weighted": (C.c_int, [_H, _P, _P, C.c_uint64, _P, C.c_uint32, C.c_uint64, _P, _P, _P]),
    "tmt_download_state": (C.c_int, [_H, _P, _P, _P, _P]),
    "tmt_download_doc_topic": (C.c_int, [_H, _P]),
    "tmt_get_info": (C.c_int, [_H, C.POINTER(TmtInfo)]),
    "tmt_last_error": (C.c_char_p, [_H]),
    "tmt_destroy": (None, [_H]),
    "tmt_prepare_corpus": (C.c_int, [C.c_uint64, _P, _P, C.c_uint32, C.c_uint64, C.c_uint64, C.c_uint64,
                                     _P, _P, _P, _P, _P, C.POINTER(C.c_uint32)]),
    "tmt_prepare_corpus_device": (C.c_int, [C.c_int32, C.c_uint64, _P, _P, C.c_uint32, C.c_uint64, C.c_uint64,
                                            C.c_uint64, _P, _P, _P, _P, _P, C.POINTER(C.c_uint32), C.c_char_p,
                                            C.c_uint64]),
    "tmt_ll_counts_noalloc": (C.c_int, [_P, C.c_uint64, C.c_uint32, _P, _P, _P, C.c_uint32, _P, C.c_float, _P, _P,
                                        C.c_char_p, C.c_size_t]),
    "tmt_server_start": (C.c_int, [C.POINTER(TmtServerConfig), C.POINTER(_H)]),
    "tmt_server_add_model": (C.c_int, [_H, C.c_uint32, C.c_uint32, _P, C.c_float, _P, _P, C.POINTER(C.c_uint32)]),
    "tmt_server_set_model_priors": (C.c_int, [_H, C.c_uint32, C.c_uint32, _P, _P]),
    "tmt_server_add_model_f32": (C.c_int, [_H, C.c_uint32, C.c_uint32, _P, C.c_float, _P, _P, C.POINTER(C.c_uint32)]),
    "tmt_server_submit_weighted": (C.c_int, [_H, C.c_uint32, _P, _P, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64,
                                             C.POINTER(C.c_uint64)]),
    "tmt_server_submit_batch_weighted": (C.c_int, [_H, _P, _P, _P, _P, C.c_uint64, C.c_uint32, C.c_uint64, _P, _P]),
    "tmt_server_submit": (C.c_int, [_H, C.c_uint32, _P, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64,
                                    C.POINTER(C.c_uint64)]),
    "tmt_server_poll": (C.c_int, [_H, C.c_uint32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), _P, C.c_uint32,
                                  C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "tmt_server_submit_batch": (C.c_int, [_H, _P, _P, _P, C.c_uint64, C.c_uint32, C.c_uint64, _P, _P]),
    "tmt_server_poll_batch": (C.c_int, [_H, C.c_uint32, C.c_uint64, _P, _P, _P, C.c_uint32, _P, _P,
                                        C.POINTER(C.c_uint64)]),
    "tmt_server_get_stats": (C.c_int, [_H, C.POINTER(TmtServerStats)]),
    "tmt_server_last_error": (C.c_char_p, [_H]),
    "tmt_server_stop": (C.c_int, [_H]),
    "tmt_model_create": (C.c_int, [C.POINTER(TmtModelArgs), C.POINTER(_H)]),
    "tmt_model_add_doc": (C.c_int, [_H, C.c_char_p, C.c_uint32, C.POINTER(C.c_int64)]),
    "tmt_model_prepare": (C.c_int, [_H]),
    "tmt_model_set_word_prior": (C.c_int, [_H, C.c_char_p, _P, C.c_uint32]),
    "tmt_model_get_word_prior": (C.c_int, [_H, C.c_char_p, _P, C.POINTER(C.c_uint32)]),
    "tmt_model_train": (C.c_int, [_H, C.c_uint32]),
    "tmt_model_set_optim": (C.c_int, [_H, C.c_uint32, C.c_uint32]),
    "tmt_model_set_seed": (C.c_int, [_H, C.c_uint64]),
    "tmt_model_get_info": (C.c_int, [_H, C.POINTER(TmtModelInfo)]),
    "tmt_model_ll": (C.c_int, [_H, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "tmt_model_alpha": (C.c_int, [_H, _P]),
    "tmt_model_topic_word_dist": (C.c_int, [_H, C.c_uint32, C.c_int, _P]),
    "tmt_model_count_by_topics": (C.c_int, [_H, _P]),
    "tmt_model_vocab": (C.c_int, [_H, C.c_uint32, _P, C.c_uint64, C.POINTER(C.c_uint64)]),
    "tmt_model_vocab_freq": (C.c_int, [_H, _P, _P]),
    "tmt_model_doc": (C.c_int, [_H, C.c_uint64, _P, _P, C.POINTER(C.c_uint32)]),
    "tmt_model_doc_topic_dist": (C.c_int, [_H, C.c_uint64, C.c_int, _P, C.POINTER(C.c_double)]),
    "tmt_model_infer": (C.c_int, [_H, C.c_char_p, _P, C.c_uint64, C.c_uint32, C.c_uint64, _P, _P]),
    "tmt_model_infer_together": (C.c_int, [_H, C.c_char_p, _P, C.c_uint64, C.c_uint32, C.c_uint64, _P, _P]),
    "tmt_model_save": (C.c_int, [_H, _P, C.c_uint64, C.c_int, C.POINTER(C.POINTER(C.c_uint8)), C.POINTER(C.c_uint64)]),
    "tmt_model_free_buffer": (None, [C.POINTER(C.c_uint8)]),
    "tmt_model_load": (C.c_int, [_P, C.c_uint64, C.c_int32, C.c_uint32, C.POINTER(_H), C.POINTER(C.POINTER(C.c_uint8)),
                                 C.POINTER(C.c_uint64)]),
    "tmt_model_last_error": (C.c_char_p, [_H]),
    "tmt_model_destroy": (None, [_H]),
    "tmt_synth_corpus": (C.c_int, [C.POINTER(TmtSynthSpec), _P, _P, C.c_uint64, C.POINTER(C.c_uint64)]),
}


def _load():
    if not os.path.exists(LIB_PATH):
        try:
            from . import build as _b
            _b.build()
        except Exception as e:  # no nvcc, no prebuilt library: fail loudly
            raise ImportError(f"libtomotopy_b200.so is missing and could not be built: {e}") from e
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


class TmtError(RuntimeError):
    def __init__(self, status, msg):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")


def check(status, handle=None, what=""):
    if status != TMT_OK:
        msg = lib.tmt_last_error(handle).decode() if handle else what
        if status == -1:
            raise ValueError(msg)
        raise TmtError(status, msg or what)
