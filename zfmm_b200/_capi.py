"""ctypes binding of libzfmm_b200.so (include/zfmm.h).

The library is built in-tree (python -m zfmm_b200.build).  Loading fails
loudly when the library is missing: there is no CPU fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libzfmm_b200.so")

_lib = None

c_int = ctypes.c_int
c_double = ctypes.c_double
c_void_p = ctypes.c_void_p
c_int_p = ctypes.POINTER(ctypes.c_int)

# name -> (restype, argtypes), in include/zfmm.h order
SIGNATURES = {
    "zlfmm2d_": (None, [c_void_p] * 15),
    "zl2devaldirect_": (None, [c_void_p] * 12),
    "zfmm_zlfmm2d": (c_int, [c_double, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p,
                             c_void_p, c_void_p, c_int, c_void_p, c_int, c_int, c_int]),
    "zfmm_zl2devaldirect": (c_int, [c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                    c_void_p, c_int, c_void_p, c_void_p, c_int, c_int]),
    "zfmm_zlfmm2d_dev": (c_int, [c_double, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p,
                                 c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, c_int,
                                 c_void_p]),
    "zfmm_zl2devaldirect_dev": (c_int, [c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                        c_void_p, c_int, c_void_p, c_void_p, c_int, c_int,
                                        c_void_p]),
    "zfmm_zl2devaldirect_dev_noalloc": (c_int, [c_int, c_void_p, c_int, c_void_p, c_void_p,
                                                c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                                                c_int, c_int, c_void_p]),
    "zfmm_zl2devaldirect_noalloc_capacity": (ctypes.c_long, []),
    "zfmm_tc_selftest": (c_int, [c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    "zfmm_set_autotune": (None, [c_int]),
    "zfmm_autotune_entries": (c_int, []),
    "zfmm_autotune_save": (c_int, [ctypes.c_char_p]),
    "zfmm_autotune_load": (c_int, [ctypes.c_char_p]),
    "zfmm_plan2d_save": (c_int, [c_void_p, ctypes.c_char_p]),
    "zfmm_plan2d_load": (c_int, [ctypes.c_char_p, c_void_p]),
    "zfmm_plan3d_save": (c_int, [c_void_p, ctypes.c_char_p]),
    "zfmm_plan3d_load": (c_int, [ctypes.c_char_p, c_void_p]),
    "zhfmm2d_": (None, [c_void_p] * 16),
    "zh2devaldirect_": (None, [c_void_p] * 13),
    "zfmm_zhfmm2d": (c_int, [c_double, c_void_p, c_int, c_void_p, c_int, c_void_p, c_int,
                             c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int,
                             c_int, c_int]),
    "zfmm_zhfmm2d_dev": (c_int, [c_double, c_void_p, c_int, c_void_p, c_int, c_void_p, c_int,
                                 c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int,
                                 c_int, c_void_p]),
    "zfmm_zh2devaldirect": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p,
                                    c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int, c_int]),
    "zfmm_zh2devaldirect_dev": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p,
                                        c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int,
                                        c_int, c_void_p]),
    "zlfmm3d_": (None, [c_void_p] * 15),
    "zl3devaldirect_": (None, [c_void_p] * 12),
    "zfmm_zlfmm3d": (c_int, [c_double, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p,
                             c_void_p, c_void_p, c_int, c_void_p, c_int, c_int, c_int]),
    "zfmm_zl3devaldirect": (c_int, [c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                    c_void_p, c_int, c_void_p, c_void_p, c_int, c_int]),
    "zfmm_zlfmm3d_dev": (c_int, [c_double, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p,
                                 c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int, c_int,
                                 c_void_p]),
    "zfmm_zl3devaldirect_dev": (c_int, [c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                        c_void_p, c_int, c_void_p, c_void_p, c_int, c_int,
                                        c_void_p]),
    "zfmm_zl3dterms": (c_int, [c_double]),
    "zhfmm3d_": (None, [c_void_p] * 16),
    "zh3devaldirect_": (None, [c_void_p] * 13),
    "zfmm_zhfmm3d": (c_int, [c_double, c_void_p, c_int, c_void_p, c_int, c_void_p, c_int,
                             c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int,
                             c_int, c_int]),
    "zfmm_zh3devaldirect": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p,
                                    c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int, c_int]),
    "zfmm_zhfmm3d_dev": (c_int, [c_double, c_void_p, c_int, c_void_p, c_int, c_void_p, c_int,
                                 c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_int,
                                 c_int, c_void_p]),
    "zfmm_zh3devaldirect_dev": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p,
                                        c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int,
                                        c_int, c_void_p]),
    "zfmm_h3dterms": (c_int, [c_double, c_void_p, c_double, c_int]),
    "zfmm_set_step_timing": (None, [c_int]),
    "zfmm_last_step_times": (c_int, [c_void_p, c_int_p, c_int_p, c_int_p]),
    "zfmm_last_counts": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_long)]),
    "zfmm_launch_count": (ctypes.c_long, []),
    "zfmm_last_level_counts": (c_int, [c_void_p, c_void_p, c_int_p]),
    "zfmm_trim_pool": (ctypes.c_int, []),
    "zfmm_h2dterms": (c_int, [c_double, c_void_p, c_double, c_int]),
    "zfmm_tree_dump": (c_int, [c_int, c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_int, c_int,
                               c_int_p, c_int_p] + [c_void_p] * 12 + [c_int_p, c_void_p]),
    "zfmm_plan3d_create": (c_int, [c_double, c_int, c_void_p, c_int, c_void_p, c_int,
                                   ctypes.POINTER(c_void_p)]),
    "zfmm_plan3d_create_dev": (c_int, [c_double, c_int, c_void_p, c_int, c_void_p, c_int,
                                       c_void_p, ctypes.POINTER(c_void_p)]),
    "zfmm_plan3d_destroy": (c_int, [c_void_p]),
    "zfmm_plan3d_info": (c_int, [c_void_p, c_int_p, c_int_p, c_int_p, c_int_p]),
    "zfmm_zlfmm3d_plan": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p,
                                  c_int, c_void_p, c_void_p]),
    "zfmm_zlfmm3d_plan_dev": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p,
                                      c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "zfmm_zhfmm3d_plan": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_int, c_void_p,
                                  c_void_p, c_int, c_void_p, c_void_p]),
    "zfmm_zhfmm3d_plan_dev": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_int,
                                      c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "zfmm_plan2d_create": (c_int, [c_double, c_int, c_void_p, c_int, c_void_p, c_int,
                                   ctypes.POINTER(c_void_p)]),
    "zfmm_plan2d_create_dev": (c_int, [c_double, c_int, c_void_p, c_int, c_void_p, c_int,
                                       c_void_p, ctypes.POINTER(c_void_p)]),
    "zfmm_plan2d_destroy": (c_int, [c_void_p]),
    "zfmm_plan2d_info": (c_int, [c_void_p, c_int_p, c_int_p, c_int_p, c_int_p]),
    "zfmm_zlfmm2d_plan": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p, c_void_p,
                                  c_int, c_void_p, c_void_p]),
    "zfmm_zlfmm2d_plan_dev": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p,
                                      c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "zfmm_zhfmm2d_plan": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_int, c_void_p,
                                  c_void_p, c_int, c_void_p, c_void_p]),
    "zfmm_zhfmm2d_plan_dev": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_int,
                                      c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "zfmm_zlfmm3d_many": (c_int, [c_int, c_double, c_void_p, c_void_p, c_int, c_void_p, c_int,
                                  c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p,
                                  c_void_p, c_int, c_void_p]),
    "zfmm_zhfmm3d_many": (c_int, [c_int, c_double, c_void_p, c_void_p, c_void_p, c_int, c_void_p,
                                  c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int,
                                  c_void_p, c_void_p, c_int, c_void_p]),
    "zfmm_zlfmm3d_many_dev": (c_int, [c_int, c_double, c_void_p, c_void_p, c_int, c_void_p,
                                      c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int,
                                      c_void_p, c_void_p, c_int, c_void_p]),
    "zfmm_zhfmm3d_many_dev": (c_int, [c_int, c_double, c_void_p, c_void_p, c_void_p, c_int,
                                      c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                                      c_int, c_int, c_void_p, c_void_p, c_int, c_void_p]),
    "zfmm_probe_fp64_tflops": (c_double, [c_int]),
    "zfmm_probe_dmma_tflops": (c_double, [c_int]),
    "zfmm_last_error": (ctypes.c_char_p, []),
    "zfmm_fail_alloc_after": (None, [ctypes.c_long]),
    "zfmm_version": (ctypes.c_char_p, []),
}


class ZfmmError(RuntimeError):
    pass


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ZfmmError(
                f"{LIB_PATH} is missing: build it with `python -m zfmm_b200.build` "
                "(zfmm_b200 has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        msg = lib().zfmm_last_error().decode()
        raise ZfmmError(f"zfmm status {rc}: {msg}")
