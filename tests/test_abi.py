"""The C ABI: the library loads without a GPU and exports every function that
include/dvc_b200.h declares; no compute call is made here."""
import ctypes
import os
import re

from dvc_b200 import build, native

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "dvc_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(dvc_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for must in ("dvc_create", "dvc_destroy", "dvc_last_error", "dvc_ldpca_decode", "dvc_LdpcaDecoder",
                 "dvc_decode_wz_frames", "dvc_session_create", "dvc_server_create", "dvc_ldpca_decode_noalloc",
                 "dvc_ldpca_encode"):
        assert must in names, must


def test_library_exports_every_declared_function():
    if not os.path.exists(build.LIB):
        build.build()
    lib = ctypes.CDLL(build.LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding declares the same library
    assert native.lib() is not None
