"""CPU test: the packed table of the belief-propagation magnitude
phi(y) = -logf(tanhf(y)) returns the C library's bits for every float
argument the LDPCA decoder can form (the library packs and checks the whole
sweep, as dvc_create does before uploading it)."""
import ctypes as C

from dvc_b200 import native


def test_packed_phi_table_matches_the_library_everywhere():
    L = native.lib()
    size = C.c_size_t(0)
    msg = C.create_string_buffer(256)
    rc = L.dvc_phi_table_check(C.byref(size), msg, 256)
    assert rc == 0, msg.value.decode()
    # 2.9e8 entries packed into well under the 1.1 GB of a direct table
    assert 0 < size.value < 256 * 2**20, size.value
