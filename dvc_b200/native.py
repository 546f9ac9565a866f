"""ctypes binding of libdvc_b200.so (the C ABI in include/dvc_b200.h).

The library is built in-tree by ``dvc_b200.build``; importing this module does
not build it.  A missing library or a failing CUDA set-up raises immediately:
there is no CPU fallback.
"""
import ctypes as C
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("DVC_B200_LIB") or os.path.join(HERE, "_lib", "libdvc_b200.so")
DATA_DIR = os.path.join(HERE, "ladders")
TABLE_DIR = os.environ.get("DVC_B200_TABLES", os.path.join(HERE, "_tables"))

DVC_OK, DVC_E_ARG, DVC_E_CUDA, DVC_E_NOMEM, DVC_E_DATA = 0, -1, -2, -3, -4


class DvcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("dvc_b200 error %d: %s" % (code, msg))
        self.code = code


_lib = None
_lock = threading.Lock()


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise FileNotFoundError("libdvc_b200.so not built (%s); run python -m dvc_b200.build" % LIB_PATH)
            L = C.CDLL(LIB_PATH)
            L.dvc_create.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]
            L.dvc_create.restype = C.c_int
            L.dvc_destroy.argtypes = [C.c_void_p]
            L.dvc_destroy.restype = None
            L.dvc_last_error.argtypes = [C.c_void_p]
            L.dvc_last_error.restype = C.c_char_p
            L.dvc_ldpca_decode.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
            L.dvc_ldpca_decode.restype = C.c_int
            L.dvc_LdpcaDecoder.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.POINTER(C.c_int), C.c_ubyte, C.c_float]
            L.dvc_LdpcaDecoder.restype = C.c_int
            L.dvc_session_destroy.argtypes = [C.c_void_p]
            L.dvc_session_destroy.restype = None
            L.dvc_server_destroy.argtypes = [C.c_void_p]
            L.dvc_server_destroy.restype = None
            _declare_frame_api(L)
            _lib = L
    return _lib


def _declare_frame_api(L):
    """Declarations of the frame-level entry points (present once built)."""
    for name, args in FRAME_API.items():
        if hasattr(L, name):
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int


class WZFrame(C.Structure):
    """dvc_wz_frame (include/dvc_b200.h)."""
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("qindex", C.c_int),
                ("past_idx", C.c_int), ("future_idx", C.c_int), ("cur_idx", C.c_int),
                ("past", C.c_void_p), ("future", C.c_void_p), ("mode", C.c_void_p),
                ("skip_mode", C.c_int), ("intra_mode", C.c_int), ("ac_range", C.c_void_p),
                ("crc", C.c_void_p), ("acc_synd", C.c_void_p), ("recon", C.c_void_p),
                ("wz_bits", C.c_int), ("plane_results", C.c_void_p), ("plane_entropy", C.c_void_p),
                ("deblock_flag", C.c_void_p), ("deblock", C.c_int), ("intra_qp", C.c_int),
                ("past_mode", C.c_void_p)]


FRAME_API = {
    "dvc_decode_wz_frames": [C.c_void_p, C.c_int, C.POINTER(WZFrame)],
    "dvc_session_create": [C.c_void_p, C.c_int, C.POINTER(WZFrame), C.c_int, C.c_int, C.POINTER(C.c_void_p)],
    "dvc_session_run": [C.c_void_p, C.c_int, C.POINTER(C.c_double)],
    "dvc_session_frame": [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_int), C.c_void_p],
    "dvc_session_profile": [C.c_void_p, C.c_void_p],
    "dvc_session_replays": [C.c_void_p, C.POINTER(C.c_longlong)],
    "dvc_server_create": [C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.POINTER(C.c_void_p)],
    "dvc_server_submit": [C.c_void_p, C.POINTER(WZFrame), C.POINTER(C.c_longlong)],
    "dvc_server_poll": [C.c_void_p, C.POINTER(C.c_int)],
    "dvc_server_result": [C.c_void_p, C.c_longlong, C.c_void_p, C.POINTER(C.c_int), C.c_void_p,
                          C.POINTER(C.c_double)],
    "dvc_server_config": [C.c_void_p, C.c_int],
    "dvc_server_finished": [C.c_void_p, C.POINTER(C.c_longlong), C.c_int, C.POINTER(C.c_int)],
    "dvc_server_stats": [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.POINTER(C.c_size_t)],
    "dvc_ldpca_decode_noalloc": [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_int, C.c_void_p],
    "dvc_debug_wz_frame": [C.c_void_p, C.POINTER(WZFrame), C.c_void_p, C.c_void_p, C.c_void_p],
    "dvc_debug_wz_frame_lr": [C.c_void_p, C.POINTER(WZFrame), C.c_void_p],
    "dvc_ldpca_decode_batch": [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_longlong),
                               C.POINTER(C.c_double)],
    "dvc_recon_near_ties": [C.c_void_p, C.POINTER(C.c_longlong)],
    "dvc_ldpca_encode": [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p],
    "dvc_phi_table_check": [C.POINTER(C.c_size_t), C.c_char_p, C.c_int],
    "dvc_jbig_encode_mode_map": [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)],
    "dvc_jbig_decode_mode_map": [C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_size_t)],
    "dvc_intra_encode_frame": [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_size_t,
                               C.POINTER(C.c_size_t), C.c_void_p, C.c_void_p],
    "dvc_intra_decode_frame": [C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t), C.c_int, C.c_int, C.c_int, C.c_void_p,
                               C.c_void_p],
}


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _addr(a):
    """The address of an array's data for a pointer field of a ctypes struct
    (the caller keeps the array alive as long as the struct is used)."""
    return None if a is None else a.ctypes.data


class Context:
    """A decoder context on one CUDA device (dvc_create / dvc_destroy)."""

    def __init__(self, device=0, table_dir=None):
        self._h = C.c_void_p()
        td = table_dir or TABLE_DIR
        os.makedirs(td, exist_ok=True)
        rc = lib().dvc_create(DATA_DIR.encode(), td.encode(), device, C.byref(self._h))
        if rc != DVC_OK:
            msg = lib().dvc_last_error(self._h).decode() if self._h else "create failed"
            if self._h:
                lib().dvc_destroy(self._h)
                self._h = C.c_void_p()
            raise DvcError(rc, msg)

    @property
    def handle(self):
        return self._h

    def check(self, rc):
        if rc != DVC_OK:
            raise DvcError(rc, lib().dvc_last_error(self._h).decode())

    def close(self):
        if self._h:
            lib().dvc_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def ldpca_decode(self, lr, acc_bytes, crc, max_iter=50):
        """Batched LDPCA decode. lr: (count, n) float32 p0/p1; acc_bytes: (count, n/8) uint8;
        crc: (count,) uint8. Returns (decoded (count, n) uint8, results (count, 4) int32, entropy (count,))."""
        lr = np.ascontiguousarray(lr, np.float32)
        if lr.ndim == 1:
            lr = lr[None]
        count, n = lr.shape
        acc = np.ascontiguousarray(acc_bytes, np.uint8).reshape(count, n // 8)
        crc = np.ascontiguousarray(crc, np.uint8).reshape(count)
        dec = np.zeros((count, n), np.uint8)
        res = np.zeros((count, 4), np.int32)
        ent = np.zeros(count, np.float32)
        self.check(lib().dvc_ldpca_decode(self._h, n, count, _ptr(lr), _ptr(acc), _ptr(crc), _ptr(dec), _ptr(res),
                                          _ptr(ent), max_iter))
        return dec, res, ent

    def ldpca_decode_batch(self, lengths, lr, acc, crc, start=None, max_iter=50, want_decoded=True):
        """dvc_ldpca_decode_batch: codewords of mixed lengths in one persistent launch.

        lengths: int per codeword (1584 or 6336); lr: float32 LRs of all
        codewords concatenated; acc: accumulated-syndrome bytes concatenated
        (n/8 each); crc: uint8 per codeword; start: first ladder code per
        codeword, or None for the entropy bound.  Returns (decoded bits
        concatenated or None, results [count, 4], entropy [count], BP iterations
        run, kernel milliseconds)."""
        n = np.ascontiguousarray(lengths, np.int32)
        count = len(n)
        lr = np.ascontiguousarray(lr, np.float32)
        acc = np.ascontiguousarray(acc, np.uint8)
        crc = np.ascontiguousarray(crc, np.uint8)
        assert lr.size == int(n.sum()) and acc.size == int(n.sum()) // 8 and crc.size == count
        st = None if start is None else np.ascontiguousarray(start, np.int32)
        dec = np.zeros(int(n.sum()), np.uint8) if want_decoded else None
        res = np.zeros((count, 4), np.int32)
        ent = np.zeros(count, np.float32)
        work = C.c_longlong(0)
        ms = C.c_double(0)
        self.check(lib().dvc_ldpca_decode_batch(self._h, count, _ptr(n), _ptr(lr), _ptr(acc), _ptr(crc), _ptr(st),
                                                _ptr(dec), _ptr(res), _ptr(ent), max_iter, C.byref(work),
                                                C.byref(ms)))
        return dec, res, ent, work.value, ms.value

    def ldpca_decode_noalloc(self, n, count, d_lr, d_acc, d_crc, d_decoded, d_results, d_entropy, max_iter=50,
                             stream=0):
        """dvc_ldpca_decode_noalloc on caller-owned device buffers (integer device addresses);
        enqueues on `stream` and returns without waiting. Returns the status code."""
        return lib().dvc_ldpca_decode_noalloc(self._h, n, count, C.c_void_p(d_lr), C.c_void_p(d_acc),
                                              C.c_void_p(d_crc), C.c_void_p(d_decoded) if d_decoded else None,
                                              C.c_void_p(d_results), C.c_void_p(d_entropy) if d_entropy else None,
                                              max_iter, C.c_void_p(stream) if stream else None)

    def ldpca_encode(self, bits):
        """Device LDPCA encoder. bits: (count, n) 0/1. Returns (accumulated syndrome bytes (count, n/8), crc (count,))."""
        bits = np.ascontiguousarray(bits, np.uint8)
        if bits.ndim == 1:
            bits = bits[None]
        count, n = bits.shape
        acc = np.zeros((count, n // 8), np.uint8)
        crc = np.zeros(count, np.uint8)
        self.check(lib().dvc_ldpca_encode(self._h, n, count, _ptr(bits), _ptr(acc), _ptr(crc)))
        return acc, crc

    def last_error(self):
        return lib().dvc_last_error(self._h).decode()

    def LdpcaDecoder(self, lr, acc_bits, crc, rate_lower_bound):
        """Reference-shaped call: returns (decoded bits, rate, log LR)."""
        lr = np.ascontiguousarray(lr, np.float32).copy()
        acc = np.ascontiguousarray(acc_bits, np.uint8)
        dec = np.zeros(len(lr), np.uint8)
        rate = C.c_int(0)
        self.check(lib().dvc_LdpcaDecoder(self._h, len(lr), _ptr(lr), _ptr(acc), _ptr(dec), C.byref(rate),
                                          C.c_ubyte(int(crc)), C.c_float(rate_lower_bound)))
        return dec, rate.value, lr

    def _frame_array(self, items, copy_recon=True):
        """ctypes frame array.  An item may name another item's decoded output as
        a reference with past_from / future_from (its index); the pointer then
        equals that item's recon pointer, which dvc_session_create resolves.
        copy_recon=False passes the caller's starting content itself, for calls
        that only read it (dvc_server_submit copies its inputs)."""
        keep, arr, outs = [], (WZFrame * len(items))(), []
        recs = [np.zeros((it["height"], it["width"]), np.uint8) if it.get("recon") is None else
                np.array(it["recon"], np.uint8, copy=True if copy_recon else None, order="C") for it in items]
        for i, it in enumerate(items):
            w, h = it["width"], it["height"]
            past = recs[it["past_from"]] if it.get("past_from") is not None else \
                np.ascontiguousarray(it["past"], np.uint8)
            fut = recs[it["future_from"]] if it.get("future_from") is not None else \
                np.ascontiguousarray(it["future"], np.uint8)
            mode = None if it.get("mode") is None else np.ascontiguousarray(it["mode"], np.uint8)
            acr = np.ascontiguousarray(it["ac_range"], np.int32)
            crc = np.ascontiguousarray(it["crc"], np.uint8)
            acc = np.ascontiguousarray(it["acc"], np.uint8)
            rec = recs[i]
            pmode = None if it.get("past_mode") is None else np.ascontiguousarray(it["past_mode"], np.uint8)
            keep += [past, fut, mode, acr, crc, acc, rec, pmode]
            arr[i] = WZFrame(w, h, it["qindex"], it["past_idx"], it["future_idx"], it["cur_idx"], _addr(past),
                             _addr(fut), _addr(mode), it.get("skip_mode", 0), it.get("intra_mode", 0), _addr(acr),
                             _addr(crc), _addr(acc), _addr(rec), 0, None, None, None,
                             it.get("deblock", 0), it.get("intra_qp", 0), _addr(pmode))
            outs.append(len(crc))
        return arr, keep, outs

    def server(self, mem_budget_bytes=16 << 30, streams=8, max_cohort=8, batch_window_us=None):
        """Continuous-batching server (dvc_server_*)."""
        srv = Server(self, mem_budget_bytes, streams, max_cohort)
        if batch_window_us is not None:
            self.check(lib().dvc_server_config(srv._h, batch_window_us))
        return srv

    def session(self, items, max_batch=0, streams=1):
        """Device-resident session (dvc_session_*); items may reference each
        other's outputs through past_from / future_from."""
        return Session(self, items, max_batch, streams)

    def debug_wz_frame(self, item):
        """One frame through dvc_debug_wz_frame: the decode result plus si_initial, alpha, si_final."""
        return self.decode_wz_frames([item], debug=True)[0]

    def debug_wz_frame_lr(self, item):
        """One frame through dvc_debug_wz_frame_lr: the decode result plus "lr",
        the likelihood ratios of every bitplane ([qbits, w*h/16] float32)."""
        return self.decode_wz_frames([item], debug="lr")[0]

    def recon_near_ties(self):
        """dvc_recon_near_ties: reconstruction steps so far whose rounding could depend on exp's last bits."""
        n = C.c_longlong(0)
        self.check(lib().dvc_recon_near_ties(self._h, C.byref(n)))
        return n.value

    def decode_wz_frames(self, items, debug=False):
        """Decode independent WZ frames as one batch.

        items: list of dicts with keys width, height, qindex, past_idx, future_idx,
        cur_idx, past, future (uint8 HxW), mode (uint8 or None), skip_mode, intra_mode,
        ac_range (16 ints), crc (uint8 [qbits]), acc (uint8 [qbits, n/8]), recon
        (uint8 HxW with intra pixels, or None).  Returns a list of dicts with
        recon, wz_bits, planes ([qbits,4] int32), entropy, deblock_flag.
        """
        keep = []
        arr = (WZFrame * len(items))()
        outs = []
        for i, it in enumerate(items):
            w, h = it["width"], it["height"]
            past = np.ascontiguousarray(it["past"], np.uint8)
            fut = np.ascontiguousarray(it["future"], np.uint8)
            mode = None if it.get("mode") is None else np.ascontiguousarray(it["mode"], np.uint8)
            acr = np.ascontiguousarray(it["ac_range"], np.int32)
            crc = np.ascontiguousarray(it["crc"], np.uint8)
            acc = np.ascontiguousarray(it["acc"], np.uint8)
            rec = np.zeros((h, w), np.uint8) if it.get("recon") is None else np.ascontiguousarray(it["recon"], np.uint8).copy()
            qb = len(crc)
            planes = np.zeros((qb, 4), np.int32)
            ent = np.zeros(qb, np.float32)
            dbf = np.zeros((h, w), np.uint8)
            pmode = None if it.get("past_mode") is None else np.ascontiguousarray(it["past_mode"], np.uint8)
            keep += [past, fut, mode, acr, crc, acc, pmode]
            arr[i] = WZFrame(w, h, it["qindex"], it["past_idx"], it["future_idx"], it["cur_idx"], _ptr(past),
                             _ptr(fut), _ptr(mode), it.get("skip_mode", 0), it.get("intra_mode", 0), _ptr(acr),
                             _ptr(crc), _ptr(acc), _ptr(rec), 0, _ptr(planes), _ptr(ent), _ptr(dbf),
                             it.get("deblock", 0), it.get("intra_qp", 0), _ptr(pmode))
            outs.append(dict(recon=rec, planes=planes, entropy=ent, deblock_flag=dbf))
        if debug == "lr":
            w, h = items[0]["width"], items[0]["height"]
            lr = np.zeros((len(items[0]["crc"]), w * h // 16), np.float32)
            self.check(lib().dvc_debug_wz_frame_lr(self._h, arr, _ptr(lr)))
            outs[0]["lr"] = lr
        elif debug:
            w, h = items[0]["width"], items[0]["height"]
            si0 = np.zeros((h, w), np.uint8)
            si1 = np.zeros((h, w), np.uint8)
            alpha = np.zeros((h, w), np.float32)
            self.check(lib().dvc_debug_wz_frame(self._h, arr, _ptr(si0), _ptr(alpha), _ptr(si1)))
            outs[0].update(si_initial=si0, si_final=si1, alpha=alpha)
        else:
            self.check(lib().dvc_decode_wz_frames(self._h, len(items), arr))
        for i, o in enumerate(outs):
            o["wz_bits"] = arr[i].wz_bits
        return outs


class Session:
    """dvc_session: inputs uploaded once, decoded on every run() from device memory."""

    def __init__(self, ctx, items, max_batch=0, streams=1):
        self.ctx = ctx
        arr, keep, self.qbits = ctx._frame_array(items)
        self.w, self.h = items[0]["width"], items[0]["height"]
        self._h = C.c_void_p()
        ctx.check(lib().dvc_session_create(ctx.handle, len(items), arr, max_batch, streams, C.byref(self._h)))
        self.count = len(items)

    def run(self, profile=False):
        ms = C.c_double(0)
        self.ctx.check(lib().dvc_session_run(self._h, 1 if profile else 0, C.byref(ms)))
        return ms.value

    def frame(self, i, recon=True):
        rec = np.zeros((self.h, self.w), np.uint8) if recon else None
        bits = C.c_int(0)
        planes = np.zeros((self.qbits[i], 4), np.int32)
        self.ctx.check(lib().dvc_session_frame(self._h, i, _ptr(rec), C.byref(bits), _ptr(planes)))
        return rec, bits.value, planes

    def replays(self):
        """Runs so far that replayed the captured CUDA graph."""
        n = C.c_longlong(0)
        self.ctx.check(lib().dvc_session_replays(self._h, C.byref(n)))
        return n.value

    def profile(self):
        out = np.zeros(5, np.float64)
        self.ctx.check(lib().dvc_session_profile(self._h, _ptr(out)))
        return dict(ldpca_ms=out[0], ldpca_launches=int(out[1]), ldpca_codewords=int(out[2]),
                    kernel_launches=int(out[3]), runs=int(out[4]))

    def close(self):
        if self._h:
            lib().dvc_session_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """dvc_server: submit() frames from any stream, poll() to schedule, result() to collect."""

    def __init__(self, ctx, mem_budget_bytes, streams, max_cohort):
        self.ctx = ctx
        self._h = C.c_void_p()
        ctx.check(lib().dvc_server_create(ctx.handle, mem_budget_bytes, streams, max_cohort, C.byref(self._h)))
        self._meta = {}

    def submit(self, item):
        arr, keep, qbits = self.ctx._frame_array([item], copy_recon=False)
        t = C.c_longlong(0)
        self.ctx.check(lib().dvc_server_submit(self._h, arr, C.byref(t)))
        self._meta[t.value] = (item["width"], item["height"], qbits[0])
        return t.value

    def poll(self):
        n = C.c_int(0)
        self.ctx.check(lib().dvc_server_poll(self._h, C.byref(n)))
        return n.value

    def result(self, ticket):
        """Result of a finished ticket; raises DvcError if it has not finished."""
        w, h, qb = self._meta[ticket]
        rec = np.zeros((h, w), np.uint8)
        bits = C.c_int(0)
        planes = np.zeros((qb, 4), np.int32)
        lat = C.c_double(0)
        self.ctx.check(lib().dvc_server_result(self._h, ticket, _ptr(rec), C.byref(bits), _ptr(planes), C.byref(lat)))
        del self._meta[ticket]
        return dict(recon=rec, wz_bits=bits.value, planes=planes, latency_ms=lat.value)

    def finished(self, cap=4096):
        """Tickets of finished requests not yet collected."""
        buf = (C.c_longlong * cap)()
        n = C.c_int(0)
        self.ctx.check(lib().dvc_server_finished(self._h, buf, cap, C.byref(n)))
        return [buf[i] for i in range(n.value)]

    def stats(self):
        p, f, b = C.c_longlong(0), C.c_longlong(0), C.c_size_t(0)
        self.ctx.check(lib().dvc_server_stats(self._h, C.byref(p), C.byref(f), C.byref(b)))
        return dict(pending=p.value, in_flight=f.value, bytes_in_flight=b.value)

    def close(self):
        if self._h:
            lib().dvc_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
