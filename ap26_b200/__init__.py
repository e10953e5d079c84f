"""ap26_b200 -- B200-native AP26 per-K search (Python view of libap26.so).

The product is the C ABI in ``include/ap26.h`` (``libap26.so``) and the
``ap26`` command built from ``ap26_b200/csrc``.  This module binds that ABI
with ctypes for tests, benchmarks and Python callers.  There is no CPU
fallback: if ``libap26.so`` is missing the import fails, and every GPU entry
point reports AP26_E_NODEV / CUDA errors instead of computing on the host.

The reference interface it mirrors (ibethune/ap26):
  * ``Context.search_k(K, shift)``  <->  ``SearchAP26(K, SHIFT, ...)``
    (src/opencl/AP26.h:78) -- raw reports ``(k, K, first)``;
  * ``report(...)`` <-> ``ReportSolution`` (src/common/AP26.cpp:549-602);
  * ``hash_hex(...)`` <-> ``write_hash`` (AP26.cpp:295-357).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libap26.so")
CLI_PATH = os.path.join(HERE, "bin", "ap26")

OK = 0
E_ARG, E_CAPACITY, E_CUDA, E_DOMAIN, E_TIMEOUT, E_OVERFLOW, E_NOMEM, E_INVALID, E_NODEV = \
    -1, -2, -3, -4, -5, -6, -7, -8, -9

N53_PER_K = 137375320
N59_PER_K = 4808136200
MOD = 258559632607830
PRIM23 = 223092870
KMAX_SAFE = 400_000_000       # AP26_KMAX_SAFE
SHIFT_MAX = 16000             # AP26_SHIFT_MAX


class Opts(ctypes.Structure):
    _fields_ = [("dense_primes", ctypes.c_int32), ("warp_queue", ctypes.c_int32),
                ("block_threads", ctypes.c_int32), ("late_stage", ctypes.c_int32),
                ("chunk_tiles", ctypes.c_int32), ("use_graphs", ctypes.c_int32),
                ("profile", ctypes.c_int32), ("cand_ring_log2", ctypes.c_int32),
                ("mem_budget", ctypes.c_int64), ("wait_timeout_s", ctypes.c_double),
                ("tail_group", ctypes.c_int32), ("batch_wave", ctypes.c_int32)]


class AP(ctypes.Structure):
    _fields_ = [("k", ctypes.c_int32), ("K", ctypes.c_int32), ("first", ctypes.c_int64),
                ("n", ctypes.c_int64)]


class Stats(ctypes.Structure):
    _fields_ = [("candidates", ctypes.c_int64), ("late_items", ctypes.c_int64),
                ("prp_tests", ctypes.c_int64), ("aps", ctypes.c_int64),
                ("device_ms", ctypes.c_double), ("error_flags", ctypes.c_int32),
                ("launches", ctypes.c_int32), ("sieve_ms", ctypes.c_double),
                ("sieve_cells", ctypes.c_int64), ("sieve_launches", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("chain_walks", ctypes.c_int64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Item(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int64), ("kmin", ctypes.c_int32), ("kmax", ctypes.c_int32),
                ("shift", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class ItemResult(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int64), ("status", ctypes.c_int32), ("n_aps", ctypes.c_int32),
                ("first_ap", ctypes.c_int64), ("candidates", ctypes.c_int64),
                ("ks_searched", ctypes.c_int32), ("result_hash", ctypes.c_int32),
                ("latency_ms", ctypes.c_double)]


FINAL_MAX_SOL = 3


class Final(ctypes.Structure):
    """ap26_final: device-side ReportSolution of one raw report."""
    _fields_ = [("hash_add", ctypes.c_int64), ("status", ctypes.c_int32),
                ("n_sol", ctypes.c_int32), ("sol_len", ctypes.c_int32 * FINAL_MAX_SOL),
                ("reserved", ctypes.c_int32), ("sol_first", ctypes.c_int64 * FINAL_MAX_SOL)]

    def sols(self):
        return [(self.sol_len[i], self.sol_first[i]) for i in range(self.n_sol)]


class Sol(ctypes.Structure):
    _fields_ = [("len", ctypes.c_int32), ("K", ctypes.c_int32), ("first", ctypes.c_int64)]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python ap26_b200/build.py` "
                          "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    P, I, I64, V = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, None
    sig = {
        "ap26_version": (I, []),
        "ap26_strerror": (ctypes.c_char_p, [I]),
        "ap26_last_error": (ctypes.c_char_p, [P]),
        "ap26_create": (I, [I, P, P]),
        "ap26_destroy": (V, [P]),
        "ap26_get_opts": (I, [P, P]),
        "ap26_set_opts": (I, [P, P]),
        "ap26_list_variants": (I, [P, I]),
        "ap26_search_k": (I, [P, I, I, P, I, P, P]),
        "ap26_search_k_sol": (I, [P, I, I, I, P, P, I, P, P]),
        "ap26_search_k_sol_words": (I, [P, I, I, I, P, P, P, P, I, P, P]),
        "ap26_sprp_bases": (I, [P, P, P, I64, P, P]),
        "ap26_report_batch": (I, [P, P, I64, P, P, P]),
        "ap26_search_batch": (I, [P, P, I, P, I64, P, P, P]),
        "ap26_serve_submit": (I, [P, P]),
        "ap26_serve_submit_from": (I, [P, P, I, I, ctypes.c_int32]),
        "ap26_serve_step": (I, [P, P]),
        "ap26_serve_wait": (I, [P, ctypes.c_double]),
        "ap26_serve_poll": (I, [P, P, P, I64, P]),
        "ap26_serve_checkpoint": (I, [P, I64, P, P, P, P, P, P]),
        "ap26_serve_memory": (I, [P, P, P]),
        "ap26_sieve_range": (I, [P, I, I, I64, I64, P, I64, P, P]),
        "ap26_sieve_count": (I, [P, P, I, I, P, P]),
        "ap26_sprp_batch": (I, [P, P, I64, P, P]),
        "ap26_chain_batch": (I, [P, I, P, I64, P, P, P]),
        "ap26_autotune": (I, [P, I, I, P]),
        "ap26_probe_peaks": (I, [P, P, P]),
        "ap26_sieve_count_noalloc": (I, [I, P, I, I, P, P]),
        "ap26_will_search": (I, [I]),
        "ap26_report": (I, [P, I, I, I64, P, I, P]),
        "ap26_hash_hex": (I, [I, I, ctypes.c_int32, P]),
        "ap26_sort_aps": (I, [P, I, I]),
        "ap26_write_state": (I, [ctypes.c_char_p, I, I, I, I, I, ctypes.c_int32,
                                 ctypes.c_double, P]),
        "ap26_read_state": (I, [ctypes.c_char_p, I, I, I, P, P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()

# Every symbol include/ap26.h declares (checked by the CPU test suite).
EXPORTS = ("ap26_version", "ap26_strerror", "ap26_last_error", "ap26_create", "ap26_destroy",
           "ap26_get_opts", "ap26_set_opts", "ap26_list_variants", "ap26_search_k",
           "ap26_search_k_sol", "ap26_search_k_sol_words", "ap26_search_batch",
           "ap26_serve_submit", "ap26_serve_submit_from", "ap26_serve_step", "ap26_serve_wait",
           "ap26_serve_poll", "ap26_serve_checkpoint", "ap26_serve_memory",
           "ap26_sieve_range", "ap26_sieve_count",
           "ap26_sprp_batch", "ap26_sprp_bases", "ap26_report_batch", "ap26_chain_batch",
           "ap26_autotune", "ap26_probe_peaks",
           "ap26_sieve_count_noalloc",
           "ap26_will_search",
           "ap26_report", "ap26_hash_hex", "ap26_sort_aps", "ap26_write_state",
           "ap26_read_state")


class AP26Error(RuntimeError):
    def __init__(self, code, where="", detail=""):
        msg = f"{where}: {lib.ap26_strerror(code).decode()} ({code})"
        if detail:
            msg += f": {detail}"
        super().__init__(msg)
        self.code = code


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# ---- host services ------------------------------------------------------------
def will_search(K):
    return bool(lib.ap26_will_search(int(K)))


def hash_hex(kmin, kmax, result_hash):
    buf = ctypes.create_string_buffer(17)
    lib.ap26_hash_hex(int(kmin), int(kmax), int(result_hash), buf)
    return buf.value.decode()


class Reporter:
    """ReportSolution state: the running result hash and the SOL lines."""

    def __init__(self, result_hash=0):
        self.hash = ctypes.c_int32(result_hash)
        self.sol = []

    def report(self, k, K, first):
        buf = ctypes.create_string_buffer(1 << 14)
        used = ctypes.c_int(0)
        rc = lib.ap26_report(ctypes.byref(self.hash), int(k), int(K), int(first), buf,
                             len(buf), ctypes.byref(used))
        if rc != OK:
            raise AP26Error(rc, "ap26_report")
        if used.value:
            self.sol.extend(buf.value.decode().splitlines())

    def report_all(self, aps):
        for a in aps:
            self.report(a[0], a[1], a[2])

    def sol_file(self, kmin, kmax):
        """SOL-AP26.txt content the reference writes for [kmin, kmax]."""
        return "".join(l + "\n" for l in self.sol) + hash_hex(kmin, kmax, self.hash.value) + "\n"


def sort_aps(aps, shift):
    """aps: list of (k, K, first, n); returns them in the reference AVX2 order."""
    arr = (AP * len(aps))(*[AP(int(a[0]), int(a[1]), int(a[2]), int(a[3])) for a in aps])
    rc = lib.ap26_sort_aps(arr, len(aps), int(shift))
    if rc != OK:
        raise AP26Error(rc, "ap26_sort_aps")
    return [(a.k, a.K, a.first, a.n) for a in arr]


def list_variants():
    """Compiled sieve variants: [{dense_primes, warp_queue, block_threads, late_stage}]."""
    n = lib.ap26_list_variants(None, 0)
    arr = (Opts * n)()
    lib.ap26_list_variants(arr, n)
    return [{"dense_primes": o.dense_primes, "warp_queue": o.warp_queue,
             "block_threads": o.block_threads, "late_stage": o.late_stage,
             "tail_group": o.tail_group} for o in arr]


def _aps_to_list(arr, n):
    return [(arr[i].k, arr[i].K, arr[i].first, arr[i].n) for i in range(n)]


# ---- device context ---------------------------------------------------------------
class Context:
    """One CUDA device context of libap26 (ap26_create / ap26_destroy)."""

    def __init__(self, device=0, **opts):
        o = Opts(**opts)
        h = ctypes.c_void_p()
        rc = lib.ap26_create(int(device), ctypes.byref(o), ctypes.byref(h))
        if rc != OK:
            raise AP26Error(rc, "ap26_create")
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            lib.ap26_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, where):
        if rc != OK:
            raise AP26Error(rc, where, lib.ap26_last_error(self.h).decode())

    @property
    def opts(self):
        o = Opts()
        self._check(lib.ap26_get_opts(self.h, ctypes.byref(o)), "ap26_get_opts")
        return {f: getattr(o, f) for f, _ in o._fields_}

    def set_opts(self, **kw):
        cur = self.opts
        cur.update(kw)
        o = Opts(**cur)
        self._check(lib.ap26_set_opts(self.h, ctypes.byref(o)), "ap26_set_opts")
        return self.opts

    def search_k(self, K, shift=0, cap=1 << 16):
        """Raw reports [(k, K, first, n)] of one K, AVX2 order, and stats."""
        out = (AP * cap)()
        n = ctypes.c_int(0)
        st = Stats()
        self._check(lib.ap26_search_k(self.h, int(K), int(shift), out, cap, ctypes.byref(n),
                                      ctypes.byref(st)), "ap26_search_k")
        return _aps_to_list(out, n.value), st

    def search_k_sol(self, K, shift=0, result_hash=0, iter=0, cap=1 << 12):
        """SearchAP26 + ReportSolution of every result on the device, from
        shift word `iter` (the reference's ITER) on: (new result_hash, SOL
        lines [(len, K, first)] in SOL order, stats)."""
        out = (Sol * cap)()
        h = ctypes.c_int32(result_hash)
        n = ctypes.c_int(0)
        st = Stats()
        self._check(lib.ap26_search_k_sol(self.h, int(K), int(shift), int(iter), ctypes.byref(h),
                                          out, cap, ctypes.byref(n), ctypes.byref(st)),
                    "ap26_search_k_sol")
        return h.value, [(out[i].len, out[i].K, out[i].first) for i in range(n.value)], st

    def search_k_sol_words(self, K, shift=0, result_hash=0, iter=0, cap=1 << 12):
        """search_k_sol with per-word progress: (new result_hash, SOL lines,
        word of each SOL line, hash after each shift word (10), stats)."""
        out = (Sol * cap)()
        words = (ctypes.c_int32 * cap)()
        at = (ctypes.c_int32 * 10)()
        h = ctypes.c_int32(result_hash)
        n = ctypes.c_int(0)
        st = Stats()
        self._check(lib.ap26_search_k_sol_words(self.h, int(K), int(shift), int(iter),
                                                ctypes.byref(h), at, out, words, cap,
                                                ctypes.byref(n), ctypes.byref(st)),
                    "ap26_search_k_sol_words")
        return (h.value, [(out[i].len, out[i].K, out[i].first) for i in range(n.value)],
                list(words[:n.value]), list(at), st)

    def report_batch(self, aps, result_hash=None):
        """Device-side ReportSolution of raw reports [(k, K, first[, n])]:
        returns (rc, [Final], new result_hash or None).  rc is the first
        non-OK status (the per-report statuses are in the Finals)."""
        arr = (AP * max(1, len(aps)))(*[AP(int(a[0]), int(a[1]), int(a[2]),
                                           int(a[3]) if len(a) > 3 else 0) for a in aps])
        fin = (Final * max(1, len(aps)))()
        h = ctypes.c_int32(result_hash or 0)
        rc = lib.ap26_report_batch(self.h, arr, len(aps), fin,
                                   ctypes.byref(h) if result_hash is not None else None, None)
        if rc in (E_CUDA, E_NODEV):
            raise AP26Error(rc, "ap26_report_batch")
        return rc, list(fin[:len(aps)]), (h.value if result_hash is not None else None)

    def sprp_bases(self, N, a):
        N = np.ascontiguousarray(N, dtype=np.uint64)
        a = np.ascontiguousarray(a, dtype=np.uint32)
        v = np.zeros(len(N), np.uint8)
        st = Stats()
        self._check(lib.ap26_sprp_bases(self.h, _ptr(N), _ptr(a), len(N), _ptr(v),
                                        ctypes.byref(st)), "ap26_sprp_bases")
        return v, st

    def search_batch(self, items, ap_cap=1 << 20):
        """items: [(id, kmin, kmax, shift)] -> (per-item list of reports, results, stats)."""
        its = (Item * len(items))(*[Item(int(a), int(b), int(c), int(d), 0) for a, b, c, d in items])
        res = (ItemResult * len(items))()
        aps = (AP * ap_cap)()
        n = ctypes.c_int64(0)
        st = Stats()
        self._check(lib.ap26_search_batch(self.h, its, len(items), aps, ap_cap, ctypes.byref(n),
                                          res, ctypes.byref(st)), "ap26_search_batch")
        per = []
        for r in res:
            per.append([(aps[i].k, aps[i].K, aps[i].first, aps[i].n)
                        for i in range(r.first_ap, r.first_ap + r.n_aps)])
        return per, list(res), st

    def sieve_range(self, K, shift, q0, q1, cap=1 << 22):
        cand = np.zeros(cap, np.int64)
        n = ctypes.c_int64(0)
        st = Stats()
        self._check(lib.ap26_sieve_range(self.h, int(K), int(shift), int(q0), int(q1), _ptr(cand),
                                         cap, ctypes.byref(n), ctypes.byref(st)),
                    "ap26_sieve_range")
        return cand[:n.value].copy(), st

    def sieve_count(self, Ks, shift):
        ks = np.ascontiguousarray(Ks, dtype=np.int32)
        counts = np.zeros(len(ks), np.int64)
        st = Stats()
        self._check(lib.ap26_sieve_count(self.h, _ptr(ks), len(ks), int(shift), _ptr(counts),
                                         ctypes.byref(st)), "ap26_sieve_count")
        return counts, st

    def sprp_batch(self, N):
        N = np.ascontiguousarray(N, dtype=np.uint64)
        v = np.zeros(len(N), np.uint8)
        st = Stats()
        self._check(lib.ap26_sprp_batch(self.h, _ptr(N), len(N), _ptr(v), ctypes.byref(st)),
                    "ap26_sprp_batch")
        return v, st

    def chain_batch(self, K, n):
        n = np.ascontiguousarray(n, dtype=np.int64)
        k = np.zeros(len(n), np.int32)
        f = np.zeros(len(n), np.int64)
        st = Stats()
        self._check(lib.ap26_chain_batch(self.h, int(K), _ptr(n), len(n), _ptr(k), _ptr(f),
                                         ctypes.byref(st)), "ap26_chain_batch")
        return k, f, st

    def autotune(self, K, shift=0):
        o = Opts()
        self._check(lib.ap26_autotune(self.h, int(K), int(shift), ctypes.byref(o)),
                    "ap26_autotune")
        return {f: getattr(o, f) for f, _ in o._fields_}

    def probe_peaks(self):
        """(shared-memory GB/s, int32 multiply-add Tops/s) measured on this device."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(lib.ap26_probe_peaks(self.h, ctypes.byref(a), ctypes.byref(b)),
                    "ap26_probe_peaks")
        return a.value, b.value

    # serving
    def serve_submit(self, uid, kmin, kmax, shift):
        it = Item(int(uid), int(kmin), int(kmax), int(shift), 0)
        return lib.ap26_serve_submit(self.h, ctypes.byref(it))

    def serve_submit_from(self, uid, kmin, kmax, shift, K, ITER, result_hash):
        it = Item(int(uid), int(kmin), int(kmax), int(shift), 0)
        return lib.ap26_serve_submit_from(self.h, ctypes.byref(it), int(K), int(ITER),
                                          int(result_hash))

    def serve_step(self):
        active = ctypes.c_int(0)
        self._check(lib.ap26_serve_step(self.h, ctypes.byref(active)), "ap26_serve_step")
        return active.value

    def serve_wait(self, max_wait_s):
        """True once the oldest queued slice has finished (or none is queued)."""
        rc = lib.ap26_serve_wait(self.h, float(max_wait_s))
        if rc == E_TIMEOUT:
            return False
        self._check(rc, "ap26_serve_wait")
        return True

    def serve_checkpoint(self, uid):
        """(kmin, kmax, shift, K, ITER, result_hash) of a unit's device checkpoint."""
        v = [ctypes.c_int() for _ in range(5)]
        h = ctypes.c_int32()
        self._check(lib.ap26_serve_checkpoint(self.h, int(uid), *[ctypes.byref(x) for x in v],
                                              ctypes.byref(h)), "ap26_serve_checkpoint")
        return tuple(x.value for x in v) + (h.value,)

    def serve_memory(self):
        """(bytes held, budget) of the serving pool."""
        a, b = ctypes.c_int64(), ctypes.c_int64()
        self._check(lib.ap26_serve_memory(self.h, ctypes.byref(a), ctypes.byref(b)),
                    "ap26_serve_memory")
        return a.value, b.value

    def serve_poll(self, ap_cap=1 << 16):
        res = ItemResult()
        aps = (AP * ap_cap)()
        n = ctypes.c_int64(0)
        rc = lib.ap26_serve_poll(self.h, ctypes.byref(res), aps, ap_cap, ctypes.byref(n))
        if rc < 0:
            raise AP26Error(rc, "ap26_serve_poll")
        if rc == 0:
            return None
        return res, _aps_to_list(aps, n.value)
