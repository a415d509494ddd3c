"""Python host API of the B200 SPID-Join equi-join, over the C ABI of libspidjoin.so.

Mirrors the reference's host interface ``pidjoin::JoinInstance``
(include/join_internals.hpp:301-323 of yonsei-hpcp/spid-join): construct with the
rank layout, ``LoadColumn`` the "left" (R) and "right" (S) columns, then
``PrepareJoin`` / ``StartJoin`` / ``FinishJoin`` / ``RecordLogs``. Columns are
numpy ``uint32`` arrays of shape (n, 2) (the ``kv_pair_t`` layout: key, payload)
or device tensors given as ``(data_ptr, n)``. Errors raise ``SpjError`` instead
of exiting the process (the reference calls ``exit(-1)``).

The library has no CPU path: without a CUDA device every join call raises.
"""
import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libspidjoin.so")

SPJ_OK = 0
STATUS = {-1: "SPJ_E_ARG", -2: "SPJ_E_NOMEM", -3: "SPJ_E_CUDA", -4: "SPJ_E_STATE", -5: "SPJ_E_OVERFLOW",
          -6: "SPJ_E_TIMEOUT", -7: "SPJ_E_NODEVICE", -8: "SPJ_E_UNSUPPORTED"}
ALG = {"phj": 0, "nphj": 1, "smj": 2, "nl": 3}
SKEW_ADAPTIVE, SKEW_FIXED = 0, 1

# every symbol include/spidjoin.h declares
EXPORTS = (
    "spj_design_default", "spj_last_error", "spj_version", "spj_create", "spj_load_column", "spj_prepare",
    "spj_start", "spj_finish", "spj_record_logs", "spj_destroy", "spj_plan_create", "spj_plan_output_capacity",
    "spj_plan_execute", "spj_plan_stats", "spj_plan_destroy", "spj_partition_histogram", "spj_checksum_device",
    "spj_generate_host", "spj_generate_device", "spj_plan_kernel_times", "spj_join_noalloc",
    "spj_batch_create", "spj_batch_output_capacity", "spj_batch_bind", "spj_batch_execute", "spj_batch_stats",
    "spj_server_create", "spj_server_output_capacity", "spj_server_submit", "spj_server_wait", "spj_server_stats",
    "spj_server_reset_stats", "spj_server_destroy", "spj_server_hold", "spj_exchange_split",
    "spj_tuning_set", "spj_tuning_get", "spj_exchange_count", "spj_exchange_scatter", "spj_select",
    "spj_dist_unique_id", "spj_dist_create", "spj_dist_set_heavy", "spj_dist_join", "spj_dist_heavy_keys",
    "spj_dist_destroy", "spj_dist_abort", "spj_plan_describe",
)


class SpjError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class Predicate(ctypes.Structure):
    """spj_predicate_t: a selection on a tuple's key (field 1) or payload (field 2):
    op 0 ==, 1 <=, 2 >=, 3 <, 4 > lo; 5 lo <= value <= hi (src/dpu/include/select.h)."""
    _fields_ = [("field", ctypes.c_int), ("op", ctypes.c_int), ("lo", ctypes.c_uint32), ("hi", ctypes.c_uint32)]


PRED_FIELD = {"none": 0, "key": 1, "payload": 2}
PRED_OP = {"==": 0, "<=": 1, ">=": 2, "<": 3, ">": 4, "between": 5}


def predicate(field="key", op="==", lo=0, hi=0):
    """A Predicate from names: predicate("payload", "between", 10, 99)."""
    return Predicate(PRED_FIELD[field] if isinstance(field, str) else field,
                     PRED_OP[op] if isinstance(op, str) else op, lo, hi)


class Design(ctypes.Structure):
    """spj_design_t = join_design_t (include/idpHandler.hpp:131-145) + B200 tuning."""
    _fields_ = [("input_size", ctypes.c_int64), ("rank_num", ctypes.c_int), ("zipf_factor", ctypes.c_int),
                ("rs_ratio", ctypes.c_int), ("rank_set", ctypes.c_int), ("bank_set", ctypes.c_int),
                ("tpch_example", ctypes.c_int), ("join_alg", ctypes.c_int), ("radix_bits", ctypes.c_int),
                ("skew_mode", ctypes.c_int), ("unit_tuples", ctypes.c_int), ("heavy_sample", ctypes.c_int),
                ("table_slots", ctypes.c_int), ("select_r", Predicate), ("select_s", Predicate),
                ("reserved", ctypes.c_int * 4)]


class Result(ctypes.Structure):
    _fields_ = [("pairs", ctypes.c_void_p), ("n_pairs", ctypes.c_int64), ("num_rank", ctypes.c_int),
                ("rank_offsets", ctypes.POINTER(ctypes.c_int64))]


class Stats(ctypes.Structure):
    _fields_ = [("h2d_ms", ctypes.c_double), ("partition_ms", ctypes.c_double), ("join_ms", ctypes.c_double),
                ("finish_ms", ctypes.c_double), ("d2h_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
                ("n_pairs", ctypes.c_int64), ("units", ctypes.c_int64), ("heavy_keys", ctypes.c_int64),
                ("heavy_tuples", ctypes.c_int64), ("max_r_partition", ctypes.c_int64),
                ("max_s_partition", ctypes.c_int64), ("radix_bits", ctypes.c_int), ("table_slots", ctypes.c_int),
                ("join_alg", ctypes.c_int)]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class Tuning(ctypes.Structure):
    _fields_ = [("log2_r", ctypes.c_int), ("log2_ratio", ctypes.c_int), ("radix_bits_delta", ctypes.c_int),
                ("table_slots", ctypes.c_int), ("unit_tuples", ctypes.c_int), ("join_alg", ctypes.c_int),
                ("reserved", ctypes.c_int * 2)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("batches", ctypes.c_int64), ("max_inflight_batches", ctypes.c_int32), ("reserved0", ctypes.c_int32),
                ("mean_batch", ctypes.c_double), ("hbm_peak_bytes", ctypes.c_uint64),
                ("hbm_budget_bytes", ctypes.c_uint64), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double)]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_ if f[0] != "reserved0"}


class PlanShape(ctypes.Structure):
    _fields_ = [("join_alg", ctypes.c_int32), ("radix_bits", ctypes.c_int32), ("scatter_passes", ctypes.c_int32),
                ("table_slots", ctypes.c_int32), ("global_table_slots", ctypes.c_int64),
                ("heavy_sample", ctypes.c_int32), ("unit_tuples", ctypes.c_int32), ("out_chunk", ctypes.c_int32),
                ("chunk_tuples", ctypes.c_int32)]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class KernelTimes(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("hist_ms", "scan_ms", "scatter_ms", "units_ms", "join_ms", "fixup_ms", "total_ms")]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


_lib = None


def lib():
    """Loads libspidjoin.so (built by ``make -C spid-join_b200``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SpjError(-7, f"{LIB_PATH} is missing: build it with `make -C {HERE}`")
        L = ctypes.CDLL(LIB_PATH)
        vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
        L.spj_last_error.restype = ctypes.c_char_p
        L.spj_version.restype = ctypes.c_char_p
        L.spj_design_default.argtypes = [ctypes.POINTER(Design)]
        L.spj_design_default.restype = None
        L.spj_create.argtypes = [i32, i32, i32, ctypes.POINTER(vp)]
        L.spj_load_column.argtypes = [vp, vp, i64, i32]
        L.spj_prepare.argtypes = [vp, ctypes.POINTER(Design)]
        L.spj_start.argtypes = [vp, ctypes.POINTER(Design)]
        L.spj_finish.argtypes = [vp, ctypes.POINTER(Result)]
        L.spj_record_logs.argtypes = [vp, ctypes.POINTER(Stats), i32]
        L.spj_destroy.argtypes = [vp]
        L.spj_destroy.restype = None
        L.spj_plan_create.argtypes = [i64, i64, ctypes.POINTER(Design), ctypes.POINTER(vp)]
        L.spj_plan_describe.argtypes = [i64, i64, ctypes.POINTER(Design), i32, i32, i64, ctypes.POINTER(PlanShape)]
        L.spj_plan_output_capacity.argtypes = [vp]
        L.spj_plan_output_capacity.restype = i64
        L.spj_plan_execute.argtypes = [vp, vp, vp, vp, vp, vp]
        L.spj_plan_stats.argtypes = [vp, ctypes.POINTER(Stats)]
        L.spj_plan_kernel_times.argtypes = [vp, i32, ctypes.POINTER(KernelTimes)]
        L.spj_plan_destroy.argtypes = [vp]
        L.spj_plan_destroy.restype = None
        L.spj_partition_histogram.argtypes = [vp, i64, i32, vp, vp]
        L.spj_checksum_device.argtypes = [vp, vp, vp, vp]
        L.spj_generate_host.argtypes = [ctypes.c_uint64, i64, i64, ctypes.c_double, vp, vp,
                                        ctypes.POINTER(ctypes.c_uint64), i32]
        L.spj_generate_device.argtypes = [ctypes.c_uint64, i64, i64, ctypes.c_double, vp, vp, vp, vp]
        L.spj_join_noalloc.argtypes = [vp, i64, vp, i64, vp, i64, vp, vp]
        L.spj_select.argtypes = [vp, i64, ctypes.POINTER(Predicate), vp, vp, vp]
        L.spj_batch_create.argtypes = [i32, vp, vp, ctypes.POINTER(Design), ctypes.POINTER(vp)]
        L.spj_batch_output_capacity.argtypes = [vp, i32]
        L.spj_batch_output_capacity.restype = i64
        L.spj_batch_bind.argtypes = [vp, vp, vp, vp, vp]
        L.spj_batch_execute.argtypes = [vp, vp]
        L.spj_batch_stats.argtypes = [vp, i32, ctypes.POINTER(Stats)]
        L.spj_server_create.argtypes = [ctypes.POINTER(Design), ctypes.c_uint64, i32, i32, ctypes.POINTER(vp)]
        L.spj_server_output_capacity.argtypes = [vp, i64, i64]
        L.spj_server_output_capacity.restype = i64
        L.spj_server_submit.argtypes = [vp, vp, i64, vp, i64, vp, i64, vp, ctypes.POINTER(i64)]
        L.spj_server_wait.argtypes = [vp, i64, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
        L.spj_server_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
        L.spj_server_reset_stats.argtypes = [vp]
        L.spj_server_hold.argtypes = [vp, i32]
        L.spj_server_destroy.argtypes = [vp]
        L.spj_server_destroy.restype = None
        L.spj_exchange_split.argtypes = [vp, i64, i32, i32, vp, i32, i32, vp, vp, vp]
        L.spj_exchange_count.argtypes = [vp, i64, i32, i32, vp, i32, i32, vp, vp]
        L.spj_exchange_scatter.argtypes = [vp, i64, i32, i32, vp, i32, i32, vp, vp, vp, vp]
        L.spj_dist_unique_id.argtypes = [vp]
        L.spj_dist_create.argtypes = [vp, i32, i32, ctypes.POINTER(Design), ctypes.POINTER(vp)]
        L.spj_dist_set_heavy.argtypes = [vp, i32, ctypes.c_double, i32]
        L.spj_dist_join.argtypes = [vp, vp, i64, vp, i64, ctypes.POINTER(vp), ctypes.POINTER(i64), vp]
        L.spj_dist_heavy_keys.argtypes = [vp, vp, i32]
        L.spj_dist_abort.argtypes = [vp]
        L.spj_dist_destroy.argtypes = [vp]
        L.spj_dist_destroy.restype = None
        L.spj_tuning_set.argtypes = [ctypes.POINTER(Tuning), i32]
        L.spj_tuning_get.argtypes = [ctypes.POINTER(Tuning), i32]
        _lib = L
    return _lib


def check(rc):
    if rc != SPJ_OK:
        raise SpjError(rc, lib().spj_last_error().decode())
    return rc


def make_design(**kw):
    """A design with the reference's defaults; keyword overrides by field name
    (``join_alg`` may also be "phj", "smj", "nl", "nphj")."""
    d = Design()
    lib().spj_design_default(ctypes.byref(d))
    for k, v in kw.items():
        if k == "join_alg" and isinstance(v, str):
            v = ALG[v]
        if k not in {f[0] for f in Design._fields_}:
            raise KeyError(k)
        setattr(d, k, v if isinstance(v, Predicate) else int(v))
    return d


B200_SMS, B200_SMEM_PER_BLOCK = 148, 232448


def describe(n_r, n_s, design=None, num_sms=B200_SMS, max_smem_per_block=B200_SMEM_PER_BLOCK, batch_tuples=0):
    """The planner's choice for one join (spj_plan_describe): a dict with the
    local-join algorithm ("phj", "nphj", "smj", "nl"), fan-out, passes, table
    sizes, heavy-key sample, unit, output chunk and chunk size. Needs no GPU."""
    d = design if design is not None else make_design()
    sh = PlanShape()
    check(lib().spj_plan_describe(n_r, n_s, ctypes.byref(d), num_sms, max_smem_per_block, batch_tuples,
                                  ctypes.byref(sh)))
    out = sh.as_dict()
    out["join_alg"] = {v: k for k, v in ALG.items()}[out["join_alg"]]
    return out


def _host_tuples(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    if a.ndim != 2 or a.shape[1] != 2:
        raise ValueError("tuples must have shape (n, 2)")
    return a


def generate_host(n_r, n_s, zipf=0.0, seed=0x5EED5EED, nthreads=0):
    """The seeded benchmark relations and the checksum of their exact join."""
    R = np.zeros((n_r, 2), dtype=np.uint32)
    S = np.zeros((max(n_s, 0), 2), dtype=np.uint32)
    cs = ctypes.c_uint64()
    check(lib().spj_generate_host(seed, n_r, n_s, float(zipf), R.ctypes.data, S.ctypes.data if n_s else None,
                                  ctypes.byref(cs), nthreads))
    return R, S, int(cs.value)


@dataclass
class ResultBuffers:
    """ResultBuffers_t (include/type_defs.hpp:82): one buffer per rank + byte sizes."""
    buffers: list
    byte_sizes: list

    def pairs(self):
        return np.concatenate(self.buffers) if self.buffers else np.zeros((0, 2), np.uint32)


def _dpu_blocks(pairs, blocks=64):
    """One rank's pairs in the reference's transfer layout: `blocks` blocks of
    ceil(n / blocks) pairs, the pairs dealt evenly in order, (0, 0) padding."""
    n = pairs.shape[0]
    per = -(-n // blocks)
    out = np.zeros((blocks * per, 2), dtype=np.uint32)
    base, extra = divmod(n, blocks)
    lo = 0
    for b in range(blocks):
        cnt = base + (1 if b < extra else 0)
        out[b * per:b * per + cnt] = pairs[lo:lo + cnt]
        lo += cnt
    return out


class JoinInstance:
    """pidjoin::JoinInstance on one B200 (include/join_internals.hpp:301-323)."""

    def __init__(self, num_rank_allocated=1, num_rankgroup=1, num_rank_in_rankgroup=None):
        if num_rank_in_rankgroup is None:
            num_rank_in_rankgroup = num_rank_allocated // max(num_rankgroup, 1)
        self._h = ctypes.c_void_p()
        check(lib().spj_create(num_rank_allocated, num_rankgroup, num_rank_in_rankgroup, ctypes.byref(self._h)))
        self._keep = {}

    def LoadColumn(self, data, num_tuples=None, col_name="left"):
        side = {"left": 0, "right": 1}.get(col_name)
        if side is None:
            raise SpjError(-1, f"Column name error: {col_name} should be left or right")
        if isinstance(data, tuple):  # (device pointer, n)
            ptr, n = data
        else:
            arr = _host_tuples(data)
            self._keep[side] = arr
            ptr, n = arr.ctypes.data, arr.shape[0]
        if num_tuples is not None:
            n = int(num_tuples)
        check(lib().spj_load_column(self._h, ptr, n, side))

    def PrepareJoin(self, design=None):
        check(lib().spj_prepare(self._h, ctypes.byref(design) if design is not None else None))

    def StartJoin(self, design=None):
        check(lib().spj_start(self._h, ctypes.byref(design) if design is not None else None))

    def FinishJoin(self, copy=True, dpu_blocks=False):
        """Per-rank buffers. dpu_blocks: the reference's transfer layout, 64
        blocks of ceil(pairs / 64) per rank, the rank's pairs dealt evenly in
        order, each block padded with (0, 0) (as pidjoin.hpp's FinishJoin)."""
        res = Result()
        check(lib().spj_finish(self._h, ctypes.byref(res)))
        n = res.n_pairs
        if n:
            buf = (ctypes.c_uint32 * (2 * n)).from_address(res.pairs)
            flat = np.frombuffer(buf, dtype=np.uint32).reshape(n, 2)
        else:
            flat = np.zeros((0, 2), dtype=np.uint32)
        if copy:
            flat = flat.copy()
        offs = [res.rank_offsets[i] for i in range(res.num_rank + 1)]
        bufs = [flat[offs[i]:offs[i + 1]] for i in range(res.num_rank)]
        if dpu_blocks:
            bufs = [_dpu_blocks(b) for b in bufs]
            return ResultBuffers(bufs, [8 * b.shape[0] for b in bufs])
        return ResultBuffers(bufs, [8 * (offs[i + 1] - offs[i]) for i in range(res.num_rank)])

    def RecordLogs(self, print_=False):
        st = Stats()
        check(lib().spj_record_logs(self._h, ctypes.byref(st), int(print_)))
        return st.as_dict()

    def close(self):
        if self._h:
            lib().spj_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """Device-resident plan: allocation at creation; execute() allocates nothing."""

    def __init__(self, n_r, n_s, design=None):
        self._p = ctypes.c_void_p()
        design = design if design is not None else make_design()
        check(lib().spj_plan_create(n_r, n_s, ctypes.byref(design), ctypes.byref(self._p)))
        self.n_r, self.n_s = n_r, n_s

    @property
    def output_capacity(self):
        return lib().spj_plan_output_capacity(self._p)

    def execute(self, r_ptr, s_ptr, out_ptr, n_out_ptr, stream=0):
        check(lib().spj_plan_execute(self._p, r_ptr, s_ptr, out_ptr, n_out_ptr, stream))

    def stats(self):
        st = Stats()
        check(lib().spj_plan_stats(self._p, ctypes.byref(st)))
        return st.as_dict()

    def kernel_times(self, back=0):
        kt = KernelTimes()
        check(lib().spj_plan_kernel_times(self._p, back, ctypes.byref(kt)))
        return kt.as_dict()

    def close(self):
        if self._p:
            lib().spj_plan_destroy(self._p)
            self._p = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many joins in one launch sequence (spj_batch_*): create with the sizes,
    bind device pointers once, execute many times (graph-capturable)."""

    def __init__(self, n_r, n_s, design=None):
        self.J = len(n_r)
        design = design if design is not None else make_design()
        self._nr = (ctypes.c_int64 * self.J)(*[int(x) for x in n_r])
        self._ns = (ctypes.c_int64 * self.J)(*[int(x) for x in n_s])
        self._p = ctypes.c_void_p()
        check(lib().spj_batch_create(self.J, self._nr, self._ns, ctypes.byref(design), ctypes.byref(self._p)))

    def output_capacity(self, j):
        return lib().spj_batch_output_capacity(self._p, j)

    def bind(self, r_ptrs, s_ptrs, out_ptrs, n_out_ptr=None):
        arr = lambda xs: (ctypes.c_void_p * self.J)(*[int(x) for x in xs])
        self._bound = (arr(r_ptrs), arr(s_ptrs), arr(out_ptrs))
        check(lib().spj_batch_bind(self._p, self._bound[0], self._bound[1], self._bound[2], n_out_ptr))

    def execute(self, stream=0):
        check(lib().spj_batch_execute(self._p, stream))

    def stats(self, j):
        st = Stats()
        check(lib().spj_batch_stats(self._p, j, ctypes.byref(st)))
        return st.as_dict()

    def kernel_times(self, back=0):
        kt = KernelTimes()
        check(lib().spj_plan_kernel_times(self._p, back, ctypes.byref(kt)))
        return kt.as_dict()

    def close(self):
        if self._p:
            lib().spj_plan_destroy(self._p)
            self._p = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The served join stream (spj_server_*): submit joins over device columns,
    a worker thread in the library batches whatever has arrived and fits the
    HBM budget, and wait() returns once a join's output is in device memory."""

    def __init__(self, hbm_budget_bytes=120 << 30, max_batch=64, streams=4, design=None):
        design = design if design is not None else make_design()
        self._p = ctypes.c_void_p()
        check(lib().spj_server_create(ctypes.byref(design), int(hbm_budget_bytes), max_batch, streams,
                                      ctypes.byref(self._p)))

    def output_capacity(self, n_r, n_s):
        c = lib().spj_server_output_capacity(self._p, n_r, n_s)
        if c < 0:
            check(-1)
        return c

    def submit(self, r_ptr, n_r, s_ptr, n_s, out_ptr, out_capacity, n_out_ptr):
        i = ctypes.c_int64()
        check(lib().spj_server_submit(self._p, r_ptr, n_r, s_ptr, n_s, out_ptr, out_capacity, n_out_ptr,
                                      ctypes.byref(i)))
        return i.value

    def wait(self, req_id, timeout_ms=-1.0):
        """Returns the request's submit-to-completion latency in milliseconds."""
        lat = ctypes.c_double()
        check(lib().spj_server_wait(self._p, req_id, timeout_ms, ctypes.byref(lat)))
        return lat.value

    def stats(self):
        st = ServerStats()
        check(lib().spj_server_stats(self._p, ctypes.byref(st)))
        return st.as_dict()

    def reset_stats(self):
        check(lib().spj_server_reset_stats(self._p))

    def hold(self, on=True):
        """Pauses (or resumes) admission; joins submitted meanwhile queue up."""
        check(lib().spj_server_hold(self._p, 1 if on else 0))

    def close(self):
        if self._p:
            lib().spj_server_destroy(self._p)
            self._p = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def exchange_layout(C, me):
    """The receive layout of one exchange from the send-count matrix C
    (C[src][dst]: tuples rank src sends to rank dst): this rank's receive count,
    where its segment starts in every destination's buffer (the senders with a
    lower rank come first), and the largest receive count of any rank (the
    receive buffers' common size)."""
    world = len(C)
    recv = sum(int(C[s][me]) for s in range(world))
    off = [sum(int(C[s][d]) for s in range(me)) for d in range(world)]
    need = max(sum(int(C[s][d]) for s in range(world)) for d in range(world))
    return recv, off, need


class DistributedJoin:
    """A join of R and S sharded over the ranks of a torch.distributed process
    group, one GPU per rank: the multi-GPU form of the reference's rank-to-rank
    shuffle (src/queryHostFunc.cc:481-777). Every rank routes its shards by
    destination rank ((glb_partition_hash(key) * world) >> 32), exchanges them,
    and joins what it received with its own plan; the union over the ranks is
    the join of the union of the shards.

    Skew across ranks is handled as SPID-Join handles it across DPU rank sets:
    keys whose estimated share of the global S exceeds heavy_share / world (from
    an even sample of every rank's S, all-gathered) are heavy; their S tuples
    stay on the rank that holds them and their R tuples are replicated to every
    rank, so no rank receives a hot key's whole S.

    The exchange is either fused (`fused=True`: one kernel routes every tuple
    straight into its destination's receive buffer in symmetric memory, after an
    all-gather of the size matrix) or an NCCL all-to-all after a device split.
    `split(T, heavy, mode) -> (grouped, counts)` and `join(R, S) -> (pairs, n)`
    replace the device split and the local join; the CPU tests of the exchange
    protocol pass host versions of both and run gloo ranks."""

    MAX_HEAVY = 256

    def __init__(self, group=None, design=None, split=None, join=None, fused=False, heavy=True,
                 heavy_share=0.25, sample=1 << 16):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.design = design if design is not None else make_design()
        self._split = split if split is not None else self._device_split
        self._join = join if join is not None else self._device_join
        self.fused = fused
        self.heavy = heavy
        self.heavy_share = heavy_share
        self.sample = sample
        self.last_heavy = []
        self._plans = {}
        self._bufs = {}

    # ---- heavy keys
    def heavy_keys(self, S):
        """The sorted heavy keys (python ints), the same list on every rank."""
        import torch
        n = int(S.shape[0])
        k = min(n, self.sample)
        cand = torch.zeros((64, 2), dtype=torch.int64, device=S.device)
        if k > 0:
            idx = torch.linspace(0, n - 1, k, device=S.device).long()
            keys = S[idx, 0].long() & 0xFFFFFFFF
            keys = keys[keys != 0]
            if keys.numel():
                u, c = torch.unique(keys, return_counts=True)
                top = torch.topk(c, min(64, c.numel()))
                cand[:top.values.numel(), 0] = u[top.indices]
                cand[:top.values.numel(), 1] = (top.values.double() * (n / k)).long()
        allc = torch.empty((self.world * 64, 2), dtype=torch.int64, device=S.device)
        self.dist.all_gather_into_tensor(allc, cand, group=self.group)
        tot = torch.tensor([n], dtype=torch.int64, device=S.device)
        self.dist.all_reduce(tot, group=self.group)
        est = {}
        for key, cnt in allc.tolist():
            if key:
                est[key] = est.get(key, 0) + cnt
        bar = self.heavy_share * int(tot.item()) / self.world
        hot = sorted((k2 for k2, c in est.items() if c >= bar and c > 0), key=lambda k2: -est[k2])
        return sorted(hot[:self.MAX_HEAVY])

    def _replicated_rows(self, R, heavy):
        """Every rank's R tuples of the heavy keys, gathered on every rank."""
        import torch
        hk = torch.tensor([h - (1 << 32) if h >= (1 << 31) else h for h in heavy], dtype=torch.int32,
                          device=R.device)
        rows = R[torch.isin(R[:, 0], hk)] if R.shape[0] else R[:0]
        cnt = torch.tensor([rows.shape[0]], dtype=torch.int64, device=R.device)
        allcnt = torch.empty(self.world, dtype=torch.int64, device=R.device)
        self.dist.all_gather_into_tensor(allcnt, cnt, group=self.group)
        m = int(allcnt.max().item())
        if m == 0:
            return R[:0]
        pad = torch.zeros((m, 2), dtype=R.dtype, device=R.device)
        pad[:rows.shape[0]] = rows
        allrows = torch.empty((self.world * m, 2), dtype=R.dtype, device=R.device)
        self.dist.all_gather_into_tensor(allrows.view(-1), pad.view(-1), group=self.group)
        return allrows[allrows[:, 0] != 0]

    # ---- exchanges
    def _heavy_dev(self, heavy, device):
        """The heavy keys as the device array the exchange kernels binary-search:
        ascending unsigned order (the kernels require it), as int32 bit patterns."""
        import torch
        heavy = sorted(int(h) & 0xFFFFFFFF for h in heavy)
        return torch.tensor([h - (1 << 32) if h >= (1 << 31) else h for h in heavy] or [0], dtype=torch.int32,
                            device=device)

    def _device_split(self, T, heavy, mode):
        import torch
        hd = self._heavy_dev(heavy, T.device)
        out = torch.empty_like(T)
        cnt = torch.empty(2 * self.world, dtype=torch.int64, device=T.device)
        check(lib().spj_exchange_split(T.data_ptr(), T.shape[0], self.world, self.rank, hd.data_ptr(), len(heavy),
                                       mode, out.data_ptr(), cnt.data_ptr(), torch.cuda.current_stream().cuda_stream))
        return out, cnt[:self.world]

    def exchange(self, T, heavy=(), mode=0, extra=0):
        """All-to-all exchange of the (n, 2) int32 tuples T routed by destination
        rank; returns (buffer, received): the received tuples are buffer[:received],
        with `extra` spare rows after them."""
        import torch
        grouped, cnt = self._split(T, list(heavy), mode)
        recv_cnt = torch.empty_like(cnt)
        self.dist.all_to_all_single(recv_cnt, cnt, group=self.group)
        send, recv = [int(x) for x in cnt.tolist()], [int(x) for x in recv_cnt.tolist()]
        got = torch.empty((sum(recv) + extra, 2), dtype=T.dtype, device=T.device)
        src = grouped[:sum(send)].contiguous().view(torch.int64).view(-1)
        self.dist.all_to_all_single(got[:sum(recv)].view(torch.int64).view(-1), src, output_split_sizes=recv,
                                    input_split_sizes=send, group=self.group)
        return got, sum(recv)

    def _fused_exchange(self, T, slot, heavy=(), mode=0, extra=0):
        """The split fused into the send: each routed tuple is written straight
        into its destination rank's receive buffer (symmetric memory, peer stores
        over NVLink) by spj_exchange_scatter, after one all-gather of the size
        matrix; cross-GPU barriers before (receivers are done with the last
        exchange) and after (every sender is done)."""
        import torch
        import torch.distributed._symmetric_memory as symm
        stream = torch.cuda.current_stream().cuda_stream
        world = self.world
        hd = self._heavy_dev(list(heavy), T.device)
        cnt = torch.empty(world, dtype=torch.int64, device=T.device)
        check(lib().spj_exchange_count(T.data_ptr(), T.shape[0], world, self.rank, hd.data_ptr(), len(heavy), mode,
                                       cnt.data_ptr(), stream))
        allc = torch.empty(world * world, dtype=torch.int64, device=T.device)
        self.dist.all_gather_into_tensor(allc, cnt, group=self.group)
        recv, off, need = exchange_layout(allc.view(world, world).tolist(), self.rank)
        need += extra
        entry = self._bufs.get(slot)
        if entry is None or entry[0].shape[0] < need:  # the same decision on every rank: the matrix is global
            group = self.group if self.group is not None else self.dist.group.WORLD
            buf = symm.empty((int(need * 1.25) + 1024, 2), dtype=torch.int32, device=T.device)
            handle = symm.rendezvous(buf, group)
            ptrs = torch.tensor(list(handle.buffer_ptrs), dtype=torch.int64, device=T.device)
            entry = (buf, handle, ptrs)
            self._bufs[slot] = entry
        buf, handle, ptrs = entry
        offs = torch.tensor(off, dtype=torch.int64, device=T.device)
        cursor = torch.empty(world, dtype=torch.int64, device=T.device)
        handle.barrier(channel=0, timeout_ms=60000)
        check(lib().spj_exchange_scatter(T.data_ptr(), T.shape[0], world, self.rank, hd.data_ptr(), len(heavy), mode,
                                         ptrs.data_ptr(), offs.data_ptr(), cursor.data_ptr(), stream))
        handle.barrier(channel=0, timeout_ms=60000)
        return buf, recv

    def _device_join(self, R, S):
        import torch
        key = (R.shape[0], S.shape[0])
        if key not in self._plans:
            for p in self._plans.values():
                p.close()
            self._plans = {key: Plan(key[0], key[1], self.design)}
        plan = self._plans[key]
        out = torch.empty((plan.output_capacity, 2), dtype=torch.int32, device=R.device)
        n = torch.zeros(1, dtype=torch.int64, device=R.device)
        pad = torch.zeros((1, 2), dtype=torch.int32, device=R.device)
        r = R if R.shape[0] else pad
        s = S if S.shape[0] else pad
        plan.execute(r.data_ptr(), s.data_ptr(), out.data_ptr(), n.data_ptr(),
                     torch.cuda.current_stream().cuda_stream)
        return out, n

    def run(self, R, S):
        """R, S: this rank's shards, (n, 2) int32 tensors (key, payload) on this
        rank's device. Returns (pairs, n): this rank's part of the join."""
        # heavy keys matter only across ranks; heavy="always" also routes them on one rank
        heavy = self.heavy_keys(S) if self.heavy and (self.world > 1 or self.heavy == "always") else []
        self.last_heavy = heavy
        rows = self._replicated_rows(R, heavy) if heavy else R[:0]
        h = int(rows.shape[0])
        if self.fused:
            rb, nr = self._fused_exchange(R, "R", heavy, 2 if heavy else 0, extra=h)
            sb, ns = self._fused_exchange(S, "S", heavy, 1 if heavy else 0)
        else:
            rb, nr = self.exchange(R, heavy, 2 if heavy else 0, extra=h)
            sb, ns = self.exchange(S, heavy, 1 if heavy else 0)
        if h:
            rb[nr:nr + h] = rows
        return self._join(rb[:nr + h], sb[:ns])

    def close(self):
        for p in self._plans.values():
            p.close()
        self._plans = {}
        self._bufs = {}


class _DeviceView:
    """A (n, 2) int32 device array at a raw pointer, for torch.as_tensor."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n, 2), "typestr": "<i4", "data": (ptr, False), "version": 2,
                                         "strides": None}


class ShardedJoin:
    """The sharded join run by the library itself (spj_dist_*): the same
    protocol as DistributedJoin -- heavy keys from an all-gathered sample of
    every rank's S, their R tuples replicated, every other tuple routed to rank
    (glb_partition_hash(key) * world) >> 32 -- with NCCL driven from C, so a C or
    C++ caller needs no Python. `group`: a torch.distributed group whose ranks
    share the NCCL id (broadcast over it); or world/rank/unique_id given directly
    (world 1 needs neither). heavy: 0 off, 1 with more than one rank, 2 always."""

    def __init__(self, group=None, design=None, heavy=1, heavy_share=0.25, sample=1 << 16, world=None, rank=None,
                 unique_id=None):
        uid = ctypes.create_string_buffer(128)
        if world is None:
            import torch.distributed as dist
            world, rank = (dist.get_world_size(group), dist.get_rank(group)) if dist.is_initialized() else (1, 0)
        if unique_id is not None:
            uid.raw = bytes(unique_id)
        elif world == 1:
            check(lib().spj_dist_unique_id(uid))
        else:
            import torch.distributed as dist
            obj = [None]
            if rank == 0:
                check(lib().spj_dist_unique_id(uid))
                obj = [uid.raw]
            src = dist.get_global_rank(group, 0) if group is not None else 0
            dist.broadcast_object_list(obj, src=src, group=group)
            uid.raw = obj[0]
        self.world, self.rank = int(world), int(rank)
        self.design = design if design is not None else make_design()
        self.h = ctypes.c_void_p()
        check(lib().spj_dist_create(uid, self.world, self.rank, ctypes.byref(self.design), ctypes.byref(self.h)))
        check(lib().spj_dist_set_heavy(self.h, int(heavy), float(heavy_share), int(sample)))

    def run(self, R, S, stream=None):
        """R, S: this rank's shards, (n, 2) int32 CUDA tensors. Returns (pairs, n):
        this rank's part of the join, a (n, 2) int32 tensor that views the
        handle's output (valid until the next run or close)."""
        import torch
        st = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        pp, n = ctypes.c_void_p(), ctypes.c_int64()
        check(lib().spj_dist_join(self.h, R.data_ptr() if R.shape[0] else None, R.shape[0],
                                  S.data_ptr() if S.shape[0] else None, S.shape[0], ctypes.byref(pp),
                                  ctypes.byref(n), st))
        if n.value == 0:
            return torch.empty((0, 2), dtype=torch.int32, device=R.device), 0
        return torch.as_tensor(_DeviceView(pp.value, n.value), device=R.device), n.value

    def abort(self):
        """Aborts the communicator (callable from another thread): this rank's
        pending collectives end with an error; the handle can then only be closed."""
        check(lib().spj_dist_abort(self.h))

    @property
    def last_heavy(self):
        k = lib().spj_dist_heavy_keys(self.h, None, 0)
        buf = (ctypes.c_uint32 * max(k, 1))()
        lib().spj_dist_heavy_keys(self.h, buf, k)
        return [int(buf[i]) for i in range(k)]

    def close(self):
        if self.h:
            lib().spj_dist_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------- autotuning --
TUNING_KEYS = ("log2_r", "log2_ratio", "radix_bits_delta", "table_slots", "unit_tuples", "join_alg")


def set_tuning(entries):
    """Installs the process-wide per-size-class tuning table (list of dicts with
    TUNING_KEYS; [] clears it). Applies to joins planned in batches."""
    arr = (Tuning * max(1, len(entries)))()
    for i, e in enumerate(entries):
        for k in TUNING_KEYS:
            setattr(arr[i], k, int(e.get(k, 0)))
    check(lib().spj_tuning_set(arr, len(entries)))


def get_tuning():
    n = lib().spj_tuning_get(None, 0)
    arr = (Tuning * max(1, n))()
    lib().spj_tuning_get(arr, n)
    return [{k: getattr(arr[i], k) for k in TUNING_KEYS} for i in range(n)]


def load_tuning(path):
    import json
    with open(path) as f:
        t = json.load(f)
    set_tuning(t["entries"])
    return t


def autotune(classes, zipf=1.0, reps=3, batch_tuples=1 << 26, max_joins=256, candidates=None, log=None):
    """Autotuner of the batch planner: for every size class (log2|R|, log2(|S|/|R|))
    it builds a batch of joins of that class (about `batch_tuples` tuples, from the
    seeded device generator), times every candidate setting with CUDA events (a
    warm-up, then `reps` runs), checks every join's count and checksum, and keeps
    the fastest. A candidate is (fan-out offset, table slots, work-unit tuples,
    algorithm), the last as spj_tuning_t.join_alg (0 = the partitioned hash join;
    2 = the non-partitioned one, which skips the partitioning passes; 3-tuples
    mean 0); the fan-out offset also sets the pass count (one scatter pass up to
    2^8 partitions). Returns the table (the fields of spj_tuning_t plus the
    measured times); set_tuning() installs it. Needs a GPU."""
    import torch
    set_tuning([])  # measure against the planner's own choices
    if candidates is None:
        # tables no larger than the default: in a mixed batch the largest table sets
        # the shared memory (and so the CTAs per SM) of every join kernel
        candidates = ([(dl, 0, ut, a) for a in (0, 2) for dl in (0, -1, 1) for ut in (0, 131072)] +
                      [(0, 4096, 0, 0), (-1, 8192, 0, 0)])
    candidates = [tuple(c) + (0,) * (4 - len(c)) for c in candidates]
    table = []
    for lr, lt in classes:
        n_r = 1 << lr
        n_s = n_r << lt
        J = int(max(2, min(max_joins, batch_tuples // (n_r + n_s))))
        R, S, exp = [], [], []
        for j in range(J):
            dR = torch.empty((n_r, 2), dtype=torch.int32, device="cuda")
            dS = torch.empty((n_s, 2), dtype=torch.int32, device="cuda")
            e = torch.zeros(1, dtype=torch.int64, device="cuda")
            check(lib().spj_generate_device(0x7E57 + 7919 * j + 104729 * lr + 31 * lt, n_r, n_s, zipf,
                                            dR.data_ptr(), dS.data_ptr(), e.data_ptr(), None))
            R.append(dR)
            S.append(dS)
            exp.append(e)
        exp = torch.cat(exp)
        # planner's fan-out for this class (offset 0, automatic table and units)
        probe = Batch([n_r] * J, [n_s] * J, make_design(rank_num=1))
        outs = [torch.empty((probe.output_capacity(j), 2), dtype=torch.int32, device="cuda") for j in range(J)]
        n_out = torch.zeros(J, dtype=torch.int64, device="cuda")
        probe.bind([t.data_ptr() for t in R], [t.data_ptr() for t in S], [o.data_ptr() for o in outs],
                   n_out.data_ptr())
        probe.execute(0)
        torch.cuda.synchronize()
        base_bits = probe.stats(0)["radix_bits"]
        probe.close()
        del outs
        sums = torch.zeros(J, dtype=torch.int64, device="cuda")
        best, default_ms = None, None
        for dl, ts, ut, ta in candidates:
            bits = base_bits + dl
            if bits < 1 or bits > 15 or (ta == 2 and (dl or ts)):
                continue
            design = make_design(rank_num=1, radix_bits=bits if dl else 0, table_slots=ts, unit_tuples=ut,
                                 join_alg=ta - 1 if ta else 0)
            try:
                b = Batch([n_r] * J, [n_s] * J, design)
                outs = [torch.empty((b.output_capacity(j), 2), dtype=torch.int32, device="cuda") for j in range(J)]
                n_out.zero_()
                b.bind([t.data_ptr() for t in R], [t.data_ptr() for t in S], [o.data_ptr() for o in outs],
                       n_out.data_ptr())
                b.execute(0)
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ev0.record()
                for _ in range(reps):
                    b.execute(0)
                ev1.record()
                torch.cuda.synchronize()
                ms = ev0.elapsed_time(ev1) / reps
                for j in range(J):
                    check(lib().spj_checksum_device(outs[j].data_ptr(), n_out[j:j + 1].data_ptr(),
                                                    sums[j:j + 1].data_ptr(), None))
                ok = bool(((sums == exp) & (n_out == n_s)).all().item())
                for j in range(J):
                    b.stats(j)  # raises on a capacity error
                b.close()
                del outs
            except SpjError:
                continue
            if not ok:
                raise SpjError(-5, f"autotune candidate {(dl, ts, ut, ta)} gave a wrong result for class {(lr, lt)}")
            if (dl, ts, ut, ta) == (0, 0, 0, 0):
                default_ms = ms
            if best is None or ms < best[0]:
                best = (ms, dl, ts, ut, ta)
        entry = {"log2_r": lr, "log2_ratio": lt, "radix_bits_delta": best[1], "table_slots": best[2],
                 "unit_tuples": best[3], "join_alg": best[4], "joins": J, "ms": best[0], "planner_ms": default_ms}
        if log:
            log(entry)
        table.append(entry)
        del R, S
        torch.cuda.empty_cache()
    return table
