"""ctypes binding of libpt_b200.so (the C ABI declared in include/pt.h).

The library must have been built (``python -m libpt_b200.build``); loading
fails loudly otherwise -- there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libpt_b200.so")

PT_ARGS = ("d_ov", "f_ov", "t1", "t2", "i_oovo", "i_oovv", "i_ovvv")
FT_ARGS = ("d_ov", "f2_ov", "l1", "t2", "l2", "i_oovv", "i2_t2f2_oovo",
           "i3_ovvv", "i6_oovo", "i7_ovvv")
KINDS = ("rpt", "upt", "rft", "uft")
KIND_ID = {k: i for i, k in enumerate(KINDS)}

LIBPT_OK = 0
LIBPT_ERR_ARG = 1
LIBPT_ERR_NOMEM = 2
LIBPT_ERR_TIMEOUT = 4
LIBPT_ERR_CANCELLED = 6
ERRORS = {1: "LIBPT_ERR_ARG", 2: "LIBPT_ERR_NOMEM", 3: "LIBPT_ERR_CUDA",
          4: "LIBPT_ERR_TIMEOUT", 5: "LIBPT_ERR_UNSUPPORTED",
          6: "LIBPT_ERR_CANCELLED"}
PREC_FP64 = 0
PREC_TF32X3 = 1
PREC_EMU64 = 2          # | (slices << 8), slices 4..7; 0: chosen for 1 uEh
PREC_FP32 = 3           # FP32 tensor-core form (5 INT8 digit planes)

_lib = None


class LibptError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def args_of(kind):
    return PT_ARGS if kind[1:] == "pt" else FT_ARGS


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run "
                          "`python -m libpt_b200.build` (needs nvcc)")
    L = ctypes.CDLL(LIB_PATH)
    sz, dp, fp, vp = (ctypes.c_size_t, ctypes.POINTER(ctypes.c_double),
                      ctypes.POINTER(ctypes.c_float), ctypes.c_void_p)
    for kind in KINDS:
        nsz = 2 if kind[0] == "r" else 4
        npt = len(args_of(kind))
        for mp, ptr in ((False, dp), (True, fp)):
            name = "libpt_" + kind + ("_mp" if mp else "")
            f = getattr(L, name)
            f.restype = ctypes.c_double
            f.argtypes = [sz] * nsz + [ptr] * npt
            g = getattr(L, name + "_dev")
            g.restype = ctypes.c_int
            g.argtypes = [sz] * nsz + [vp] * npt + [vp, dp]
    L.libpt_print_banner.restype = None
    L.libpt_set_malloc.argtypes = [vp]
    L.libpt_set_free.argtypes = [vp]
    L.libpt_last_error.restype = ctypes.c_char_p
    L.libpt_plan_create.restype = ctypes.c_int
    L.libpt_plan_create.argtypes = [ctypes.c_int, sz, sz, sz, sz,
                                    ctypes.POINTER(vp), ctypes.c_int,
                                    ctypes.c_int, vp, ctypes.POINTER(vp)]
    L.libpt_plan_queue_length.restype = ctypes.c_int64
    L.libpt_plan_queue_length.argtypes = [vp]
    L.libpt_plan_slices.restype = ctypes.c_int
    L.libpt_plan_slices.argtypes = [vp]
    L.libpt_plan_flops.restype = ctypes.c_double
    L.libpt_plan_flops.argtypes = [vp, ctypes.c_int64, ctypes.c_int64]
    L.libpt_plan_run.restype = ctypes.c_int
    L.libpt_plan_run.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), sz]
    L.libpt_plan_run_all.restype = ctypes.c_int
    L.libpt_plan_run_all.argtypes = [vp]
    L.libpt_plan_energy.restype = ctypes.c_int
    L.libpt_plan_energy.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), sz,
                                    dp]
    L.libpt_plan_timing.restype = ctypes.c_int
    L.libpt_plan_timing.argtypes = [vp, ctypes.c_int]
    L.libpt_plan_kernel_stats.restype = ctypes.c_int
    L.libpt_plan_kernel_stats.argtypes = [
        vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64),
        ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
        ctypes.POINTER(ctypes.c_int64)]
    L.libpt_selftest.restype = ctypes.c_int
    L.libpt_selftest.argtypes = [ctypes.c_int] * 4 + [dp]
    L.libpt_selftest_variants.restype = ctypes.c_int
    L.libpt_selftest_variants.argtypes = [ctypes.c_int]
    L.libpt_kernel_bench.restype = ctypes.c_int
    L.libpt_kernel_bench.argtypes = [ctypes.c_int] * 5 + [dp, dp]
    L.libpt_selftest_wait.restype = ctypes.c_int
    L.libpt_selftest_wait.argtypes = [ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double,
                                      ctypes.POINTER(ctypes.c_int)]
    L.libpt_rpt_inputs_df.restype = ctypes.c_int
    L.libpt_rpt_inputs_df.argtypes = [sz, sz, sz] + [vp] * 8 + [vp]
    L.libpt_upt_inputs_df.restype = ctypes.c_int
    L.libpt_upt_inputs_df.argtypes = [sz] * 5 + [vp] * 9 + [vp]
    L.libpt_selftest_recip.restype = ctypes.c_int
    L.libpt_selftest_recip.argtypes = [ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, dp]
    # serving (pt_serve.h)
    L.libpt_footprint.restype = sz
    L.libpt_footprint.argtypes = [ctypes.c_int] + [sz] * 4 + [ctypes.c_int] * 3 + [sz]
    L.libpt_server_create.restype = ctypes.c_int
    L.libpt_server_create.argtypes = [sz, ctypes.c_int, ctypes.POINTER(vp)]
    L.libpt_server_submit.restype = ctypes.c_int
    L.libpt_server_submit.argtypes = ([vp, ctypes.c_int] + [sz] * 4 +
                                      [ctypes.POINTER(vp)] + [ctypes.c_int] * 3 +
                                      [ctypes.POINTER(ctypes.c_uint64)])
    L.libpt_server_wait.restype = ctypes.c_int
    L.libpt_server_wait.argtypes = [vp, ctypes.c_uint64, ctypes.c_double, dp, dp]
    L.libpt_server_cancel.restype = ctypes.c_int
    L.libpt_server_cancel.argtypes = [vp, ctypes.c_uint64]
    L.libpt_server_solve_times.restype = ctypes.c_int
    L.libpt_server_solve_times.argtypes = [vp, ctypes.c_uint64,
                                           ctypes.POINTER(ctypes.c_double)]
    L.libpt_server_inputs_released.restype = ctypes.c_int
    L.libpt_server_inputs_released.argtypes = [vp, ctypes.c_uint64,
                                               ctypes.POINTER(ctypes.c_int)]
    L.libpt_server_stats_get.restype = ctypes.c_int
    L.libpt_server_stats_get.argtypes = [vp, ctypes.POINTER(ServerStats)]
    L.libpt_server_destroy.restype = ctypes.c_int
    L.libpt_server_destroy.argtypes = [vp]
    L.libpt_plan_destroy.restype = ctypes.c_int
    L.libpt_plan_destroy.argtypes = [vp]
    L.libpt_shard_entries.restype = ctypes.c_int64
    L.libpt_shard_entries.argtypes = [ctypes.c_int64, ctypes.c_int,
                                      ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int64)]
    L.libpt_plan_run_shard.restype = ctypes.c_int
    L.libpt_plan_run_shard.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.libpt_plan_energy_slots.restype = ctypes.c_int
    L.libpt_plan_energy_slots.argtypes = [vp, ctypes.POINTER(vp)]
    L.libpt_energy_sum.restype = ctypes.c_int
    L.libpt_energy_sum.argtypes = [dp, sz, dp]
    _lib = L
    return L


def check(code):
    if code != LIBPT_OK:
        raise LibptError(code, lib().libpt_last_error().decode())


def _sizes(case):
    s = [int(case["oa"]), int(case["va"])]
    if case["kind"][0] == "u":
        s += [int(case["ob"]), int(case["vb"])]
    return s


def solve_host(case, mp=False):
    """Energy through the reference-compatible host-pointer entry point
    (libpt_rpt / _upt / _rft / _uft and their _mp forms)."""
    kind = case["kind"]
    dt = np.float32 if mp else np.float64
    ct = ctypes.c_float if mp else ctypes.c_double
    arrs = [np.ascontiguousarray(case[n], dtype=dt) for n in args_of(kind)]
    f = getattr(lib(), "libpt_" + kind + ("_mp" if mp else ""))
    return f(*_sizes(case), *[a.ctypes.data_as(ctypes.POINTER(ct))
                              for a in arrs])


def solve_device(case, tensors, mp=False, stream=None):
    """Energy through the device-pointer twin; `tensors` maps argument names
    to CUDA torch tensors (contiguous, float64 or float32 for mp)."""
    kind = case["kind"]
    f = getattr(lib(), "libpt_" + kind + ("_mp" if mp else "") + "_dev")
    e = ctypes.c_double(0.0)
    ptrs = [ctypes.c_void_p(tensors[n].data_ptr()) for n in args_of(kind)]
    check(f(*_sizes(case), *ptrs, ctypes.c_void_p(stream or 0),
            ctypes.byref(e)))
    return e.value


def selftest(precision, m, n, k, variant=0, device_maps=False, dbits=7):
    """Error of one contraction kernel (tile variant `variant`; tensor maps
    from device memory when device_maps; emulated FP64 digit width dbits)
    against an FP64 product, over the dot products' magnitude scale
    (libpt_selftest)."""
    e = ctypes.c_double(-1.0)
    word = precision | (variant << 16) | ((1 << 24) if device_maps else 0)
    if dbits == 8:
        word |= 1 << 15
    check(lib().libpt_selftest(word, m, n, k, ctypes.byref(e)))
    return e.value


def kernel_bench(precision, m, n, k, reps=10, variant=0, device_maps=False):
    """(mean ms per launch, check error) of one resident contraction job of
    4 m n k flops (libpt_kernel_bench)."""
    ms, e = ctypes.c_double(0.0), ctypes.c_double(-1.0)
    word = precision | (variant << 16) | ((1 << 24) if device_maps else 0)
    check(lib().libpt_kernel_bench(word, m, n, k, reps, ctypes.byref(ms),
                                   ctypes.byref(e)))
    return ms.value, e.value


def selftest_variants(precision):
    """Number of tile variants of a precision mode (libpt_selftest_variants)."""
    return lib().libpt_selftest_variants(precision)


def selftest_wait(stages, arrive, limit_ms):
    """(status code, hand-offs seen) of the bounded-wait probe
    (libpt_selftest_wait): the producer stops after `arrive` of `stages`
    hand-offs; a missing one makes the wait run out (LIBPT_ERR_TIMEOUT)."""
    seen = ctypes.c_int(-1)
    code = lib().libpt_selftest_wait(stages, arrive, limit_ms,
                                     ctypes.byref(seen))
    return code, seen.value


def rpt_inputs_df(b_oo, b_ov, b_vv, t2_abab=None, stream=None):
    """Restricted (T) integral arrays (and t2, when t2_abab is given) in the
    pt.h layout, built on the device from density-fitted factors
    (libpt_rpt_inputs_df).  b_oo, b_ov, b_vv: CUDA float64 tensors of shapes
    (naux, o, o), (naux, o, v), (naux, v, v); t2_abab: (o, o, v, v).  Returns
    a dict of the produced CUDA tensors by pt.h argument name."""
    import torch
    naux, o, v = b_ov.shape
    f64 = dict(dtype=torch.float64, device=b_ov.device)
    out = dict(i_oovo=torch.empty(2 * o * o * v * o, **f64),
               i_oovv=torch.empty(2 * o * o * v * v, **f64),
               i_ovvv=torch.empty(o * v * (v * (v - 1) // 2) + o * v * v * v,
                                  **f64))
    if t2_abab is not None:
        out["t2"] = torch.empty(2 * o * o * v * v, **f64)
    ins = [b_oo.contiguous(), b_ov.contiguous(), b_vv.contiguous(),
           None if t2_abab is None else t2_abab.contiguous()]
    ptr = lambda t: None if t is None else t.data_ptr()   # noqa: E731
    check(lib().libpt_rpt_inputs_df(
        o, v, naux, *[ptr(t) for t in ins], ptr(out.get("t2")),
        ptr(out["i_oovo"]), ptr(out["i_oovv"]), ptr(out["i_ovvv"]),
        stream or 0))
    torch.cuda.synchronize()   # the inputs (and any copies above) stay alive
    return out


def upt_inputs_df(fa, fb, stream=None):
    """Unrestricted (T) integral arrays in the pt.h layout built on the
    device (libpt_upt_inputs_df) from each spin's factors fa, fb = (b_oo,
    b_ov, b_vv) CUDA float64 tensors of shapes (naux, o, o), (naux, o, v),
    (naux, v, v).  Returns a dict of the produced CUDA tensors."""
    import torch
    naux, oa, va = fa[1].shape
    ob, vb = fb[1].shape[1:]
    npa, npb = va * (va - 1) // 2, vb * (vb - 1) // 2
    f64 = dict(dtype=torch.float64, device=fa[1].device)
    out = dict(
        i_oovo=torch.empty(oa * oa * va * oa + oa * ob * va * ob +
                           ob * ob * vb * ob + ob * oa * vb * oa, **f64),
        i_oovv=torch.empty(oa * oa * va * va + 2 * oa * ob * va * vb +
                           ob * ob * vb * vb, **f64),
        i_ovvv=torch.empty(oa * va * npa + oa * vb * va * vb + ob * vb * npb +
                           ob * va * vb * va, **f64))
    ins = [t.contiguous() for t in (*fa, *fb)]
    check(lib().libpt_upt_inputs_df(
        oa, va, ob, vb, naux, *[t.data_ptr() for t in ins],
        out["i_oovo"].data_ptr(), out["i_oovv"].data_ptr(),
        out["i_ovvv"].data_ptr(), stream or 0))
    torch.cuda.synchronize()   # the inputs (and any copies above) stay alive
    return out


def selftest_recip(lo_exp, hi_exp, n):
    """Largest distance in ulps between the energy epilogues' reciprocal and
    the IEEE division 1.0 / d over n values d = +-m 2^x, x in [lo_exp,
    hi_exp] (libpt_selftest_recip)."""
    worst = ctypes.c_double(-1.0)
    check(lib().libpt_selftest_recip(lo_exp, hi_exp, n, ctypes.byref(worst)))
    return worst.value


HOST_MALLOC = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_size_t)
HOST_FREE = ctypes.CFUNCTYPE(None, ctypes.c_void_p)


def set_host_allocator(malloc_fn=None, free_fn=None):
    """Installs host allocation hooks (libpt_set_malloc / libpt_set_free,
    src/misc.c:33-47): Python callables, wrapped as C function pointers and
    kept alive here; None restores malloc / free."""
    global _hooks
    m = HOST_MALLOC(malloc_fn) if malloc_fn else None
    f = HOST_FREE(free_fn) if free_fn else None
    _hooks = (m, f)
    lib().libpt_set_malloc(ctypes.cast(m, ctypes.c_void_p) if m else None)
    lib().libpt_set_free(ctypes.cast(f, ctypes.c_void_p) if f else None)


_hooks = (None, None)


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("rounds", ctypes.c_uint64),
                ("graph_rounds", ctypes.c_uint64), ("triples", ctypes.c_uint64),
                ("launches", ctypes.c_uint64), ("flops", ctypes.c_double),
                ("pool_bytes", ctypes.c_size_t),
                ("bytes_in_use", ctypes.c_size_t),
                ("peak_bytes_in_use", ctypes.c_size_t),
                ("max_resident", ctypes.c_uint64)]


def footprint(kind, sizes, mp=False, precision=PREC_FP64, host=True,
              round_triples=0):
    """Device bytes the server takes for a solve (libpt_footprint)."""
    s = list(sizes)
    if len(s) == 2:
        s += s
    return lib().libpt_footprint(KIND_ID[kind], *s, 1 if mp else 0, precision,
                                 1 if host else 0, round_triples)


class Server:
    """Continuous-batching request loop (libpt_server_*, pt_serve.h)."""

    def __init__(self, mem_budget=0, max_active=0):
        h = ctypes.c_void_p()
        check(lib().libpt_server_create(mem_budget, max_active,
                                        ctypes.byref(h)))
        self.h = h
        self._keep = {}

    def submit(self, case, tensors=None, mp=False, precision=PREC_FP64):
        """Queues a solve; tensors: device tensors by name, else the case's
        host arrays.  Returns its ticket."""
        kind = case["kind"]
        s = _sizes(case)
        if len(s) == 2:
            s += s
        names = args_of(kind)
        if tensors is None:
            dt = np.float32 if mp else np.float64
            arrs = [np.ascontiguousarray(case[n], dtype=dt) for n in names]
            ptrs = (ctypes.c_void_p * len(names))(
                *[a.ctypes.data for a in arrs])
            keep, host = arrs, 1
        else:
            keep = [tensors[n] for n in names]
            ptrs = (ctypes.c_void_p * len(names))(*[t.data_ptr() for t in keep])
            host = 0
        t = ctypes.c_uint64()
        check(lib().libpt_server_submit(self.h, KIND_ID[kind], *s, ptrs,
                                        1 if mp else 0, precision, host,
                                        ctypes.byref(t)))
        self._keep[t.value] = keep     # inputs live until the solve is done
        return t.value

    def wait(self, ticket, timeout=-1.0):
        """(energy, latency seconds) of a solve."""
        e, lat = ctypes.c_double(), ctypes.c_double()
        code = lib().libpt_server_wait(self.h, ticket, timeout,
                                       ctypes.byref(e), ctypes.byref(lat))
        if code != LIBPT_ERR_TIMEOUT:   # done: its inputs may go
            self._keep.pop(ticket, None)
        check(code)
        return e.value, lat.value

    def cancel(self, ticket):
        """Cancels a solve (libpt_server_cancel); its wait then raises
        LIBPT_ERR_CANCELLED unless it had already ended."""
        check(lib().libpt_server_cancel(self.h, ticket))

    def times(self, ticket):
        """(admission wait, preparation, wait for the first round, running)
        seconds of an ended solve (libpt_server_solve_times)."""
        t = (ctypes.c_double * 4)()
        check(lib().libpt_server_solve_times(self.h, ticket, t))
        return tuple(t)

    def release_inputs(self):
        """Drops the references to inputs the server no longer reads;
        returns how many solves still hold theirs."""
        for t in list(self._keep):
            r = ctypes.c_int(0)
            check(lib().libpt_server_inputs_released(self.h, t,
                                                     ctypes.byref(r)))
            if r.value:
                del self._keep[t]
        return len(self._keep)

    def stats(self):
        st = ServerStats()
        check(lib().libpt_server_stats_get(self.h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def close(self):
        if self.h:
            lib().libpt_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def shard_entries(queue_length, rank, size):
    """Queue entries rank `rank` of `size` owns (q % size == rank)."""
    n = lib().libpt_shard_entries(queue_length, rank, size, None)
    if n < 0:
        raise LibptError(1, lib().libpt_last_error().decode())
    a = np.empty(n, dtype=np.int64)
    lib().libpt_shard_entries(queue_length, rank, size,
                              a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    return a


def energy_sum(energies):
    """The library's queue-order compensated sum of per-triple energies."""
    a = np.ascontiguousarray(energies, dtype=np.float64)
    e = ctypes.c_double()
    check(lib().libpt_energy_sum(
        a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size,
        ctypes.byref(e)))
    return e.value


class _DeviceArray:
    """float64 device memory owned by the library, exposed to torch."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {
            "shape": (n,), "typestr": "<f8", "data": (ptr, False),
            "version": 3, "strides": None}


class Plan:
    """Resident operands of one solve and its triples queue (libpt_plan_*)."""

    def __init__(self, case, tensors, mp=False, precision=PREC_FP64,
                 stream=None):
        kind = case["kind"]
        s = _sizes(case)
        if len(s) == 2:
            s += s
        ptrs = (ctypes.c_void_p * len(args_of(kind)))(
            *[tensors[n].data_ptr() for n in args_of(kind)])
        h = ctypes.c_void_p()
        check(lib().libpt_plan_create(KIND_ID[kind], *s, ptrs, 1 if mp else 0,
                                      precision, ctypes.c_void_p(stream or 0),
                                      ctypes.byref(h)))
        self.h = h
        self.n = lib().libpt_plan_queue_length(h)
        self.slices = lib().libpt_plan_slices(h)

    def flops(self, first=0, n=None):
        return lib().libpt_plan_flops(self.h, first,
                                      self.n - first if n is None else n)

    def run(self, idx=None):
        if idx is None:
            check(lib().libpt_plan_run_all(self.h))
            return
        a = np.ascontiguousarray(idx, dtype=np.int64)
        check(lib().libpt_plan_run(
            self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), a.size))

    def energy(self, idx=None):
        e = ctypes.c_double(0.0)
        if idx is None:
            check(lib().libpt_plan_energy(self.h, None, 0, ctypes.byref(e)))
        else:
            a = np.ascontiguousarray(idx, dtype=np.int64)
            check(lib().libpt_plan_energy(
                self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                a.size, ctypes.byref(e)))
        return e.value

    def run_shard(self, rank, size):
        """Zero the energy slots, run the entries rank `rank` of `size` owns."""
        check(lib().libpt_plan_run_shard(self.h, rank, size))

    def energy_slots(self):
        """The plan's per-triple energies as a CUDA float64 tensor (a view of
        the plan's own device memory, valid while the plan lives)."""
        import torch
        ptr = ctypes.c_void_p()
        check(lib().libpt_plan_energy_slots(self.h, ctypes.byref(ptr)))
        return torch.as_tensor(_DeviceArray(ptr.value, self.n), device="cuda")

    def timing(self, enable=True):
        check(lib().libpt_plan_timing(self.h, 1 if enable else 0))

    def kernel_stats(self):
        """dict(gemm_ms, gemm_launches, gemm_flops, epi_ms, launches) since
        the last call (kernel-level CUDA-event timings)."""
        gm, gf, em = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        gl, la = ctypes.c_int64(), ctypes.c_int64()
        check(lib().libpt_plan_kernel_stats(self.h, ctypes.byref(gm),
                                            ctypes.byref(gl), ctypes.byref(gf),
                                            ctypes.byref(em), ctypes.byref(la)))
        return dict(gemm_ms=gm.value, gemm_launches=gl.value,
                    gemm_flops=gf.value, epi_ms=em.value, launches=la.value)

    def close(self):
        if self.h:
            lib().libpt_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
