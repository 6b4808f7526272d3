"""ctypes binding of libnrgb.so (include/nrgb.h).

The library is the product: there is no Python or CPU fallback.  Loading
fails loudly when the shared object is missing or no CUDA device is present.
"""
from __future__ import annotations

import ctypes as C
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# NRGB_LIB overrides the library's path (for example to compare two builds)
LIBPATH = os.environ.get("NRGB_LIB") or os.path.join(HERE, "libnrgb.so")

EXPORTS = ["nrgb_create", "nrgb_destroy", "nrgb_last_error", "nrgb_version",
           "nrgb_syev_batched", "nrgb_syev_batched_dev", "nrgb_gemm_grouped_dev", "nrgb_gemm_grouped_split_dev",
           "nrgb_eig_recalc_step", "nrgb_eig_recalc_step_dev", "nrgb_profile", "nrgb_profile_only", "nrgb_kernel_stats",
           "nrgb_kernel_work",
           "nrgb_basis_change_noalloc", "nrgb_run", "nrgb_set_eig_mode",
           "nrgb_set_wait_limit", "nrgb_inject_barrier_shortfall",
           "nrgb_autotune", "nrgb_set_schedule", "nrgb_get_schedule",
           "nrgb_mat_upload", "nrgb_mat_download", "nrgb_mat_shape", "nrgb_mat_free", "nrgb_run_begin",
           "nrgb_step", "nrgb_recalc", "nrgb_dm_backward", "nrgb_spectrum_fdm", "nrgb_spectrum_dmnrg",
           "nrgb_server_create", "nrgb_server_submit", "nrgb_server_wait", "nrgb_server_error",
           "nrgb_server_counters", "nrgb_server_destroy", "nrgb_project_bytes"]


class GemmTerm(C.Structure):
    _fields_ = [("a", C.c_void_p), ("b", C.c_void_p), ("lda", C.c_int), ("ldb", C.c_int),
                ("k", C.c_int), ("trans_a", C.c_int), ("trans_b", C.c_int), ("alpha", C.c_double)]


class DiagTerm(C.Structure):
    _fields_ = [("blk", C.c_int), ("off", C.c_int), ("len", C.c_int), ("src", C.c_int),
                ("scale", C.c_double), ("shift", C.c_double)]


class OffdiagTerm(C.Structure):
    _fields_ = [("blk", C.c_int), ("offi", C.c_int), ("offj", C.c_int), ("rows", C.c_int), ("cols", C.c_int),
                ("src", C.c_int), ("factor", C.c_double)]


class StepPlan(C.Structure):
    _fields_ = [("nblocks", C.c_int), ("dim", C.POINTER(C.c_int)), ("ndiag", C.c_int),
                ("diag", C.POINTER(DiagTerm)), ("noff", C.c_int), ("off", C.POINTER(OffdiagTerm)),
                ("fixeps", C.c_double), ("keepenergy", C.c_double), ("keep", C.c_int), ("keepmin", C.c_int),
                ("safeguard", C.c_double), ("safeguardmax", C.c_int), ("keep_all", C.c_int),
                ("betabar", C.c_double)]


class RecalcTerm(C.Structure):
    _fields_ = [("z1", C.c_int), ("off1", C.c_int), ("r1", C.c_int), ("zp", C.c_int), ("offp", C.c_int),
                ("rp", C.c_int), ("op", C.c_int), ("factor", C.c_double)]


class RecalcOut(C.Structure):
    _fields_ = [("k1", C.c_int), ("kp", C.c_int), ("term0", C.c_int), ("nterms", C.c_int)]


class DmTerm(C.Structure):
    _fields_ = [("z1", C.c_int), ("off1", C.c_int), ("k1", C.c_int), ("zp", C.c_int), ("offp", C.c_int),
                ("kp", C.c_int), ("rho", C.c_int), ("factor", C.c_double)]


class DmOut(C.Structure):
    _fields_ = [("r1", C.c_int), ("rp", C.c_int), ("term0", C.c_int), ("nterms", C.c_int)]


class FdmPair(C.Structure):
    _fields_ = [("op1", C.c_int), ("op2", C.c_int), ("rho_i", C.c_int), ("rho_j", C.c_int), ("e_i", C.c_int),
                ("e_j", C.c_int), ("reti", C.c_int), ("retj", C.c_int), ("factor", C.c_double)]


class DmnrgPair(C.Structure):
    _fields_ = [("op1", C.c_int), ("op2", C.c_int), ("rho_1", C.c_int), ("rho_p", C.c_int), ("e_1", C.c_int),
                ("e_p", C.c_int), ("factor", C.c_double)]


class GemmOut(C.Structure):
    _fields_ = [("c", C.c_void_p), ("ldc", C.c_int), ("m", C.c_int), ("n", C.c_int),
                ("beta", C.c_double), ("term0", C.c_int), ("nterms", C.c_int)]


_lib = None


def load(path: str = LIBPATH):
    """Load libnrgb.so and declare its signatures (no device needed)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("libnrgb.so not built: run nrgljubljana-old_b200/build.py")
    lib = C.CDLL(path)
    vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
    lib.nrgb_create.argtypes = [C.c_int, C.POINTER(vp)]
    lib.nrgb_destroy.argtypes = [vp]
    lib.nrgb_last_error.argtypes = [vp]
    lib.nrgb_last_error.restype = C.c_char_p
    lib.nrgb_version.restype = C.c_char_p
    lib.nrgb_syev_batched.argtypes = [vp, C.c_int, ip, C.POINTER(vp), C.POINTER(vp)]
    lib.nrgb_syev_batched_dev.argtypes = [vp, C.c_int, ip, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), vp]
    lib.nrgb_gemm_grouped_dev.argtypes = [vp, C.c_int, C.POINTER(GemmOut), C.c_int, C.POINTER(GemmTerm), vp]
    lib.nrgb_gemm_grouped_split_dev.argtypes = [vp, C.c_int, C.c_int, C.POINTER(GemmOut), C.c_int,
                                                C.POINTER(GemmTerm), vp]
    lib.nrgb_run.argtypes = [vp, C.c_char_p, C.c_char_p, dp]
    lib.nrgb_set_eig_mode.argtypes = [vp, C.c_int]
    lib.nrgb_set_wait_limit.argtypes = [vp, C.c_int]
    lib.nrgb_autotune.argtypes = [vp, C.c_char_p, C.c_int]
    lib.nrgb_mat_upload.argtypes = [vp, C.c_int, C.c_int, vp, ip]
    lib.nrgb_mat_download.argtypes = [vp, C.c_int, vp]
    lib.nrgb_mat_shape.argtypes = [vp, C.c_int, ip, ip]
    lib.nrgb_mat_free.argtypes = [vp, C.c_int]
    lib.nrgb_run_begin.argtypes = [vp]
    lib.nrgb_step.argtypes = [vp, C.POINTER(StepPlan), ip, ip, ip, dp, dp]
    lib.nrgb_recalc.argtypes = [vp, C.c_int, C.POINTER(RecalcOut), C.c_int, C.POINTER(RecalcTerm), ip]
    lib.nrgb_dm_backward.argtypes = [vp, C.c_int, C.POINTER(DmOut), C.c_int, C.POINTER(DmTerm), ip]
    lib.nrgb_spectrum_fdm.argtypes = [vp, C.c_int, C.POINTER(FdmPair), C.c_double, C.c_double, C.c_int,
                                      C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, dp]
    lib.nrgb_spectrum_dmnrg.argtypes = [vp, C.c_int, C.POINTER(DmnrgPair), C.c_double, C.c_double, C.c_double,
                                        C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, dp]
    lib.nrgb_set_schedule.argtypes = [vp, C.c_int, C.c_int]
    lib.nrgb_get_schedule.argtypes = [vp, ip, ip, ip]
    lib.nrgb_inject_barrier_shortfall.argtypes = [vp, C.c_int]
    lib.nrgb_eig_recalc_step.argtypes = [vp, C.c_int, ip, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                                         C.c_int, ip, ip, C.POINTER(vp), C.POINTER(vp)]
    lib.nrgb_eig_recalc_step_dev.argtypes = [vp, C.c_int, ip, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                                             C.c_int, ip, ip, C.POINTER(vp), C.POINTER(vp), vp]
    lib.nrgb_profile.argtypes = [vp, C.c_int]
    lib.nrgb_profile_only.argtypes = [vp, C.c_char_p]
    lib.nrgb_kernel_stats.argtypes = [vp, C.c_char_p, C.POINTER(C.c_long), dp]
    lib.nrgb_kernel_work.argtypes = [vp, C.c_char_p, dp]
    lib.nrgb_basis_change_noalloc.argtypes = [C.c_int, ip, ip, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                                              C.POINTER(vp), vp]
    lib.nrgb_server_create.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.POINTER(vp)]
    lib.nrgb_server_submit.argtypes = [vp, C.c_char_p, C.c_char_p, C.POINTER(C.c_longlong)]
    lib.nrgb_server_wait.argtypes = [vp, C.c_longlong, C.c_double, dp]
    lib.nrgb_server_error.argtypes = [vp, C.c_longlong]
    lib.nrgb_server_error.restype = C.c_char_p
    lib.nrgb_server_counters.argtypes = [vp, dp]
    lib.nrgb_server_destroy.argtypes = [vp]
    lib.nrgb_project_bytes.argtypes = [C.c_char_p, dp]
    _lib = lib
    return lib


class Context:
    """One nrgb context on a CUDA device."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        rc = self.lib.nrgb_create(device, C.byref(h))
        if rc != 0:
            raise RuntimeError("nrgb_create failed (status %d): no usable CUDA device" % rc)
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.nrgb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError("%s failed: %s" % (what, self.lib.nrgb_last_error(self.h).decode()))

    # -- eigensolver --
    def syev_batched(self, mats):
        """Host-memory batch: list of symmetric float64 numpy arrays ->
        (eigenvalues list, eigenvector list).  Inputs are not modified."""
        import numpy as np
        n = (C.c_int * len(mats))(*[m.shape[0] for m in mats])
        bufs = [np.asfortranarray(m, dtype=np.float64).copy(order="F") for m in mats]
        ws = [np.empty(m.shape[0]) for m in mats]
        a = (C.c_void_p * len(mats))(*[b.ctypes.data for b in bufs])
        w = (C.c_void_p * len(mats))(*[x.ctypes.data for x in ws])
        self._check(self.lib.nrgb_syev_batched(self.h, len(mats), n, a, w), "nrgb_syev_batched")
        return ws, bufs

    def syev_batched_dev(self, ns, a_ptrs, w_ptrs, z_ptrs, stream=0):
        k = len(ns)
        self._check(self.lib.nrgb_syev_batched_dev(
            self.h, k, (C.c_int * k)(*ns), (C.c_void_p * k)(*a_ptrs), (C.c_void_p * k)(*w_ptrs),
            (C.c_void_p * k)(*z_ptrs), C.c_void_p(stream)), "nrgb_syev_batched_dev")

    def gemm_grouped_dev(self, outs, terms, stream=0):
        o = (GemmOut * len(outs))(*outs)
        t = (GemmTerm * len(terms))(*terms)
        self._check(self.lib.nrgb_gemm_grouped_dev(self.h, len(outs), o, len(terms), t, C.c_void_p(stream)),
                    "nrgb_gemm_grouped_dev")

    def gemm_grouped_split_dev(self, slices, outs, terms, stream=0):
        """Split-precision (INT8 slices, tensor cores) form of gemm_grouped_dev."""
        o = (GemmOut * len(outs))(*outs)
        t = (GemmTerm * len(terms))(*terms)
        self._check(self.lib.nrgb_gemm_grouped_split_dev(self.h, slices, len(outs), o, len(terms), t,
                                                         C.c_void_p(stream)), "nrgb_gemm_grouped_split_dev")

    @staticmethod
    def _ptrs(xs):
        return (C.c_void_p * len(xs))(*[int(x) if x is not None else None for x in xs])

    def eig_recalc_step(self, ns, h, w, z, bra, ket, op, out):
        """Host-memory step: pointers are addresses of column-major float64 buffers."""
        nb, no = len(ns), len(bra)
        self._check(self.lib.nrgb_eig_recalc_step(
            self.h, nb, (C.c_int * nb)(*ns), self._ptrs(h), self._ptrs(w), self._ptrs(z) if z else None,
            no, (C.c_int * no)(*bra), (C.c_int * no)(*ket), self._ptrs(op), self._ptrs(out)),
            "nrgb_eig_recalc_step")

    def eig_recalc_step_dev(self, ns, a, w, z, bra, ket, op, out, stream=0):
        nb, no = len(ns), len(bra)
        self._check(self.lib.nrgb_eig_recalc_step_dev(
            self.h, nb, (C.c_int * nb)(*ns), self._ptrs(a), self._ptrs(w), self._ptrs(z),
            no, (C.c_int * no)(*bra), (C.c_int * no)(*ket), self._ptrs(op), self._ptrs(out),
            C.c_void_p(stream)), "nrgb_eig_recalc_step_dev")

    def profile(self, enable=True, only=None):
        """Launch accounting on (counters reset) or off; with `only` (a kernel
        name, or a prefix ending in '*'), only those launches are timed."""
        if enable and only:
            self._check(self.lib.nrgb_profile_only(self.h, only.encode()), "nrgb_profile_only")
        else:
            self._check(self.lib.nrgb_profile(self.h, 1 if enable else 0), "nrgb_profile")

    def kernel_stats(self, name="*"):
        n = C.c_long()
        ms = C.c_double()
        self._check(self.lib.nrgb_kernel_stats(self.h, name.encode(), C.byref(n), C.byref(ms)),
                    "nrgb_kernel_stats")
        return n.value, ms.value

    def kernel_work(self, name="*"):
        """Algorithmic work (bytes or flops) stated for the launches of `name`."""
        w = C.c_double()
        self._check(self.lib.nrgb_kernel_work(self.h, name.encode(), C.byref(w)), "nrgb_kernel_work")
        return w.value

    def set_eig_mode(self, mode: int):
        """0: one batched eigensolver call per step; 1: one call per block."""
        self._check(self.lib.nrgb_set_eig_mode(self.h, mode), "nrgb_set_eig_mode")

    def autotune(self):
        """Measure and set the device's schedule; returns the report (dict)."""
        import json
        buf = C.create_string_buffer(1 << 16)
        self._check(self.lib.nrgb_autotune(self.h, buf, len(buf)), "nrgb_autotune")
        return json.loads(buf.value.decode())

    def set_schedule(self, cluster_limit: int = 0, gemm_large_from: int = 0):
        self._check(self.lib.nrgb_set_schedule(self.h, cluster_limit, gemm_large_from), "nrgb_set_schedule")

    def get_schedule(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._check(self.lib.nrgb_get_schedule(self.h, C.byref(a), C.byref(b), C.byref(c)), "nrgb_get_schedule")
        return {"cluster_limit": a.value, "gemm_large_from": b.value, "cluster_capacity": c.value}

    # -- step-level plan --
    def mat_upload(self, M):
        import numpy as np
        M = np.asfortranarray(np.atleast_2d(np.asarray(M, dtype=np.float64)))
        h = C.c_int()
        self._check(self.lib.nrgb_mat_upload(self.h, M.shape[0], M.shape[1], M.ctypes.data, C.byref(h)),
                    "nrgb_mat_upload")
        return h.value

    def mat_download(self, handle):
        import numpy as np
        r, c = C.c_int(), C.c_int()
        self._check(self.lib.nrgb_mat_shape(self.h, handle, C.byref(r), C.byref(c)), "nrgb_mat_shape")
        out = np.empty((r.value, c.value), order="F")
        self._check(self.lib.nrgb_mat_download(self.h, handle, out.ctypes.data), "nrgb_mat_download")
        return out

    def mat_free(self, handle):
        self._check(self.lib.nrgb_mat_free(self.h, handle), "nrgb_mat_free")

    def run_begin(self):
        self._check(self.lib.nrgb_run_begin(self.h), "nrgb_run_begin")

    def step(self, dims, diag_terms, off_terms, rules):
        """One NRG step (nrgb_step); rules: dict of the truncation fields.
        Returns (z_handles, w_handles, kept, egs, zsums)."""
        import numpy as np
        nb = len(dims)
        dim = (C.c_int * nb)(*dims)
        dt = (DiagTerm * max(1, len(diag_terms)))(*diag_terms)
        ot = (OffdiagTerm * max(1, len(off_terms)))(*off_terms)
        plan = StepPlan(nb, dim, len(diag_terms), dt, len(off_terms), ot, rules["fixeps"], rules["keepenergy"],
                        rules["keep"], rules["keepmin"], rules["safeguard"], rules["safeguardmax"],
                        rules.get("keep_all", 0), rules["betabar"])
        zh, wh, kept = (C.c_int * nb)(), (C.c_int * nb)(), (C.c_int * nb)()
        egs = C.c_double()
        zs = (C.c_double * (3 * nb))()
        self._check(self.lib.nrgb_step(self.h, C.byref(plan), zh, wh, kept, C.byref(egs), zs), "nrgb_step")
        return list(zh), list(wh), list(kept), egs.value, np.array(list(zs)).reshape(nb, 3)

    def recalc(self, outs, terms):
        n = len(outs)
        o = (RecalcOut * max(1, n))(*outs)
        t = (RecalcTerm * max(1, len(terms)))(*terms)
        hs = (C.c_int * max(1, n))()
        self._check(self.lib.nrgb_recalc(self.h, n, o, len(terms), t, hs), "nrgb_recalc")
        return list(hs)[:n]

    def dm_backward(self, outs, terms):
        """Density-matrix backward step (nrgb_dm_backward): one new handle per
        output, out = sum factor * Z1sub rho Zpsub^T."""
        n = len(outs)
        o = (DmOut * max(1, n))(*outs)
        t = (DmTerm * max(1, len(terms)))(*terms)
        hs = (C.c_int * max(1, n))()
        self._check(self.lib.nrgb_dm_backward(self.h, n, o, len(terms), t, hs), "nrgb_dm_backward")
        return list(hs)[:n]

    def spectrum_fdm(self, pairs, T, wn, fermionic, bins_per_decade, emin, emax, discard=1e-16):
        """FDM spectral weights of block pairs binned on the log grid
        (nrgb_spectrum_fdm): returns (positive, negative) bin arrays."""
        import numpy as np
        nb = int((math.ceil(math.log10(emax)) - math.floor(math.log10(emin))) * bins_per_decade + 1.0)
        p = (FdmPair * max(1, len(pairs)))(*pairs)
        out = np.zeros(2 * nb)
        self._check(self.lib.nrgb_spectrum_fdm(self.h, len(pairs), p, T, wn, int(fermionic), bins_per_decade, emin,
                                               emax, discard, nb, out.ctypes.data_as(C.POINTER(C.c_double))),
                    "nrgb_spectrum_fdm")
        return out[:nb], out[nb:]

    def spectrum_dmnrg(self, pairs, scale, ewin_min, ewin_max, fermionic, bins_per_decade, emin, emax,
                       discard=1e-16):
        """DM-NRG spectral weights of block pairs binned on the log grid
        (nrgb_spectrum_dmnrg): returns (positive, negative) bin arrays."""
        import numpy as np
        nb = int((math.ceil(math.log10(emax)) - math.floor(math.log10(emin))) * bins_per_decade + 1.0)
        p = (DmnrgPair * max(1, len(pairs)))(*pairs)
        out = np.zeros(2 * nb)
        self._check(self.lib.nrgb_spectrum_dmnrg(self.h, len(pairs), p, scale, ewin_min, ewin_max, int(fermionic),
                                                 bins_per_decade, emin, emax, discard, nb,
                                                 out.ctypes.data_as(C.POINTER(C.c_double))), "nrgb_spectrum_dmnrg")
        return out[:nb], out[nb:]

    def set_wait_limit(self, poll_log2: int):
        """Device barrier waits give up after 2**poll_log2 polls (default 23)."""
        self._check(self.lib.nrgb_set_wait_limit(self.h, poll_log2), "nrgb_set_wait_limit")

    def inject_barrier_shortfall(self, on: bool):
        """Fault injection: panel launches wait for a CTA that never arrives."""
        self._check(self.lib.nrgb_inject_barrier_shortfall(self.h, 1 if on else 0),
                    "nrgb_inject_barrier_shortfall")

    def run(self, workdir: str, outdir: str):
        stats = (C.c_double * 8)()
        self._check(self.lib.nrgb_run(self.h, workdir.encode(), outdir.encode(), stats), "nrgb_run")
        return dict(zip(RUN_KEYS, list(stats)))


RUN_KEYS = ["wall_s", "diag_s", "recalc_s", "dm_s", "spec_s", "launches", "h2d_bytes", "d2h_bytes"]
SERVED_KEYS = RUN_KEYS + ["latency_s", "queue_s", "projected_bytes", "peak_bytes", "eig_calls", "order"]
COUNTER_KEYS = ["done", "failed", "eig_calls", "eig_requests", "eig_blocks", "peak_running",
                "peak_admitted_bytes", "budget_bytes"]


def project_bytes(workdir: str) -> float:
    """Projected device bytes of one run (host only, no device needed)."""
    lib = load()
    b = C.c_double()
    rc = lib.nrgb_project_bytes(workdir.encode(), C.byref(b))
    if rc != 0:
        raise RuntimeError("nrgb_project_bytes failed (status %d) for %s" % (rc, workdir))
    return b.value


class Server:
    """Run server on one device: submit() queues an NRG run, wait() returns
    its statistics (SERVED_KEYS).  Thread-safe."""

    def __init__(self, device: int = 0, max_runs: int = 8, mem_budget_bytes: float = 0.0,
                 batch_window_us: float = 2000.0):
        self.lib = load()
        h = C.c_void_p()
        rc = self.lib.nrgb_server_create(device, max_runs, mem_budget_bytes, batch_window_us, C.byref(h))
        if rc != 0:
            raise RuntimeError("nrgb_server_create failed (status %d)" % rc)
        self.h = h

    def submit(self, workdir: str, outdir: str) -> int:
        t = C.c_longlong()
        rc = self.lib.nrgb_server_submit(self.h, workdir.encode(), outdir.encode(), C.byref(t))
        if rc != 0:
            raise RuntimeError("nrgb_server_submit failed: %s" % self.lib.nrgb_server_error(self.h, 0).decode())
        return t.value

    def wait(self, ticket: int, timeout_s: float = -1.0):
        stats = (C.c_double * 14)()
        rc = self.lib.nrgb_server_wait(self.h, ticket, timeout_s, stats)
        if rc == 7:
            raise TimeoutError("run %d not finished after %.1f s" % (ticket, timeout_s))
        if rc != 0:
            raise RuntimeError("run %d failed: %s" % (ticket, self.lib.nrgb_server_error(self.h, ticket).decode()))
        return dict(zip(SERVED_KEYS, list(stats)))

    def counters(self):
        out = (C.c_double * 8)()
        self.lib.nrgb_server_counters(self.h, out)
        return dict(zip(COUNTER_KEYS, list(out)))

    def close(self):
        if getattr(self, "h", None):
            self.lib.nrgb_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
