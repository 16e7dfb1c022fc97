"""ctypes binding of libexmarg_b200.so (include/exmarg_b200.h) and the device context.

The library is built in-tree (exmarg_b200/build.py).  There is no CPU fallback:
if the shared library is missing or no CUDA device can be opened, every call
raises.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libexmarg_b200.so")

EXM_OK, EXM_ERR_ARG, EXM_ERR_OOM, EXM_ERR_CUDA, EXM_ERR_TIMEOUT, EXM_ERR_STATE = range(6)
DTYPE_F32, DTYPE_F16, DTYPE_BF16 = 0, 1, 2
PRIOR_VOLUME, PRIOR_TABULATED = 0, 1
QUAD_GL64 = 16   # OR'ed into the prior: 64-point Gauss-Legendre distance quadrature
# the plane gather's launch shapes, in exm_autotune / exm_set_gather_cfg order (warps per block x taps
# per register group)
GATHER_SHAPES = ("28w x1", "16w x2", "24w x2", "24w x1", "20w x2")

# every symbol include/exmarg_b200.h declares
SYMBOLS = ("exm_version", "exm_rng_integers", "exm_gauss_legendre", "exm_device_memory", "exm_ctx_timing", "exm_ctx_create_sharing", "exm_ctx_set_graph", "exm_ctx_set_priority", "exm_ctx_test_wait_expiry", "exm_ctx_set_filter_precision", "exm_ctx_create", "exm_ctx_destroy", "exm_last_error", "exm_ctx_bytes", "exm_store_init",
           "exm_store_set_node", "exm_store_generate_node", "exm_store_get_node", "exm_bank_set", "exm_pe_prepare",
           "exm_pe_intrinsic", "exm_filter", "exm_set_trajectories", "exm_select_times", "exm_np_exp32", "exm_set_times",
           "exm_gather", "exm_node_values", "exm_gather_noalloc", "exm_autotune", "exm_set_gather_cfg",
           "exm_redshift_grid", "exm_source_frame", "exm_serve_start", "exm_serve_add_bank", "exm_submit", "exm_poll",
           "exm_serve_stats", "exm_serve_stop", "exm_serve_set_min_idle", "exm_store_load", "exm_store_set_shard", "exm_bd_build", "exm_w_build", "exm_k_edges")

LOAD_DIRECT = 1
LOAD_STATS = ("seconds", "file_bytes", "host_bytes", "direct_nodes", "buffers", "chunk_bytes", "read_seconds",
              "issue_wait_seconds")

_lib = None


def _p(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def load():
    """the shared library with argument types set (raises if it is not built)"""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libexmarg_b200.so is not built: run python -m exmarg_b200.build (or __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    P, I, D, Z = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t
    sig = {
        "exm_version": ([], I),
        "exm_device_memory": ([I, ctypes.POINTER(Z), ctypes.POINTER(Z)], I),
        "exm_rng_integers": ([ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int64, P], I),
        "exm_gauss_legendre": ([I, P, P], I),
        "exm_ctx_create": ([I, Z, ctypes.POINTER(P)], I),
        "exm_ctx_destroy": ([P], None),
        "exm_ctx_create_sharing": ([P, Z, ctypes.POINTER(P)], I),
        "exm_ctx_set_graph": ([P, I], I),
        "exm_ctx_set_priority": ([P, I, P], I),
        "exm_ctx_test_wait_expiry": ([P, I], I),
        "exm_ctx_set_filter_precision": ([P, I], I),
        "exm_last_error": ([P], ctypes.c_char_p),
        "exm_ctx_bytes": ([P], Z),
        "exm_ctx_timing": ([P, I, P], I),
        "exm_store_init": ([P, I, I, I, I, I, I, P, D, D, D, D], I),
        "exm_store_set_node": ([P, I, D, D, D, P], I),
        "exm_store_generate_node": ([P, I, D, D, D, P, P, P, ctypes.c_float, ctypes.c_uint32], I),
        "exm_store_get_node": ([P, I, P], I),
        "exm_bank_set": ([P, I, I, I, I, P, P, P, P, P], I),
        "exm_pe_prepare": ([P, D, I, P, P, I], I),
        "exm_pe_intrinsic": ([P, I, P, P, P, P, P, I, I, P, P], I),
        "exm_filter": ([P, P, P, P, P, P], I),
        "exm_set_trajectories": ([P, P], I),
        "exm_select_times": ([P, ctypes.c_int64, I, I, P, P], I),
        "exm_np_exp32": ([P, P, P, ctypes.c_int64], I),
        "exm_set_times": ([P, I, P, P], I),
        "exm_gather": ([P, I, I, P, P, P, P], I),
        "exm_node_values": ([P, P], I),
        "exm_gather_noalloc": ([P, I, I, P, P, P, P, I, P, P, I, I, P, P, P, P], I),
        "exm_autotune": ([P, I, I, I, P, P, P], I),
        "exm_set_gather_cfg": ([P, I, I], I),
        "exm_redshift_grid": ([P, I, I, P, P, I, P, P, I, P, P], I),
        "exm_serve_start": ([P, Z, I, I, I, I], I),
        "exm_serve_add_bank": ([P, I, I, I, I, P, P, P, P, P, D, I, P, P, I, P], I),
        "exm_submit": ([P, I, P, P, P, P, ctypes.c_int64, P], I),
        "exm_poll": ([P, ctypes.c_int64, ctypes.c_int64, P, P], I),
        "exm_serve_stats": ([P, P], I),
        "exm_serve_stop": ([P], I),
        "exm_serve_set_min_idle": ([P, D], I),
        "exm_source_frame": ([P, P, P, P], I),
        "exm_store_load": ([P, I, I, P, P, P, P, P, P, I, ctypes.c_longlong, I, P], I),
        "exm_store_set_shard": ([P, D], I),
        "exm_bd_build": ([P, I, I, I, I, P, P, P, I, P, I, P, P, P, P], I),
        "exm_w_build": ([P, I, P, I, I, I, P, P, P, P, P, I, P, P, P, I, P, P, P, P], I),
        "exm_k_edges": ([P, I, I, P, P, I, P, P, I, P, P, P, P], I),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def rng_integers(seed, high, count):
    """np.random.default_rng(seed).integers(0, high, count), by the library's host PCG64 code"""
    out = np.empty(int(count), np.int64)
    rc = load().exm_rng_integers(int(seed), int(high), int(count), _p(out))
    if rc != EXM_OK:
        _raise(rc, "bad rng arguments")
    return out


def gauss_legendre(n):
    """the n-point Gauss-Legendre nodes and weights on [-1, 1], by the library's host code"""
    x, w = np.empty(int(n)), np.empty(int(n))
    rc = load().exm_gauss_legendre(int(n), _p(x), _p(w))
    if rc != EXM_OK:
        _raise(rc, "n must be 1..256")
    return x, w


def device_memory(device=0):
    """(free, total) bytes of a CUDA device"""
    f, t = ctypes.c_size_t(), ctypes.c_size_t()
    rc = load().exm_device_memory(int(device), ctypes.byref(f), ctypes.byref(t))
    if rc != EXM_OK:
        _raise(rc, "cannot query CUDA device %d" % device)
    return f.value, t.value


def _raise(code, msg):
    if code == EXM_ERR_ARG:
        raise ValueError(msg)
    if code == EXM_ERR_OOM:
        raise MemoryError(msg)
    raise RuntimeError(msg)


class Context:
    """one device context of libexmarg_b200 (tables, bank, workspaces, one stream)"""

    def __init__(self, device=0, hbm_budget=0, share_store_of=None):
        self.lib = load()
        h = ctypes.c_void_p()
        if share_store_of is not None:
            rc = self.lib.exm_ctx_create_sharing(share_store_of.h, int(hbm_budget), ctypes.byref(h))
            if rc != EXM_OK:
                _raise(rc, share_store_of.lib.exm_last_error(share_store_of.h).decode())
            device = share_store_of.device
            self.parent = share_store_of            # keeps the store's owner alive
            self.filter_precision = getattr(share_store_of, "filter_precision", "reference")   # inherited
        else:
            rc = self.lib.exm_ctx_create(int(device), int(hbm_budget), ctypes.byref(h))
            if rc != EXM_OK:
                _raise(rc, "cannot open CUDA device %d for libexmarg_b200 (status %d)" % (device, rc))
        self.h = h
        self.device = device
        self.store_token = share_store_of.store_token if share_store_of is not None else None
        self.bank_token = None
        self.prep_token = None
        self.nm = self.nfreq = self.n_time = None
        self.gather_cfg = None          # the launch shape chosen by autotune or set_gather_cfg (None: default)
        self.gather_chunk_pct = 150     # templates per gather block, percent of one wave of blocks per lag
        self.store_shape = None         # (nodes, lags, phase planes, nb, nd, dtype) of the resident store
        self.device_total = device_memory(device)[1]   # identifies the device model in the autotune cache

    def set_graph(self, enable=True):
        """replay each segment's device work as one captured CUDA graph"""
        self._check(self.lib.exm_ctx_set_graph(self.h, 1 if enable else 0))

    FILTER_PRECISIONS = ("reference", "fp64")

    def set_filter_precision(self, precision):
        """'reference' (ln|z| rounded to float32 as the reference leaves it) or 'fp64' (ln|z| kept to float64)"""
        if precision not in self.FILTER_PRECISIONS:
            raise ValueError("filter_precision must be 'reference' or 'fp64'")
        if getattr(self, "filter_precision", "reference") != precision:
            self._check(self.lib.exm_ctx_set_filter_precision(self.h, self.FILTER_PRECISIONS.index(precision)))
            self.filter_precision = precision

    def test_wait_expiry(self, enable=True):
        """test support: the plane gather stages nothing, so its bounded waits run out (EXM_ERR_TIMEOUT)"""
        self._check(self.lib.exm_ctx_test_wait_expiry(self.h, 1 if enable else 0))

    def set_priority(self, priority):
        """stream priority (0 default, lower numbers first; clamped); returns the device's
        (greatest, least) priorities"""
        rng = np.zeros(2, np.int32)
        self._check(self.lib.exm_ctx_set_priority(self.h, int(priority), _p(rng)))
        return int(rng[0]), int(rng[1])

    def close(self):
        if getattr(self, "h", None):
            self.lib.exm_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != EXM_OK:
            _raise(rc, self.lib.exm_last_error(self.h).decode())

    @property
    def bytes(self):
        return int(self.lib.exm_ctx_bytes(self.h))

    def timing(self, enable=True):
        """stage times accumulated since the previous call (CUDA events on the context's stream),
        then reset; enable turns timing on or off for the following calls"""
        out = np.zeros(16, np.float64)
        self._check(self.lib.exm_ctx_timing(self.h, 1 if enable else 0, _p(out)))
        keys = ("total_ms", "filter_ms", "select_ms", "taps_ms", "gather_ms", "epilogue_ms", "gather_launches",
                "node_taps", "tlw_taps", "segments", "launches", "slow_taps", "boundary_taps")
        return dict(zip(keys, out[:len(keys)]))

    # store ------------------------------------------------------------
    def store_init(self, n_nodes, shape, tau_idx, beta0, dbeta, delta0, ddelta, dtype=DTYPE_F32):
        ntau, nphif, nb, nd = shape
        tau = np.ascontiguousarray(tau_idx, np.int64)
        self._check(self.lib.exm_store_init(self.h, n_nodes, ntau, nphif, nb, nd, dtype, _p(tau), beta0, dbeta,
                                            delta0, ddelta))
        self.store_token = self.prep_token = None
        self.store_shape = (int(n_nodes), int(ntau), int(nphif), int(nb), int(nd), int(dtype))

    def store_set_node(self, k, s, alpha_lo, alpha_hi, T):
        T = np.ascontiguousarray(T, np.float32)
        self._check(self.lib.exm_store_set_node(self.h, k, s, alpha_lo, alpha_hi, _p(T)))

    def store_load(self, first, s, alpha_lo, alpha_hi, paths=None, offsets=None, hosts=None, readers=6, chunk_bytes=0,
                   direct=False):
        """nodes first.. from files (paths[i] at byte offsets[i]) or host tables (hosts[i], where paths[i] is
        None) in one pipelined pass; returns the loader's statistics (LOAD_STATS)"""
        n = len(s)
        s, alo, ahi = (np.ascontiguousarray(x, np.float64) for x in (s, alpha_lo, alpha_hi))
        if not (alo.size == ahi.size == n):
            raise ValueError("one s, alpha_lo, alpha_hi per node")
        c_paths = c_offs = c_hosts = None
        keep = []
        if paths is not None:
            if len(paths) != n or offsets is None or len(offsets) != n:
                raise ValueError("one path and one offset per node")
            c_paths = (ctypes.c_char_p * n)(*[None if p is None else os.fsencode(p) for p in paths])
            c_offs = np.ascontiguousarray([0 if o is None else int(o) for o in offsets], np.int64)
        if hosts is not None:
            if len(hosts) != n:
                raise ValueError("one host table (or None) per node")
            keep = [None if h is None else np.ascontiguousarray(h, np.float32) for h in hosts]
            c_hosts = (ctypes.c_void_p * n)(*[None if h is None else h.ctypes.data for h in keep])
        st = np.zeros(len(LOAD_STATS))
        self._check(self.lib.exm_store_load(self.h, int(first), n, c_paths, _p(c_offs), c_hosts, _p(s), _p(alo), _p(ahi),
                                            int(readers), int(chunk_bytes), LOAD_DIRECT if direct else 0, _p(st)))
        del keep
        return dict(zip(LOAD_STATS, st.tolist()))

    def store_set_shard(self, s_before):
        """this context's store is a node range of a larger store; s_before: the s of the node below it"""
        self._check(self.lib.exm_store_set_shard(self.h, float(s_before)))
        self.prep_token = None

    def bd_build(self, col, row, lnq, beta, ladder):
        """stage 3 of the table build: (T (n_ladder, ntau, nphif, nb, 2 nq - 1) float32, entries not
        finite, (kernel ms, ms with copies))"""
        col = np.ascontiguousarray(col, np.float32)
        row = np.ascontiguousarray(row, np.float32)
        if col.ndim != 4 or col.shape != row.shape:
            raise ValueError("col and row must both be (orders, lags, nq, phases)")
        nord, ntau, nq, nphif = col.shape
        lnq = np.ascontiguousarray(lnq, np.float64)
        beta = np.ascontiguousarray(beta, np.float64)
        lad = np.ascontiguousarray(ladder, np.int32)
        if lnq.size != nq:
            raise ValueError("lnq must have one entry per magnitude")
        T = np.empty((lad.size, ntau, nphif, beta.size, 2 * nq - 1), np.float32)
        bad = ctypes.c_longlong(0)
        ms = np.zeros(2)
        self._check(self.lib.exm_bd_build(self.h, nord, ntau, nq, nphif, _p(col), _p(row), _p(lnq), beta.size, _p(beta),
                                          lad.size, _p(lad), _p(T), ctypes.byref(bad), _p(ms)))
        return T, int(bad.value), (float(ms[0]), float(ms[1]))

    def k_edges(self, n_max, Wd, coeff, lnq, gmo, cosm):
        """stage 2 on the boundary of the (q1, q2) grid: (col, row) float32 (n_max+1, n_tau, nq, nphif) and
        the kernel milliseconds"""
        Wd = np.ascontiguousarray(Wd, np.float64)
        n_keys, n_tau = Wd.shape
        if n_keys != (n_max + 1) * (n_max + 2) * (n_max + 3) // 6:
            raise ValueError("Wd must hold every key (n, a, b <= a) of orders 0..n_max")
        coeff, lnq, gmo, cosm = (np.ascontiguousarray(x, np.float64) for x in (coeff, lnq, gmo, cosm))
        if coeff.size != n_keys or gmo.size != n_max + 1 or cosm.shape[0] != n_max + 1:
            raise ValueError("one coefficient per key, one offset and one cosine row per order")
        nq, nphif = lnq.size, cosm.shape[1]
        col = np.empty((n_max + 1, n_tau, nq, nphif), np.float32)
        row = np.empty_like(col)
        ms = np.zeros(1)
        self._check(self.lib.exm_k_edges(self.h, n_max, n_tau, _p(Wd), _p(coeff), nq, _p(lnq), _p(gmo), nphif, _p(cosm),
                                         _p(col), _p(row), _p(ms)))
        return col, row, float(ms[0])

    def w_build(self, s_nodes, n_max, g, scale):
        """stage 1 of the table build over the pixels of geometry g (exmarg_b200.wtable.geometry): W
        (n_nodes, n_tau, n_keys) float32 and (milliseconds of the quadrature, milliseconds in all)"""
        s_nodes = np.ascontiguousarray(s_nodes, np.float64)
        n_keys = (n_max + 1) * (n_max + 2) * (n_max + 3) // 6
        scale = np.ascontiguousarray(scale, np.float64)
        if scale.shape != (s_nodes.size, n_keys):
            raise ValueError("scale must be (nodes, keys)")
        arr = {k: np.ascontiguousarray(g[k]) for k in ("resp", "j0", "w", "c2p", "s2p", "ap", "cg", "wq")}
        n_tau = int(g["tau"].size)
        W = np.empty((s_nodes.size, n_tau, n_keys), np.float32)
        bad = ctypes.c_longlong(0)
        ms = np.zeros(2)
        self._check(self.lib.exm_w_build(self.h, s_nodes.size, _p(s_nodes), int(n_max), arr["c2p"].size, arr["ap"].size,
                                         _p(arr["c2p"]), _p(arr["s2p"]), _p(arr["ap"]), _p(arr["cg"]), _p(arr["wq"]),
                                         arr["resp"].shape[0], _p(arr["resp"]), _p(arr["j0"]), _p(arr["w"]), n_tau,
                                         _p(scale), _p(W), ctypes.byref(bad), _p(ms)))
        if bad.value:
            raise FloatingPointError("conditional W table non-finite")
        return W, (float(ms[0]), float(ms[1]))

    def store_generate_node(self, k, s, alpha_lo, alpha_hi, M, P, Q, S, seed):
        M, P, Q = (np.ascontiguousarray(x, np.float32) for x in (M, P, Q))
        self._check(self.lib.exm_store_generate_node(self.h, k, s, alpha_lo, alpha_hi, _p(M), _p(P), _p(Q),
                                                     ctypes.c_float(S), ctypes.c_uint32(seed)))

    def store_get_node(self, k, shape):
        out = np.empty(shape, np.float32)
        self._check(self.lib.exm_store_get_node(self.h, k, _p(out)))
        return out

    # bank ---------------------------------------------------------------
    def bank_set(self, W, lo, n_time, u, M, q, chi):
        W = np.ascontiguousarray(W, np.complex64)
        u, M, q, chi = (np.ascontiguousarray(x, np.float64) for x in (u, M, q, chi))
        nm, nf = W.shape
        self._check(self.lib.exm_bank_set(self.h, nm, nf, int(lo), int(n_time), _p(W), _p(u), _p(M), _p(q), _p(chi)))
        self.nm, self.nfreq, self.n_time = nm, nf, int(n_time)
        self.prep_token = None

    def prepare(self, ymin, prior, density=None, gl64=False):
        q = QUAD_GL64 if gl64 else 0
        if prior == PRIOR_TABULATED:
            lny = np.ascontiguousarray(density[0], np.float64)
            p = np.ascontiguousarray(density[1], np.float64)
            self._check(self.lib.exm_pe_prepare(self.h, float(ymin), prior | q, _p(lny), _p(p), lny.size))
        else:
            self._check(self.lib.exm_pe_prepare(self.h, float(ymin), PRIOR_VOLUME | q, None, None, 0))

    # analysis -------------------------------------------------------------
    def pe_intrinsic(self, d_H, d_L, sig2_H, sig2_L, seeds, n_loud, n_random):
        d_H = np.ascontiguousarray(d_H, np.complex128)
        d_L = np.ascontiguousarray(d_L, np.complex128)
        sig2_H = np.ascontiguousarray(sig2_H, np.float64)
        sig2_L = np.ascontiguousarray(sig2_L, np.float64)
        n = d_H.shape[0]
        if d_H.shape[1] != self.nfreq or d_L.shape != d_H.shape or sig2_H.size != self.nfreq:
            raise ValueError("segment frequency bins (%d) do not match the bank (%d)" % (d_H.shape[1], self.nfreq))
        seeds = np.ascontiguousarray(seeds, np.int64)
        lnl = np.empty((n, self.nm), np.float64)
        lnb = np.empty(n, np.float64)
        self._check(self.lib.exm_pe_intrinsic(self.h, n, _p(d_H), _p(d_L), _p(sig2_H), _p(sig2_L), _p(seeds),
                                              int(n_loud), int(n_random), _p(lnl), _p(lnb)))
        return lnl, lnb

    def filter(self, d_H, d_L, sig2_H, sig2_L, want=True):
        d_H = np.ascontiguousarray(d_H, np.complex128)
        d_L = np.ascontiguousarray(d_L, np.complex128)
        sig2_H = np.ascontiguousarray(sig2_H, np.float64)
        sig2_L = np.ascontiguousarray(sig2_L, np.float64)
        out = np.empty((4, self.nm, self.n_time), np.float32) if want else None
        self._check(self.lib.exm_filter(self.h, _p(d_H), _p(d_L), _p(sig2_H), _p(sig2_L), _p(out)))
        if out is None:
            return None
        return dict(lqH=out[0], phH=out[1], lqL=out[2], phL=out[3])

    def set_trajectories(self, traj):
        out = np.ascontiguousarray(np.stack([traj["lqH"], traj["phH"], traj["lqL"], traj["phL"]]), np.float32)
        self._check(self.lib.exm_set_trajectories(self.h, _p(out)))

    def select_times(self, seed, n_loud, n_random, want=True):
        """the visited times (on the device); with want, also (sel, lw) on the host"""
        nw = n_loud + n_random
        sel = np.empty((self.nm, nw), np.int32) if want else None
        lw = np.empty((self.nm, nw), np.float32) if want else None
        self._check(self.lib.exm_select_times(self.h, int(seed), int(n_loud), int(n_random), _p(sel), _p(lw)))
        return (sel, lw) if want else None

    def np_exp32(self, x):
        """numpy's float32 exp evaluated on the device (the selection score's exp)"""
        x = np.ascontiguousarray(x, np.float32)
        y = np.empty_like(x)
        self._check(self.lib.exm_np_exp32(self.h, _p(x), _p(y), x.size))
        return y

    def set_times(self, times):
        if times is None:
            self._check(self.lib.exm_set_times(self.h, 0, None, None))
            return
        sel = np.ascontiguousarray(times[0], np.int32)
        lw = np.ascontiguousarray(times[1], np.float32)
        self._check(self.lib.exm_set_times(self.h, sel.shape[1], _p(sel), _p(lw)))

    def gather(self, mass_ids, lna, tab_ids):
        ids = np.ascontiguousarray(mass_ids, np.int64)
        lna = np.ascontiguousarray(lna, np.float64)
        tab = np.ascontiguousarray(tab_ids, np.int64)
        nsel, ns = tab.shape
        out = np.empty((ns, nsel), np.float64)
        self._check(self.lib.exm_gather(self.h, nsel, ns, _p(ids), _p(lna), _p(tab), _p(out)))
        return out

    # ---------------------------------------------------------------- native request loop

    def serve_start(self, hbm_budget=0, max_workers=4, n_loud=1024, n_random=1024, graph=False):
        self._check(self.lib.exm_serve_start(self.h, int(hbm_budget), int(max_workers), int(n_loud), int(n_random),
                                             1 if graph else 0))

    def serve_add_bank(self, W, lo, n_time, u, M, q, chi, ymin=0.1267, density=None):
        """register a bank (W (nm, nfreq) complex64); returns its id"""
        W = np.ascontiguousarray(W, np.complex64)
        u, M, q, chi = (np.ascontiguousarray(x, np.float64) for x in (u, M, q, chi))
        bid = ctypes.c_int()
        if density is None:
            lny = p = None
            prior, nd = PRIOR_VOLUME, 0
        else:
            lny, p = (np.ascontiguousarray(x, np.float64) for x in density)
            prior, nd = PRIOR_TABULATED, lny.size
        self._check(self.lib.exm_serve_add_bank(self.h, W.shape[0], W.shape[1], int(lo), int(n_time), _p(W), _p(u),
                                                _p(M), _p(q), _p(chi), float(ymin), prior, _p(lny), _p(p), nd,
                                                ctypes.byref(bid)))
        return bid.value

    def submit(self, bank_id, d_H, d_L, sig2_H, sig2_L, seed):
        """queue one segment; returns its handle at once"""
        d_H, d_L = (np.ascontiguousarray(x, np.complex128) for x in (d_H, d_L))
        sig2_H, sig2_L = (np.ascontiguousarray(x, np.float64) for x in (sig2_H, sig2_L))
        h = ctypes.c_int64()
        self._check(self.lib.exm_submit(self.h, int(bank_id), _p(d_H), _p(d_L), _p(sig2_H), _p(sig2_L), int(seed),
                                        ctypes.byref(h)))
        return h.value

    def poll(self, handle, nm, timeout_us=-1):
        """(ln_lambda (nm,), ln_b) of a finished request, or None if it has not finished within timeout_us"""
        lnl = np.empty(int(nm), np.float64)
        lnb = ctypes.c_double()
        rc = self.lib.exm_poll(self.h, int(handle), int(timeout_us), _p(lnl), ctypes.byref(lnb))
        if rc == EXM_ERR_TIMEOUT:
            return None
        self._check(rc)
        return lnl, lnb.value

    SERVE_STATS = ("served", "failed", "queued", "running", "workers", "workers_opened", "workers_closed",
                   "bytes_in_use", "budget", "busy_seconds")

    def serve_stats(self):
        out = np.zeros(len(self.SERVE_STATS), np.float64)
        self._check(self.lib.exm_serve_stats(self.h, _p(out)))
        return dict(zip(self.SERVE_STATS, out.tolist()))

    def serve_set_min_idle(self, seconds):
        """an idle worker is closed for another bank only after `seconds` idle (default 0.25)"""
        self._check(self.lib.exm_serve_set_min_idle(self.h, float(seconds)))

    def serve_stop(self):
        self._check(self.lib.exm_serve_stop(self.h))

    def gather_noalloc(self, nm, n_time, lqH, phH, lqL, phL, nwalk, sel, lw, nsel, ns, mass_ids, lna, tab_ids, out):
        """exm_gather_noalloc: every argument after n_time is a device address (int) the caller owns;
        the call allocates no device memory"""
        P = ctypes.c_void_p
        self._check(self.lib.exm_gather_noalloc(self.h, int(nm), int(n_time), P(lqH), P(phH), P(lqL), P(phL),
                                                int(nwalk), P(sel) if sel else None, P(lw) if lw else None,
                                                int(nsel), int(ns), P(mass_ids), P(lna), P(tab_ids), P(out)))

    def autotune(self, n_loud=1024, n_random=1024, reps=2):
        """time every launch shape of the plane gather on the last segment; keep the fastest.
        returns (best index, ms per launch of each shape)"""
        best, pct = ctypes.c_int(), ctypes.c_int()
        ms = np.zeros(16, np.float64)
        self._check(self.lib.exm_autotune(self.h, int(n_loud), int(n_random), int(reps), ctypes.byref(best),
                                          ctypes.byref(pct), _p(ms)))
        self.gather_cfg = best.value
        self.gather_chunk_pct = pct.value
        return best.value, ms

    def set_gather_cfg(self, cfg, chunk_pct=0):
        """launch shape (index into GATHER_SHAPES) and templates per block in percent of the default
        (0 keeps the current)"""
        self._check(self.lib.exm_set_gather_cfg(self.h, int(cfg), int(chunk_pct)))
        self.gather_cfg = int(cfg)
        if chunk_pct:
            self.gather_chunk_pct = int(chunk_pct)

    def redshift_grid(self, yN, Mdet, yq, z, m1, w):
        """pe_redshift's grid on the device (exm_redshift_grid)"""
        yN, Mdet, yq, z, m1, w = (np.ascontiguousarray(x, np.float64) for x in (yN, Mdet, yq, z, m1, w))
        self._check(self.lib.exm_redshift_grid(self.h, yN.shape[0], yN.shape[1], _p(yN), _p(Mdet), z.size, _p(yq),
                                               _p(z), m1.size, _p(m1), _p(w)))
        self.rs_shape = (m1.size, z.size)

    def source_frame(self, lamN, want=True):
        """(ln_lambda (nm1, nz) or None, ln_b) of one segment's node values"""
        lamN = np.ascontiguousarray(lamN, np.float64)
        out = np.empty(self.rs_shape, np.float64) if want else None
        lnb = np.zeros(1, np.float64)
        self._check(self.lib.exm_source_frame(self.h, _p(lamN), _p(out), _p(lnb)))
        return out, float(lnb[0])

    def node_values(self, n_nodes):
        out = np.empty((n_nodes + 1, self.nm), np.float64)
        self._check(self.lib.exm_node_values(self.h, _p(out)))
        return out


_tokens = iter(range(1, 1 << 62))


def token_of(obj):
    """a process-unique token for a bank or store object (id() values are reused after collection)"""
    t = getattr(obj, "_b200_token", None)
    if t is None:
        t = next(_tokens)
        try:
            object.__setattr__(obj, "_b200_token", t)
        except (AttributeError, TypeError):
            obj.__dict__["_b200_token"] = t
    return t


_contexts = {}


def context(device=0):
    """the process-wide context of a device (created on first use)"""
    if device not in _contexts:
        _contexts[device] = Context(device)
    return _contexts[device]
