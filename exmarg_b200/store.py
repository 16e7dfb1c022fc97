"""The table store (the contract of exmarg/search/store.py:90-127).

load_redshift_store reads every bd_*.npz node of a store directory (T (tau, phi+,
beta, Delta) float32, beta, delta, tau_idx, alpha, s_node), sorted by s_node, into
host memory (or maps them with mmap=True), exactly like the reference.  For
device='b200' the tables are copied once into HBM by the analysis context and
stay resident for every later call (upload_store); there is no per-call upload.
That copy is one pipelined pass of the native loader (exm_store_load): reader
threads fill pinned buffers while earlier chunks go to the device.  A store
loaded with mmap=True is streamed straight from its files (nothing is read into
host memory first), optionally with O_DIRECT (direct=True).
"""

import glob
import os
import struct
import zipfile
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import NamedTuple

import numpy as np

from . import _lib

NPHI = 96


class MemberLayout(NamedTuple):
    """where an array member's raw bytes lie inside an .npz and how to read them"""
    offset: int            # byte offset of the array data in the archive file
    shape: tuple
    fortran: bool
    dtype: np.dtype


_LOCAL_HEADER = struct.Struct("<4s22xHH")    # zip local file header: signature, ..., name length, extra length
_NPY_HEADERS = {(1, 0): np.lib.format.read_array_header_1_0, (2, 0): np.lib.format.read_array_header_2_0}


def npz_member_layout(path, name):
    """The layout of the uncompressed member `name` (an .npy file) of the zip archive `path`.

    The archive's central directory gives the member's local header position; the data follow the
    30-byte local header and its variable name and extra fields (their lengths are the header's last
    two little-endian 16-bit fields).  The data start with the .npy preamble (magic, version, the
    header dictionary with shape, order and dtype); the array bytes come right after it, so they can
    be read with one sequential read, mapped, or handed to a native loader by offset.  A compressed
    member has no such byte range and is refused (ValueError), as the reference's reader refuses it."""
    with zipfile.ZipFile(path) as zf:
        info = zf.getinfo(name)
    if info.compress_type != zipfile.ZIP_STORED:
        raise ValueError("member %s of %s is compressed" % (name, path))
    with open(path, "rb") as fh:
        fh.seek(info.header_offset)
        sig, n_name, n_extra = _LOCAL_HEADER.unpack(fh.read(_LOCAL_HEADER.size))
        if sig != b"PK\x03\x04":
            raise ValueError("no zip local header for %s in %s" % (name, path))
        fh.seek(info.header_offset + _LOCAL_HEADER.size + n_name + n_extra)
        version = np.lib.format.read_magic(fh)
        if version not in _NPY_HEADERS:
            raise ValueError("unsupported .npy version %s in %s" % (version, path))
        shape, fortran, dtype = _NPY_HEADERS[version](fh)
        return MemberLayout(fh.tell(), tuple(shape), bool(fortran), np.dtype(dtype))


def npz_member(path, name, mmap=False):
    """the array of member `name` of the .npz `path`: read into memory, or a read-only map (mmap=True)"""
    lay = npz_member_layout(path, name)
    order = "F" if lay.fortran else "C"
    if mmap:
        return np.asarray(np.memmap(path, dtype=lay.dtype, mode="r", offset=lay.offset, shape=lay.shape, order=order))
    count = int(np.prod(lay.shape))
    arr = np.fromfile(path, dtype=lay.dtype, count=count, offset=lay.offset)
    return arr.reshape(lay.shape, order=order)


@dataclass
class RedshiftStore:
    """signal power nodes s (sorted), amplitude-axis limits, grids, host tables and the truncation order"""
    s: np.ndarray
    alpha_lo: np.ndarray
    alpha_hi: np.ndarray
    beta: list
    delta: list
    tau_idx: np.ndarray
    tables: list
    n_max: int
    device_tokens: dict = field(default_factory=dict, repr=False)
    table_dtype: str = "f32"
    files: list = None          # the bd_*.npz of each node
    t_offsets: list = None      # byte offset of each node's T.npy data (None: not float32 C-order)
    mapped: bool = False        # tables are maps of the files (mmap=True)
    readers: int = 6
    direct: bool = False
    load_stats: dict = field(default=None, repr=False)


TABLE_DTYPES = {"f32": _lib.DTYPE_F32, "f16": _lib.DTYPE_F16, "bf16": _lib.DTYPE_BF16}


def _table_offset(path):
    """byte offset of the T.npy data in a bd_*.npz when it is float32 in C order (else None)"""
    lay = npz_member_layout(path, "T.npy")
    return lay.offset if (lay.dtype == np.dtype("<f4") and (not lay.fortran or len(lay.shape) <= 1)) else None


def load_redshift_store(store_dir, pinned=False, readers=6, mmap=False, table_dtype="f32", direct=False):
    """every node of the store in host memory (about 0.75 GB per node at the production shape);
    pinned is accepted for the reference's signature (the b200 upload stages through its own pinned
    buffers).  mmap=True maps the tables instead; the b200 upload then streams them from the files
    with `readers` threads, with O_DIRECT when direct=True.
    table_dtype: how the b200 path keeps the tables in HBM -- 'f32' (as stored), or 'f16' / 'bf16'
    (half the bytes; see quantize_table for the values it then uses)"""
    if table_dtype not in TABLE_DTYPES:
        raise ValueError("table_dtype must be 'f32', 'f16' or 'bf16'")
    files = glob.glob(os.path.join(store_dir, "bd_*.npz"))
    if not files:
        raise FileNotFoundError("no bd_*.npz in %s" % store_dir)
    head = []
    for f in files:
        with np.load(f) as h:
            head.append((float(h["s_node"]), float(h["alpha"][0]), float(h["alpha"][-1]), h["beta"], h["delta"],
                         h["tau_idx"], f))
    head.sort(key=lambda r: r[0])
    s, alo, ahi, beta, delta, tau, files = zip(*head)
    if mmap:
        tables = [npz_member(f, "T.npy", mmap=True) for f in files]
    else:
        with ThreadPoolExecutor(max_workers=max(1, int(readers))) as ex:
            tables = list(ex.map(lambda f: npz_member(f, "T.npy"), files))
    return RedshiftStore(s=np.array(s), alpha_lo=np.array(alo), alpha_hi=np.array(ahi), beta=list(beta),
                         delta=list(delta), tau_idx=tau[0], tables=tables,
                         n_max=int(os.path.basename(files[0]).split("_n")[1].split("_")[0]), table_dtype=table_dtype,
                         files=list(files), t_offsets=[_table_offset(f) for f in files], mapped=bool(mmap),
                         readers=max(1, min(64, int(readers))), direct=bool(direct))


def with_table_dtype(store, table_dtype):
    """the same store (host tables shared) kept in HBM as table_dtype ('f32', 'f16', 'bf16')"""
    import copy
    if table_dtype not in TABLE_DTYPES:
        raise ValueError("table_dtype must be 'f32', 'f16' or 'bf16'")
    out = copy.copy(store)
    out.__dict__.pop("_b200_token", None)     # a store object of its own
    out.table_dtype = table_dtype
    if hasattr(out, "device_tokens"):
        out.device_tokens = {}
    return out


def _bf16_round(x):
    """float32 -> nearest bfloat16 (ties to even), returned as float32"""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def quantize_table(T, table_dtype):
    """(values, scale): the float32 values the b200 path uses for one node table kept as
    table_dtype, and the node's scale -- the device quantizer restated on the host, bit for bit.
    f16: element = round(T / scale) to float16 (nearest, ties to even), scale = 2^(e - 15) with
    max|T| = f 2^e, f in [0.5, 1), so max|T| / scale lies in [2^14, 2^15); value = element * scale.
    bf16: element = round(T) to bfloat16, scale 1.  f32: T itself."""
    T = np.asarray(T, np.float32)
    if table_dtype == "f32":
        return T, 1.0
    if table_dtype == "bf16":
        return _bf16_round(T), 1.0
    if table_dtype != "f16":
        raise ValueError("table_dtype must be 'f32', 'f16' or 'bf16'")
    amax = float(np.abs(T).max()) if T.size else 0.0
    if not np.isfinite(amax):
        raise ValueError("node table holds a non-finite value")
    if amax > 0:
        _, e = np.frexp(np.float32(amax))
        scale = np.float32(np.ldexp(np.float32(1.0), int(e) - 15))
    else:
        scale = np.float32(1.0)
    h = (T * np.float32(1.0 / scale)).astype(np.float16)
    return (h.astype(np.float32) * scale).astype(np.float32), float(scale)


def store_grid(store):
    """(beta0, dbeta, delta0, ddelta) shared by every node; the device path needs one grid"""
    b0, d0 = np.asarray(store.beta[0], float), np.asarray(store.delta[0], float)
    for b, d in zip(store.beta, store.delta):
        if b.shape != b0.shape or d.shape != d0.shape or not (np.allclose(b, b0, rtol=0, atol=1e-12)
                                                               and np.allclose(d, d0, rtol=0, atol=1e-12)):
            raise ValueError("device 'b200' needs the same (beta, Delta) grids at every node")
    return float(b0[0]), float(b0[1] - b0[0]), float(d0[0]), float(d0[1] - d0[0])


def upload_store(store, ctx):
    """copy the store's tables into the context's HBM once (skipped if this store is already resident)"""
    token = (_lib.token_of(store), getattr(store, "table_dtype", "f32"))
    if ctx.store_token == token:
        return
    gen = getattr(store, "generator", None)
    shape = tuple(store.spec.shape) if gen is not None else tuple(np.asarray(store.tables[0]).shape)
    beta0, dbeta, delta0, ddelta = store_grid(store)
    dtype = TABLE_DTYPES[getattr(store, "table_dtype", "f32")]
    ctx.store_init(len(store.tables), shape, store.tau_idx, beta0, dbeta, delta0, ddelta, dtype)
    if gen is not None:
        for k, T in enumerate(store.tables):
            if T is None:
                M, P, Q, S, seed = gen
                ctx.store_generate_node(k, store.s[k], store.alpha_lo[k], store.alpha_hi[k], M, P, Q, S[k], seed)
            else:
                if tuple(np.asarray(T).shape) != shape:
                    raise ValueError("every node table must have the same shape")
                ctx.store_set_node(k, store.s[k], store.alpha_lo[k], store.alpha_hi[k], T)
    else:
        if any(tuple(np.shape(T)) != shape for T in store.tables):
            raise ValueError("every node table must have the same shape")
        files, offs = getattr(store, "files", None), getattr(store, "t_offsets", None)
        stream = bool(getattr(store, "mapped", False)) and files is not None and offs is not None
        paths = [f if (stream and o is not None) else None for f, o in zip(files, offs)] if stream else None
        hosts = [T if (paths is None or paths[k] is None) else None for k, T in enumerate(store.tables)]
        store.load_stats = ctx.store_load(0, store.s, store.alpha_lo, store.alpha_hi, paths=paths,
                                          offsets=offs if stream else None, hosts=hosts,
                                          readers=getattr(store, "readers", 6), direct=getattr(store, "direct", False))
    s_before = getattr(store, "shard_s_before", None)
    if s_before is not None:
        ctx.store_set_shard(s_before)
    ctx.store_token = token
    ctx.prep_token = None
