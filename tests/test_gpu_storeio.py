"""exm_store_load on the device: node tables streamed from bd_*.npz files (buffered and O_DIRECT
reads, chunks that split the rows' byte ranges at many places), from host arrays, and from a mix of
the two, land bit for bit as the file holds them; 16-bit stores quantize each node as the host
restatement does; bad inputs are refused before any transfer."""

import os
import shutil

import numpy as np
import pytest

import exmarg_b200 as eb
from exmarg_b200 import _lib, synth
from exmarg_b200.store import TABLE_DTYPES, upload_store

pytestmark = pytest.mark.gpu

SPEC = dict(ntau=3, nphif=49, nb=20, nd=13)     # 52-byte rows: no chunk boundary falls on 4 KiB
NODES = [5, 17, 30, 44]
SEED = 7


@pytest.fixture(scope="module")
def store_dir(tmp_path_factory):
    d = tmp_path_factory.mktemp("bd")
    spec = synth.TableSpec(**SPEC)
    s = synth.S_NODES_PROD[NODES]
    synth.write_store(str(d), spec, s, SEED)
    host = [synth.gen_table_node(spec, k, s, SEED) for k in range(len(s))]
    return str(d), spec, s, host


def _init(ctx, st, spec, dtype="f32"):
    ctx.store_init(len(st.s), spec.shape, spec.tau_idx, spec.beta[0], spec.beta[1] - spec.beta[0], spec.delta[0],
                   spec.delta[1] - spec.delta[0], TABLE_DTYPES[dtype])


@pytest.mark.parametrize("direct", [False, True])
@pytest.mark.parametrize("chunk", [0, 1000, 52 * 2940 - 52])
def test_files_bit_exact(store_dir, direct, chunk):
    d, spec, s, host = store_dir
    st = eb.load_redshift_store(d, mmap=True)
    ctx = _lib.Context(0)
    try:
        _init(ctx, st, spec)
        stats = ctx.store_load(0, st.s, st.alpha_lo, st.alpha_hi, paths=st.files, offsets=st.t_offsets, readers=3,
                               chunk_bytes=chunk, direct=direct)
        for k in range(len(s)):
            assert np.array_equal(ctx.store_get_node(k, spec.shape), host[k])
        assert stats["file_bytes"] == len(s) * host[0].nbytes and stats["host_bytes"] == 0
    finally:
        ctx.close()


def test_host_and_file_sources_mixed(store_dir):
    d, spec, s, host = store_dir
    st = eb.load_redshift_store(d, mmap=True)
    ctx = _lib.Context(0)
    try:
        _init(ctx, st, spec)
        paths = [st.files[0], None, st.files[2], None]
        hosts = [None, host[1], None, host[3]]
        stats = ctx.store_load(0, st.s, st.alpha_lo, st.alpha_hi, paths=paths, offsets=st.t_offsets, hosts=hosts,
                               readers=2, chunk_bytes=4096)
        for k in range(len(s)):
            assert np.array_equal(ctx.store_get_node(k, spec.shape), host[k])
        assert stats["file_bytes"] == stats["host_bytes"] == 2 * host[0].nbytes
    finally:
        ctx.close()


@pytest.mark.parametrize("mmap", [True, False])
@pytest.mark.parametrize("dt", ["f16", "bf16"])
def test_upload_16bit(store_dir, mmap, dt):
    d, spec, s, host = store_dir
    st = eb.load_redshift_store(d, mmap=mmap, readers=4, table_dtype=dt)
    ctx = _lib.Context(0)
    try:
        upload_store(st, ctx)
        assert (st.load_stats["file_bytes"] > 0) == mmap
        for k in range(len(s)):
            assert np.array_equal(ctx.store_get_node(k, spec.shape), eb.quantize_table(host[k], dt)[0])
    finally:
        ctx.close()


def test_pe_intrinsic_same_on_streamed_store(tmp_path):
    """the golden config1 store written as bd_*.npz and streamed back gives the in-memory store's results"""
    from tests.golden_io import Fixture
    fx = Fixture("config1")
    for k, T in enumerate(fx.store.tables):
        np.savez(os.path.join(str(tmp_path), "bd_n120_s%09.3f.npz" % fx.s_nodes[k]), T=T, beta=fx.spec.beta,
                 delta=fx.spec.delta, tau_idx=fx.spec.tau_idx, alpha=synth.ALPHA, s_node=float(fx.s_nodes[k]))
    st = eb.load_redshift_store(str(tmp_path), mmap=True, readers=3)
    kw = dict(prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud, n_random=fx.n_random)
    a = eb.pe_intrinsic(fx.seg, fx.b200_bank(), st, **kw)
    b = eb.pe_intrinsic(fx.seg, fx.b200_bank(), fx.store, **kw)
    assert st.load_stats["file_bytes"] == sum(T.nbytes for T in fx.store.tables)
    assert np.array_equal(a["ln_b"], b["ln_b"]) and np.array_equal(a["ln_lambda"], b["ln_lambda"])


def test_refuses_bad_input(store_dir, tmp_path):
    d, spec, s, host = store_dir
    st = eb.load_redshift_store(d, mmap=True)
    short = os.path.join(str(tmp_path), "short.npz")
    with open(st.files[1], "rb") as fh:
        data = fh.read()
    with open(short, "wb") as fh:
        fh.write(data[: st.t_offsets[1] + host[1].nbytes - 100])
    ctx = _lib.Context(0)
    try:
        _init(ctx, st, spec)
        paths = list(st.files)
        paths[1] = short
        with pytest.raises(ValueError, match="ends before its table"):
            ctx.store_load(0, st.s, st.alpha_lo, st.alpha_hi, paths=paths, offsets=st.t_offsets)
        with pytest.raises(ValueError, match="ascending"):
            ctx.store_load(0, st.s[::-1], st.alpha_lo, st.alpha_hi, paths=st.files, offsets=st.t_offsets)
        with pytest.raises(ValueError, match="cannot open"):
            ctx.store_load(0, st.s, st.alpha_lo, st.alpha_hi, paths=[p + ".missing" for p in st.files],
                           offsets=st.t_offsets)
        ctx.store_load(0, st.s, st.alpha_lo, st.alpha_hi, paths=st.files, offsets=st.t_offsets)   # still usable
        assert np.array_equal(ctx.store_get_node(3, spec.shape), host[3])
    finally:
        ctx.close()
    shutil.rmtree(str(tmp_path), ignore_errors=True)
