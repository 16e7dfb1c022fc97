"""The store loader's host side: load_redshift_store records, per node, the file and the byte offset of
its T.npy data (what exm_store_load reads), and upload_store streams a mapped store from its files and
sends a store read into memory from its host arrays."""

import os

import numpy as np
import pytest

import exmarg_b200 as eb
from exmarg_b200 import synth
from exmarg_b200.store import upload_store

SPEC = dict(ntau=3, nphif=49, nb=20, nd=13)
NODES = [5, 17, 30, 44]
SEED = 7


@pytest.fixture(scope="module")
def store_dir(tmp_path_factory):
    d = tmp_path_factory.mktemp("bd")
    spec = synth.TableSpec(**SPEC)
    s = synth.S_NODES_PROD[NODES]
    synth.write_store(str(d), spec, s, SEED)
    return str(d), spec, s


class FakeContext:
    """records what upload_store asks of the device context"""
    store_token = None
    prep_token = None

    def store_init(self, *args):
        self.init = args

    def store_load(self, first, s, alpha_lo, alpha_hi, paths=None, offsets=None, hosts=None, readers=6,
                   chunk_bytes=0, direct=False):
        self.load = dict(first=first, s=s, paths=paths, offsets=offsets, hosts=hosts, readers=readers, direct=direct)
        return {}


def test_offsets_point_at_the_tables(store_dir):
    d, spec, s = store_dir
    st = eb.load_redshift_store(d, mmap=True)
    assert np.array_equal(st.s, s)
    n = int(np.prod(spec.shape))
    for k, (f, off) in enumerate(zip(st.files, st.t_offsets)):
        assert off is not None
        raw = np.fromfile(f, np.float32, count=n, offset=off).reshape(spec.shape)
        assert np.array_equal(raw, synth.gen_table_node(spec, k, s, SEED))
        assert np.array_equal(raw, st.tables[k])


def test_upload_streams_a_mapped_store(store_dir):
    d, _, _ = store_dir
    st = eb.load_redshift_store(d, mmap=True, readers=3, direct=True)
    ctx = FakeContext()
    upload_store(st, ctx)
    assert ctx.load["paths"] == st.files and ctx.load["offsets"] == st.t_offsets
    assert all(h is None for h in ctx.load["hosts"])
    assert ctx.load["readers"] == 3 and ctx.load["direct"] is True and ctx.load["first"] == 0


def test_upload_sends_host_tables(store_dir):
    d, _, _ = store_dir
    st = eb.load_redshift_store(d)
    ctx = FakeContext()
    upload_store(st, ctx)
    assert ctx.load["paths"] is None
    assert all(h is T for h, T in zip(ctx.load["hosts"], st.tables))


def test_table_cli_orders_nodes_by_s(tmp_path):
    from exmarg_b200 import tables
    for s in (12.5, 0.004, 3.0):
        open(os.path.join(str(tmp_path), "sladder_n120_s%09.3f.meta.npz" % s), "w").close()
    open(os.path.join(str(tmp_path), "other.meta.npz"), "w").close()
    stems = tables.node_stems(str(tmp_path), "sladder_", ".meta.npz")
    assert [os.path.basename(t) for t in stems] == ["sladder_n120_s00000.004", "sladder_n120_s00003.000",
                                                   "sladder_n120_s00012.500"]


def test_fortran_ordered_table_goes_through_host_memory(tmp_path):
    """a T.npy member stored in Fortran order has no C-order byte range to stream: that node is sent from
    its host copy, the others from their files"""
    spec = synth.TableSpec(**SPEC)
    s = synth.S_NODES_PROD[NODES[:2]]
    synth.write_store(str(tmp_path), spec, s, SEED)
    T = synth.gen_table_node(spec, 1, s, SEED)
    f = sorted(str(p) for p in tmp_path.glob("bd_*.npz"))[1]
    with np.load(f) as z:
        members = {k: z[k] for k in z.files}
    members["T"] = np.asfortranarray(T)
    np.savez(f, **members)
    st = eb.load_redshift_store(str(tmp_path), mmap=True)
    assert st.t_offsets[0] is not None and st.t_offsets[1] is None
    assert np.array_equal(st.tables[1], T)
    ctx = FakeContext()
    upload_store(st, ctx)
    assert ctx.load["paths"] == [st.files[0], None]
    assert ctx.load["hosts"][0] is None and ctx.load["hosts"][1] is st.tables[1]


def test_compressed_store_is_refused(tmp_path):
    spec = synth.TableSpec(**SPEC)
    s = synth.S_NODES_PROD[NODES[:1]]
    T = synth.gen_table_node(spec, 0, s, SEED)
    np.savez_compressed(str(tmp_path / "bd_n120_s00001.000.npz"), T=T, beta=spec.beta, delta=spec.delta,
                        tau_idx=spec.tau_idx, alpha=synth.ALPHA, s_node=float(s[0]))
    with pytest.raises(ValueError, match="compressed"):
        eb.load_redshift_store(str(tmp_path))
