"""exmarg_b200 -- exmarg's Eq. (C7) analysis path on the NVIDIA B200 (sm_100a).

A drop-in for exmarg.search with device='b200' beside the reference's 'cpu' and 'gpu':

    store = load_redshift_store(store_dir)              # every node table (resident in HBM on first use)
    bank = mass_bank(bank_rows, segments, 'b200')       # templates W, powers u
    res = pe_intrinsic(segments, bank, store, prior)    # M, q, chi, u, ln_lambda, ln_b, rows

The numerics live in libexmarg_b200.so (C ABI: include/exmarg_b200.h), called through
ctypes; there is no CPU fallback on the 'b200' path.
"""

from .segments import D0, read_segments
from .bank import MassBank, mass_bank, from_bank, array_module
from .store import RedshiftStore, load_redshift_store, quantize_table, upload_store, with_table_dtype
from .pe import pe_intrinsic, pe_redshift, distance_weights, prepare, autotune
from .shard import pe_intrinsic_sharded, node_ranges, shard_of
from ._lib import Context, context

__all__ = ["D0", "read_segments", "MassBank", "mass_bank", "from_bank", "array_module", "RedshiftStore",
           "load_redshift_store", "upload_store", "quantize_table", "with_table_dtype", "pe_intrinsic", "pe_redshift", "pe_intrinsic_sharded", "node_ranges", "shard_of", "distance_weights", "prepare", "autotune", "Context",
           "context"]
