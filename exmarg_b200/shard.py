"""Node sharding: one store's nodes split across GPUs, one process per GPU.

pe_intrinsic's node values -- ln Lambda of every template at every store node (exmarg/search/pe.py:168-200)
-- need only that node's table, so the nodes split into contiguous ranges, one per rank, balanced by the
gather work each range covers (its (node, template) pairs and a cost per node).  A rank keeps only its range's tables in HBM (a store of 53
production nodes is 39.6 GB; a shard of it is 39.6/N) and computes its rows on the device: its context's
store is declared a shard (exm_store_set_shard, the s of the node below the range), so the boundary point
of the range's first node is set as the whole store sets it.  Every (node, template) value then comes from
exactly one rank and is -inf on the others, and one all-reduce with MAX over the process group gives every
rank the whole store's rows.  The node log-sum-exp with the whole store's distance-prior weights
(pe.py:321-336) and ln B (pe.py:338-344, :135-142) follow on the host in float64.

Each rank runs the matched filter and the time selection of every segment itself (they are per segment,
not per node); only the taps and the gather divide.  The exchange is n_segment x (n_node + 1) x n_template
float64 per call: 0.9 MB a segment at 53 nodes and 2048 templates.
"""

import copy

import numpy as np

from .pe import distance_weights, prepare
from .segments import read_segments


def node_geometry(s, alpha_lo, alpha_hi, u, ymin):
    """valid (n_node, n_template), y (n_node + 1, n_template; row n_node the boundary point) and the
    boundary node of each template (-1: none), exmarg/search/pe.py:58-84 on the whole store (host, float64)"""
    s, u = np.asarray(s, float), np.asarray(u, float)
    nn, nm = s.size, u.size
    valid = np.zeros((nn, nm), bool)
    y = np.zeros((nn + 1, nm))
    bnode = np.full(nm, -1)
    for k in range(nn):
        alo = min(alpha_lo[k], ymin * ymin)
        a = s[k] / u
        o = (np.sqrt(a) >= ymin) & (a > alo) & (a < alpha_hi[k])
        valid[k] = o
        y[k] = np.where(o, np.sqrt(a), 0.0)
        s_prev = s[k - 1] if k > 0 else 0.0
        low = o & (s_prev / u <= alo)
        bnode[low] = k
        y[nn][low] = np.sqrt(float(alo) * (1.0 + 1e-9))
    return valid, y, bnode


# the gather's cost of a node beside that of its (node, template) pairs, in pairs: staging a node's windows
# for every lag costs about as much as 3500 pairs (fit on a B200 at 2048 walked times, 87 lags: 1.43 ms a node,
# 0.40 us a pair)
NODE_WEIGHT = 3500.0


def node_ranges(store, u, ymin, n_shards, node_weight=NODE_WEIGHT):
    """n_shards contiguous node ranges [k0, k1), none empty, with about equal gather work each: the
    (node, template) pairs (a template's boundary point counts at its boundary node) plus node_weight a node"""
    nn = len(store.s)
    if not 1 <= int(n_shards) <= nn:
        raise ValueError("need 1 <= shards <= %d (the store's nodes)" % nn)
    valid, _, bnode = node_geometry(store.s, store.alpha_lo, store.alpha_hi, u, ymin)
    work = valid.sum(axis=1) + np.bincount(bnode[bnode >= 0], minlength=nn)[:nn] + float(node_weight)
    cum = np.concatenate([[0.0], np.cumsum(work)])
    cuts = [0]
    for i in range(1, int(n_shards)):
        k = int(np.searchsorted(cum, cum[-1] * i / n_shards))
        cuts.append(min(max(k, cuts[-1] + 1), nn - (int(n_shards) - i)))
    cuts.append(nn)
    return [(cuts[i], cuts[i + 1]) for i in range(int(n_shards))]


def shard_of(store, k0, k1):
    """the nodes k0..k1-1 of a store as a store of their own (host tables or files shared), declared a
    shard on upload; stores whose tables the device generates cannot be sharded"""
    nn = len(store.s)
    if not 0 <= k0 < k1 <= nn:
        raise ValueError("node range [%d, %d) outside the store's %d nodes" % (k0, k1, nn))
    if getattr(store, "generator", None) is not None:
        raise ValueError("a store generated on the device cannot be sharded: give it host tables or files")
    cache = store.__dict__.setdefault("_shards", {})
    key = (int(k0), int(k1), getattr(store, "table_dtype", "f32"))
    if key in cache:
        return cache[key]
    sub = copy.copy(store)
    sub.__dict__.pop("_b200_token", None)
    sub.__dict__.pop("_shards", None)
    for name in ("s", "alpha_lo", "alpha_hi"):
        setattr(sub, name, np.asarray(getattr(store, name))[k0:k1])
    for name in ("beta", "delta", "tables", "files", "t_offsets"):
        v = getattr(store, name, None)
        if v is not None:
            setattr(sub, name, list(v)[k0:k1])
    if hasattr(sub, "device_tokens"):
        sub.device_tokens = {}
    sub.shard_s_before = float(store.s[k0 - 1]) if k0 > 0 else 0.0
    sub.shard_range = (int(k0), int(k1))
    cache[key] = sub
    return sub


def node_weights(store, u, ymin, prior):
    """ln of the distance-prior weights (n_node + 1, n_template) of the whole store, pe.py:321-327"""
    _, y, _ = node_geometry(store.s, store.alpha_lo, store.alpha_hi, u, ymin)
    lnW = np.full(y.shape, -np.inf)
    for m in range(y.shape[1]):
        pts = np.nonzero(y[:, m] > 0)[0]
        if pts.size < 2:
            raise ValueError("template %d (u %.3f) reaches fewer than two store nodes" % (m, u[m]))
        order = pts[np.argsort(y[pts, m])]
        lnW[order, m] = distance_weights(y[order, m], prior, ymin)
    return lnW


def cell_weights(M, q, chi):
    """normalized grid-cell weights of the templates, pe.py:338-343"""
    cell = np.ones(np.size(M))
    for ax in (np.asarray(M, float), np.asarray(q, float), np.asarray(chi, float)):
        vals = np.unique(ax)
        if vals.size > 1:
            cell *= np.gradient(vals)[np.searchsorted(vals, ax)]
    return cell / cell.sum()


def log_mean(lam, w):
    """ln sum_i w_i exp(lam_i), -inf values allowed (pe.py:135-142)"""
    fin = np.isfinite(lam) & (w > 0)
    if not fin.any():
        return -np.inf
    mx = lam[fin].max()
    return float(mx + np.log(np.sum(w[fin] * np.exp(lam[fin] - mx))))


def _group_info(group):
    try:
        import torch.distributed as dist
    except ImportError:
        return None, 0, 1
    if not dist.is_available() or not dist.is_initialized():
        return None, 0, 1
    return dist, dist.get_rank(group), dist.get_world_size(group)


def exchange(lamN, group=None, device=None):
    """every rank's node values combined (elementwise max) on every rank of the process group"""
    dist, _, world = _group_info(group)
    if world == 1:
        return lamN
    import torch
    t = torch.from_numpy(np.ascontiguousarray(lamN))
    if dist.get_backend(group) == "nccl":
        t = t.to("cuda" if device is None else "cuda:%d" % device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return t.cpu().numpy()


def _device_node_values(seg, bank, store, k0, k1, prior, ymin, n_loud, n_random, seed):
    sub = shard_of(store, k0, k1)
    ctx = prepare(bank, sub, prior, ymin)
    out = np.empty((seg["rows"].size, k1 - k0 + 1, bank.u.size))
    for e, row in enumerate(seg["rows"]):
        ctx.filter(seg["d_H"][e:e + 1], seg["d_L"][e:e + 1], seg["sig2_H"], seg["sig2_L"], want=False)
        if n_loud > 0:
            ctx.select_times(seed + int(row), n_loud, n_random, want=False)
        else:
            ctx.set_times(None)
        out[e] = ctx.node_values(k1 - k0)
    return out


def pe_intrinsic_sharded(segments, bank, store, rows=None, prior="volume", ymin=0.1267, n_loud=1024,
                         n_random=1024, seed=0, group=None, ranges=None, node_values=None):
    """pe_intrinsic with the store's nodes split over the ranks of a torch.distributed process group
    (one GPU each; without an initialized group, one rank holding every node).  Every rank returns the
    whole result: dict M, q, chi, u, ln_lambda (n_segment, n_template), ln_b (n_segment,), rows, and
    node_ranges (the [k0, k1) of each rank).

    ranges: the node range of each rank (default node_ranges); node_values(seg, k0, k1) -> (n_segment,
    k1 - k0 + 1, n_template) replaces the device computation of a rank's rows (row k1 - k0: the boundary
    points whose node lies in the range)."""
    dist, rank, world = _group_info(group)
    u = np.asarray(bank.u, float)
    ranges = list(ranges) if ranges is not None else node_ranges(store, u, ymin, world)
    if len(ranges) != world:
        raise ValueError("one node range per rank")
    nn = len(store.s)
    seg = read_segments(segments, rows)
    lnW = node_weights(store, u, ymin, prior)
    k0, k1 = ranges[rank]
    if node_values is None:
        part = _device_node_values(seg, bank, store, k0, k1, prior, ymin, n_loud, n_random, seed)
    else:
        part = np.asarray(node_values(seg, k0, k1), float)
    lamN = place(part, k0, k1, nn)
    lamN = exchange(lamN, group, getattr(bank, "device_index", None))
    ln_lambda, ln_b = combine(lamN, lnW, bank.M, bank.q, bank.chi)
    return dict(M=bank.M, q=bank.q, chi=bank.chi, u=bank.u, ln_lambda=ln_lambda, ln_b=ln_b, rows=seg["rows"],
                node_ranges=ranges)


def place(part, k0, k1, nn):
    """a rank's rows (n_segment, k1 - k0 + 1, n_template) in the whole store's (n_segment, nn + 1,
    n_template), -inf at the other nodes"""
    lamN = np.full((part.shape[0], nn + 1, part.shape[2]), -np.inf)
    lamN[:, k0:k1] = part[:, :k1 - k0]
    lamN[:, nn] = part[:, k1 - k0]
    return lamN


def combine(lamN, lnW, M, q, chi):
    """ln Lambda (n_segment, n_template): the log-sum-exp over nodes of lnW + lamN (pe.py:331-336),
    and ln B (n_segment,) with the grid-cell weights"""
    v = lnW[None] + lamN
    mx = v.max(axis=1)
    fin = np.isfinite(mx)
    with np.errstate(invalid="ignore", divide="ignore"):
        ln_lambda = np.where(fin, mx + np.log(np.exp(v - np.where(fin, mx, 0.0)[:, None]).sum(axis=1)), -np.inf)
    w = cell_weights(M, q, chi)
    return ln_lambda, np.array([log_mean(L, w) for L in ln_lambda])
