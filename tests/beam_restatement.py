"""Plain-Python restatement of the two-parents-per-hop search (beam=2), the batched
form beside the reference's GreedySearch.  Test infrastructure: the CPU test pins it to
the oracle's GreedySearch at beam 1; the GPU test compares the kernel with it at beam 2."""
import numpy as np


def beam_search(oracle, base, deg, adj, q, L, k, entry, beam):
    """GreedySearch with `beam` parents per hop.  Per hop: each parent's list in turn
    is checked against the bloom filter as it stood before that list, then marked;
    candidates below a full worklist's last distance are kept in list order, sorted
    by (distance, id) in batches of 64 and merged (older entries first on equal
    distance); the next parents are the first `beam` unvisited entries."""
    R = adj.shape[1]
    base64 = base.astype(np.int64)
    qi = q.astype(np.int64)
    bits = np.zeros(39988, bool)
    d0 = float(((base64[entry] - qi) ** 2).sum())
    wl = [[d0, 0, int(entry), True]]  # distance, insertion sequence, id, visited
    seq, parents = 1, [int(entry)]
    while True:
        cand = []
        for p in parents:
            row = [int(x) for x in adj[p, :min(int(deg[p]), R)]]
            passed = [x for x in row if not (bits[oracle.bf_h1(x)] and bits[oracle.bf_h2(x)])]
            for x in passed:
                bits[oracle.bf_h1(x)] = True
                bits[oracle.bf_h2(x)] = True
            cand += passed
        tail = wl[L - 1][0] if len(wl) == L else np.inf
        kept = []
        for c in cand:
            d = float(((base64[c] - qi) ** 2).sum())
            if d < tail:
                kept.append((d, c))
        for b0 in range(0, len(kept), 64):
            batch = sorted(kept[b0:b0 + 64])
            wl += [[d, seq + e, c, False] for e, (d, c) in enumerate(batch)]
            seq += len(batch)
            wl.sort(key=lambda x: (x[0], x[1]))
            del wl[L:]
        unv = [i for i, x in enumerate(wl) if not x[3]][:beam]
        if not unv:
            break
        parents = []
        for i in unv:
            wl[i][3] = True
            parents.append(wl[i][2])
    ids = np.full(k, 0xFFFFFFFF, np.uint32)
    ds = np.full(k, np.inf, np.float32)
    for t, x in enumerate(wl[:k]):
        ids[t], ds[t] = x[2], x[0]
    return ids, ds
