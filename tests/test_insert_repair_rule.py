"""The rule the insertion row repair (k_row_repair_ins) is built on, checked
on the CPU against the oracle: after inserting edges, row k can only rise,
and every vertex that rises lies in the region grown from the seeds --
endpoints of inserted edges inside C_k and the vertices that joined C_k --
along edges (either direction) to members w with
    old_k(w) < bound(x)  for a region vertex x next to it, and
    old_k(w) < new row_{k-1}(w)  (w can rise at all),
each starting at its bound new row_{k-1}; refining the region down to the
greatest fixpoint, with every vertex outside it fixed at its old value,
gives the new row.  Rows are repaired in order k = 1..R.  This is a model of
the kernel's algorithm in Python on small graphs (the kernel itself is
tested on the GPU against the oracle in test_maint_gpu.py)."""
import numpy as np
import pytest


def _lists(V, a, b):
    o = np.argsort(a, kind="stable")
    off = np.zeros(V + 1, np.int64)
    np.add.at(off, a.astype(np.int64) + 1, 1)
    return np.cumsum(off), b[o].astype(np.int64)


def _repair_rows(V, s2, d2, iu, iv, okx, orows, nkx, row0_new):
    """New rows 1..kmax by the region rule (graph s2 -> d2 after inserting
    iu -> iv); returns (rows, largest region)."""
    oo, on = _lists(V, s2, d2)
    io, inn = _lists(V, d2, s2)
    K = int(nkx.max())
    prev = row0_new.copy()
    out = [row0_new.copy()]
    biggest = 0
    for k in range(1, K + 1):
        mem = nkx >= k
        old = np.where(okx >= k, orows[k] if k < len(orows) else 0, -1)
        t = {}
        work = []

        def add(w, bound):
            if w not in t and bound > old[w]:
                t[w] = bound
                work.append(w)

        for a, b in zip(iu, iv):
            if mem[a] and mem[b]:
                add(int(a), int(prev[a]))
                add(int(b), int(prev[b]))
        for v in np.nonzero((okx < k) & (nkx >= k))[0]:
            add(int(v), int(prev[v]))
        qi = 0
        while qi < len(work):  # grow the region
            x = work[qi]
            qi += 1
            for lst, off in ((on, oo), (inn, io)):
                for w in lst[off[x]:off[x + 1]]:
                    w = int(w)
                    if mem[w] and w not in t and old[w] < t[x] and prev[w] > old[w]:
                        add(w, int(prev[w]))
        biggest = max(biggest, len(t))

        def val(x):
            return t[x] if x in t else old[x]

        todo = list(t)
        while todo:  # refine down to the greatest fixpoint
            x = todo.pop()
            outs = [int(w) for w in on[oo[x]:oo[x + 1]] if mem[w]]
            ins = [int(w) for w in inn[io[x]:io[x + 1]] if mem[w]]
            vo = np.array([val(w) for w in outs], np.int64)
            vi = np.array([val(w) for w in ins], np.int64)
            nv = 0
            for L in range(t[x], -1, -1):
                if (vo >= L).sum() >= L and (vi >= L).sum() >= k:
                    nv = L
                    break
            if nv < t[x]:
                cap = t[x]
                t[x] = nv
                todo += [w for w in outs + ins if w in t and nv < t[w] <= cap and w not in todo]
        row = np.where(mem, np.maximum(old, 0), 0)
        for x, v in t.items():
            row[x] = v
        out.append(row)
        prev = row
    return np.stack(out), biggest


@pytest.mark.parametrize("scale,ef,seed,batch", [(9, 8, 1, 1), (10, 8, 2, 5), (10, 16, 3, 20), (11, 8, 4, 60)])
def test_region_rule_gives_the_new_rows(orc, scale, ef, seed, batch):
    V, s, d = orc.gen_rmat(scale, ef, seed)
    okm, olm, okx, orows = orc.dcore(V, s, d)
    present = set(zip(s.tolist(), d.tolist()))
    rng = np.random.default_rng(seed)
    top = np.argsort(-okx, kind="stable")[:64]
    iu, iv = [], []
    while len(iu) < batch:
        # half the edges between high-kmax vertices, half anywhere
        pool = top if len(iu) % 2 else np.arange(V)
        a, b = (int(x) for x in rng.choice(pool, 2, replace=False))
        if (a, b) not in present:
            present.add((a, b))
            iu.append(a)
            iv.append(b)
    s2 = np.concatenate([s, np.array(iu, np.uint32)])
    d2 = np.concatenate([d, np.array(iv, np.uint32)])
    nkm, nlm, nkx, nrows = orc.dcore(V, s2, d2)
    rows, biggest = _repair_rows(V, s2, d2, iu, iv, okx, orows, nkx, nrows[0])
    assert np.array_equal(rows, nrows)
    assert biggest < V  # the region is a part of the graph
