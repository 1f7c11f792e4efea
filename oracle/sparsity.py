"""Oracle (test infrastructure): pure-Python restatement of the reference's
structural sparsity detection and graph colorings, for small tapes.

Follows src/bytecode_tape/sparse.rs:463-776 (dependency sets per slot,
interaction pairs at nonlinear ops, sorted deduplicated lower triangle) and
src/sparse.rs:57-98, 292-413 (distance-2 coloring through G^2, intersection
graph coloring, largest-degree-first greedy coloring with a stable order).
Only tests import it, to check the engine library's implementation bit-exactly.
"""
from __future__ import annotations

UNUSED = 0xFFFFFFFF
INPUT, CONST = 0, 1
LINEAR = {2, 3, 12, 42}                       # Add, Sub, Neg, Fract
BINARY_NONLINEAR = {4, 5, 7, 8, 9, 43}        # Mul, Div, Powf, Atan2, Hypot, Custom
ZERO_DERIV = {36, 37, 38, 39, 40, 41, 10, 11, 6}  # Abs Signum Floor Ceil Round Trunc Max Min Rem
BINARY = {2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 43}


def hessian_pattern(op, a0, a1, ni):
    deps = []
    inter = set()
    k = 0
    for i, o in enumerate(op):
        o = int(o)
        if o == INPUT:
            deps.append({k})
            k += 1
            continue
        if o == CONST:
            deps.append(set())
            continue
        a, b = int(a0[i]), int(a1[i])
        if o in LINEAR or o in ZERO_DERIV:
            d = set(deps[a])
            if o in BINARY and b != UNUSED:
                d |= deps[b]
            deps.append(d)
        elif o in BINARY_NONLINEAR and o != 43:
            da, db = deps[a], deps[b]
            for u in da:
                for v in db:
                    inter.add((max(u, v), min(u, v)))
            if o != 4:
                for s in (da, db):
                    for u in s:
                        for v in s:
                            inter.add((max(u, v), min(u, v)))
            deps.append(da | db)
        else:  # unary nonlinear (and a unary custom op)
            d = set(deps[a])
            for u in d:
                for v in d:
                    inter.add((max(u, v), min(u, v)))
            deps.append(d)
    pairs = sorted(inter)
    return [p[0] for p in pairs], [p[1] for p in pairs]


def jacobian_pattern(op, a0, a1, ni, outs):
    deps = []
    k = 0
    for i, o in enumerate(op):
        o = int(o)
        if o == INPUT:
            deps.append({k})
            k += 1
        elif o == CONST:
            deps.append(set())
        else:
            d = set(deps[int(a0[i])])
            if o != 43 and o in BINARY and int(a1[i]) != UNUSED:
                d |= deps[int(a1[i])]
            deps.append(d)
    rows, cols = [], []
    for j, oi in enumerate(outs):
        for c in sorted(x for x in deps[int(oi)] if x < ni):
            rows.append(j)
            cols.append(c)
    return rows, cols


def _greedy(adj):
    n = len(adj)
    order = sorted(range(n), key=lambda v: -len(adj[v]))  # Python's sort is stable
    colors = [None] * n
    for v in order:
        used = {colors[u] for u in adj[v] if colors[u] is not None}
        c = 0
        while c in used:
            c += 1
        colors[v] = c
    return colors, (max(colors) + 1 if n else 0)


def greedy_coloring(dim, rows, cols):
    if dim == 0:
        return [], 0
    adj = [set() for _ in range(dim)]
    for r, c in zip(rows, cols):
        if r != c:
            adj[r].add(c)
            adj[c].add(r)
    adj2 = []
    for v in range(dim):
        s = set(adj[v])
        for u in adj[v]:
            s |= {w for w in adj[u] if w != v}
        adj2.append(sorted(s))
    return _greedy(adj2)


def _intersection(group_keys, color_keys, group_dim, color_dim):
    if color_dim == 0:
        return [], 0
    groups = [[] for _ in range(group_dim)]
    for g, c in zip(group_keys, color_keys):
        groups[g].append(c)
    adj = [set() for _ in range(color_dim)]
    for m in groups:
        for i in range(len(m)):
            for j in range(i + 1, len(m)):
                adj[m[i]].add(m[j])
                adj[m[j]].add(m[i])
    return _greedy([sorted(s) for s in adj])


def column_coloring(no, ni, rows, cols):
    return _intersection(rows, cols, no, ni)


def row_coloring(no, ni, rows, cols):
    return _intersection(cols, rows, ni, no)
