"""ORACLE - test infrastructure only.

Pure-Python restatement of the reference's CMG forest aggregation (vendored
cmg crate, rust/vendor/cmg/src/forest.rs), the checker for the library's
host-side hierarchy construction.  Small graphs only (loops are Python).

Restated functions:
  heavy_forest_serial / consider_parent  forest.rs:131-156, 320-334
  split_forest_with                      forest.rs:432-560
  low_effective_degree_correction        forest.rs:336-378
  component_labels (union-find)          forest.rs:562-607
"""

from __future__ import annotations


def heavy_forest(n, ptr, col, weight):
    parent = list(range(n))
    selected = [0.0] * n
    for v in range(n):
        for e in range(ptr[v], ptr[v + 1]):
            u, w = int(col[e]), float(weight[e])
            if w > selected[v] or (w == selected[v] and u < parent[v]):
                selected[v] = w
                parent[v] = u
    return parent, selected


def split_forest(parent):
    n = len(parent)
    forest = list(parent)
    ancestors = [0] * n
    indegree = [0] * n
    visited = [False] * n
    for t in forest:
        indegree[t] += 1
    for start in range(n):
        current = start
        cont = True
        while cont and indegree[current] == 0 and not visited[current]:
            cont = False
            in_path = 0
            walk = [current]
            fresh = [0]
            k = 0
            while k <= 5 or visited[current]:
                current = forest[current]
                if current == walk[k] or (k > 0 and current == walk[k - 1]):
                    break
                k += 1
                walk.append(current)
                in_path += 0 if visited[current] else 1
                fresh.append(in_path)
            if k > 5:
                middle = k // 2
                forest[walk[middle]] = walk[middle]
                nxt = walk[middle + 1]
                indegree[nxt] -= 1
                removed = ancestors[walk[middle]]
                for v in walk[middle + 1:k + 1]:
                    ancestors[v] -= removed
                for i in range(middle + 1):
                    visited[walk[i]] = True
                    ancestors[walk[i]] += fresh[i]
                current = nxt
                cont = True
            if not cont:
                for i in range(k + 1):
                    ancestors[walk[i]] += fresh[i]
                    visited[walk[i]] = True
    for start in range(n):
        current = start
        while True:
            if indegree[current] != 0:
                break
            previous = current
            restart = False
            while True:
                nxt = forest[current]
                if nxt == current or nxt == previous:
                    break
                if ancestors[current] > 2 and ancestors[nxt] - ancestors[current] > 2:
                    forest[current] = current
                    indegree[nxt] -= 1
                    removed = ancestors[current]
                    ap, ac = current, nxt
                    while True:
                        ancestors[ac] -= removed
                        an = forest[ac]
                        if an == ac or an == ap:
                            break
                        ap, ac = ac, an
                    current = nxt
                    restart = True
                    break
                previous = current
                current = nxt
            if not restart:
                break
    return forest


def aggregate(n, ptr, col, weight, threshold=0.125):
    """Labels (first-occurrence numbering) and the aggregate count."""
    diag = [0.0] * n
    for v in range(n):
        for e in range(ptr[v], ptr[v + 1]):
            diag[v] += float(weight[e])
    parent, selected = heavy_forest(n, ptr, col, weight)
    split = split_forest(parent)
    if any(d > 0 and s / d < threshold for d, s in zip(diag, selected)):
        incident = [0.0] * n
        for v, t in enumerate(split):
            if t != v:
                incident[v] += selected[v]
                incident[t] += selected[v]
        for v in range(n):
            if diag[v] > 0 and incident[v] / diag[v] < threshold:
                split[v] = v
    dsu = list(range(n))

    def root(v):
        while dsu[v] != v:
            dsu[v] = dsu[dsu[v]]
            v = dsu[v]
        return v

    for v, t in enumerate(split):
        a, b = root(v), root(t)
        if a != b:
            if a < b:
                dsu[b] = a
            else:
                dsu[a] = b
    labels, first = [0] * n, {}
    for v in range(n):
        r = root(v)
        if r not in first:
            first[r] = len(first)
        labels[v] = first[r]
    return labels, len(first)
