"""A CPU model of the BUILD_LOW triangle BLAS (test infrastructure).

Restates, in numpy/Python, what the device builder in
graphic_lab_task_b200/csrc/lbvh.cu computes for one triangle mesh, step by
step in the same float32 arithmetic: the bounds of the triangle box centres,
30-bit Morton codes, the stable radix sort, the binary radix tree of Karras
2012 over the sorted codes, the fitted boxes, and the host emitter's
depth-first layout (emit_pairs with the triangle leaf table of
lrt_add_geom_triangles3f, csrc/scene.cpp): node pairs, the leaf table
Pack(start, count) and the triangle order.  Only for small meshes (pure
Python tree walks).
"""
import numpy as np

LEAF = 0x80000000
ESC_ROOT = 0xFFFFFFFE


def triangle_boxes(v, t):
    """Per triangle {lo.xyz, hi.xyz} as float32 min/max of its vertices."""
    p = np.asarray(v, np.float32)[np.asarray(t).reshape(-1, 3)]
    return np.concatenate([p.min(1), p.max(1)], axis=1).astype(np.float32)


def _spread10(v):
    v = np.asarray(v, np.uint64)
    v = (v * 0x00010001) & 0xFF0000FF
    v = (v * 0x00000101) & 0x0F00F00F
    v = (v * 0x00000011) & 0xC30C30C3
    v = (v * 0x00000005) & 0x49249249
    return v.astype(np.uint32)


def morton_codes(boxes):
    c = (np.float32(0.5) * (boxes[:, :3] + boxes[:, 3:])).astype(np.float32)
    ok = ~np.isnan(c)
    lo = np.array([c[ok[:, k], k].min() for k in range(3)], np.float32)
    hi = np.array([c[ok[:, k], k].max() for k in range(3)], np.float32)
    ext = (hi - lo).astype(np.float32)
    q = np.zeros(c.shape, np.uint32)
    for k in range(3):
        u = ((c[:, k] - lo[k]) / ext[k]).astype(np.float32) if ext[k] > 0 else np.zeros(len(c), np.float32)
        s = np.clip(np.nan_to_num(u * np.float32(1024.0), nan=0.0), 0.0, 1023.0).astype(np.float32)
        q[:, k] = s.astype(np.uint32)
    return (_spread10(q[:, 0]) << 2) | (_spread10(q[:, 1]) << 1) | _spread10(q[:, 2])


def _clz(x):
    return 32 - int(x).bit_length()


def radix_tree(codes):
    """Inner nodes [first, last, kid0, kid1] over the sorted codes (kids with
    the top bit set are sorted positions)."""
    n = len(codes)
    codes = [int(c) for c in codes]

    def delta(i, j):
        if j < 0 or j >= n:
            return -1
        a, b = codes[i], codes[j]
        return _clz(a ^ b) if a != b else 32 + _clz(i ^ j)

    inner = []
    for i in range(n - 1):
        d = 1 if delta(i, i + 1) - delta(i, i - 1) >= 0 else -1
        dmin = delta(i, i - d)
        lmax = 2
        while delta(i, i + lmax * d) > dmin:
            lmax *= 2
        l, t = 0, lmax // 2
        while t >= 1:
            if delta(i, i + (l + t) * d) > dmin:
                l += t
            t //= 2
        j = i + l * d
        dnode = delta(i, j)
        s, div = 0, 2
        while True:
            t = (l + div - 1) // div
            if delta(i, i + (s + t) * d) > dnode:
                s += t
            if t <= 1:
                break
            div *= 2
        g = i + s * d + (-1 if d < 0 else 0)
        first, last = min(i, j), max(i, j)
        inner.append([first, last, (g | LEAF) if first == g else g, ((g + 1) | LEAF) if last == g + 1 else g + 1])
    return inner


def blas(v, t, max_leaf):
    """(pairs (P, 2, 8) float32 view of the layout, leaf table uint32, triangle order uint32)."""
    boxes = triangle_boxes(v, t)
    n = len(boxes)
    order = np.argsort(morton_codes(boxes), kind="stable")
    inner = radix_tree(morton_codes(boxes)[order])
    fitted = {}

    def box(kid):
        if kid & LEAF:
            return boxes[order[kid & ~LEAF]]
        if kid not in fitted:
            stack = [kid]
            while stack:  # post-order without recursion
                k = stack[-1]
                kids = [c for c in inner[k][2:] if not (c & LEAF) and c not in fitted]
                if kids:
                    stack.extend(kids)
                    continue
                stack.pop()
                a, b = box(inner[k][2]), box(inner[k][3])
                fitted[k] = np.concatenate([np.minimum(a[:3], b[:3]), np.maximum(a[3:], b[3:])])
        return fitted[kid]

    def count(kid):
        return 1 if kid & LEAF else inner[kid][1] - inner[kid][0] + 1

    def first(kid):
        return kid & ~LEAF if kid & LEAF else inner[kid][0]

    pairs, table, tri_order = [], [], []

    def leaf_word(kid):
        leaf_id = len(table)
        table.append(LEAF | ((count(kid) << 28) & 0x70000000) | (len(tri_order) & 0x0FFFFFFF))
        tri_order.extend(int(order[p]) for p in range(first(kid), first(kid) + count(kid)))
        return LEAF | (1 << 28) | leaf_id

    # emit_pairs: pair k on entering a node, its leaf children's words at once
    # (left, then right), then the left subtree, then the right one
    todo = [(0, ESC_ROOT, None)]
    while todo:
        node, parent_esc, fixup = todo.pop()
        k = len(pairs)
        if fixup is not None:
            pairs[fixup[0]][fixup[1]][1] = k
        kids = inner[node][2:]
        rec = []
        for c, kid in enumerate(kids):
            word = leaf_word(kid) if count(kid) <= max_leaf else 0
            rec.append([box(kid), word, 2 * k + 1 if c == 0 else parent_esc])
        pairs.append(rec)
        # the right subtree is visited after the whole left one: push it first
        if count(kids[1]) > max_leaf:
            todo.append((kids[1], parent_esc, (k, 1)))
        if count(kids[0]) > max_leaf:
            todo.append((kids[0], 2 * k + 1, (k, 0)))
    out = np.zeros((len(pairs), 2, 8), np.float32)
    for k, rec in enumerate(pairs):
        for c in range(2):
            b, word, esc = rec[c]
            out[k, c, :3], out[k, c, 4:7] = b[:3], b[3:]
            out[k, c, 3] = np.uint32(word).view(np.float32)
            out[k, c, 7] = np.uint32(esc).view(np.float32)
    assert n > max_leaf
    return out, np.array(table, np.uint32), np.array(tri_order, np.uint32)
