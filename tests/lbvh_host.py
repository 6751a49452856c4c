"""Test infrastructure: the device BVH builder's tree (open_rendering_framework_b200/csrc/pt_bvh_device.cu)
restated on the host in numpy / Python, so that traversal over an LBVH-shaped tree -- single-triangle
leaves with boxes that end exactly at shared vertices -- can be checked against brute force without a
GPU.  Same steps as the kernels: centroid bounds, 30-bit Morton codes, a stable sort, the Karras
hierarchy (equal codes ordered by position), bottom-up boxes and SAH leaf choice, child-pair nodes.
It restates the builder without treelet restructuring (option bvh_treelets = 0), whose trees keep the
Morton order of the leaves."""
import numpy as np

f32 = np.float32


def _spread10(x):
    x = x.astype(np.uint32) & 0x3FF
    x = (x | (x << 16)) & 0x030000FF
    x = (x | (x << 8)) & 0x0300F00F
    x = (x | (x << 4)) & 0x030C30C3
    x = (x | (x << 2)) & 0x09249249
    return x


def _clz(x):
    return 32 - int(x).bit_length()


def _as_int(u):
    return int(np.array([u & 0xFFFFFFFF], np.uint32).view(np.int32)[0])


def build(tp, trav_cost=1.2, max_leaf=8):
    """tp: [n, 9] float32 triangles.  Returns (nodes [n-1, 4, 4] float32 child-pair BVH2, v0, e1, e2
    [n, 4] float32 Moller-Trumbore records in leaf order)."""
    n = len(tp)
    P = tp.reshape(n, 3, 3).astype(f32)
    bl, bh = P.min(axis=1), P.max(axis=1)
    c = (f32(0.5) * (bl + bh)).astype(f32)
    lo, hi = c.min(axis=0), c.max(axis=0)
    ext = (hi - lo).astype(f32)
    inv = np.where(ext > 0, f32(1024.0) / np.where(ext > 0, ext, f32(1)), f32(0)).astype(f32)
    t = ((c - lo).astype(f32) * inv).astype(f32)
    q = np.where(t <= 0, 0, np.where(t >= 1023, 1023, t.astype(np.int64))).astype(np.uint32)
    keys = (_spread10(q[:, 0]) << 2) | (_spread10(q[:, 1]) << 1) | _spread10(q[:, 2])
    order = np.argsort(keys, kind="stable").astype(np.uint32)
    K = [int(k) for k in keys[order]]

    def delta(i, j):
        if j < 0 or j >= n:
            return -1
        return 32 + _clz(i ^ j) if K[i] == K[j] else _clz(K[i] ^ K[j])

    child = np.zeros((n - 1, 2), np.int64)
    rng = np.zeros((n - 1, 2), np.int64)
    ipar = np.full(n - 1, -1, np.int64)
    for i in range(n - 1):
        d = 1 if delta(i, i + 1) - delta(i, i - 1) >= 0 else -1
        dmin = delta(i, i - d)
        lmax = 2
        while delta(i, i + lmax * d) > dmin:
            lmax <<= 1
        l, s_ = 0, lmax >> 1
        while s_ >= 1:
            if delta(i, i + (l + s_) * d) > dmin:
                l += s_
            s_ >>= 1
        j = i + l * d
        dn = delta(i, j)
        s, st = 0, l
        while True:
            st = (st + 1) >> 1
            if delta(i, i + (s + st) * d) > dn:
                s += st
            if st <= 1:
                break
        g = i + s * d + min(d, 0)
        first, last = min(i, j), max(i, j)
        left = ~g if first == g else g
        right = ~(g + 1) if last == g + 1 else g + 1
        child[i] = (left, right)
        rng[i] = (first, last)
        for ch in (left, right):
            if ch >= 0:
                ipar[ch] = i
    leaf_lo, leaf_hi = bl[order], bh[order]
    nlo, nhi = np.zeros((n - 1, 3), f32), np.zeros((n - 1, 3), f32)
    ncost, ncnt = np.zeros(n - 1, f32), np.zeros(n - 1, f32)
    coll = np.zeros(n - 1, bool)

    def area(a, b):
        dx, dy, dz = (max(f32(0), f32(b[k] - a[k])) for k in range(3))
        return f32(f32(f32(dx * dy) + f32(dy * dz)) + f32(dz * dx))

    def rec(ch):
        return (leaf_lo[~ch], leaf_hi[~ch], f32(1), f32(1)) if ch < 0 else (nlo[ch], nhi[ch], ncost[ch], ncnt[ch])

    stack = [(0, False)]
    while stack:
        p, done = stack.pop()
        if not done:
            stack.append((p, True))
            stack.extend((int(ch), False) for ch in child[p] if ch >= 0)
            continue
        (al, ah, ac, an), (bl_, bh_, bc, bn) = rec(child[p][0]), rec(child[p][1])
        ml, mh = np.minimum(al, bl_), np.maximum(ah, bh_)
        cnt, A = f32(an + bn), area(ml, mh)
        wa = f32(area(al, ah) / A) if A > 0 else f32(0.5)
        wb = f32(area(bl_, bh_) / A) if A > 0 else f32(0.5)
        split = f32(f32(f32(trav_cost) + f32(wa * ac)) + f32(wb * bc))
        leaf = bool(cnt <= max_leaf and cnt <= split)
        nlo[p], nhi[p], ncost[p], ncnt[p], coll[p] = ml, mh, (cnt if leaf else split), cnt, leaf

    def code(ch):
        if ch < 0:
            return _as_int(0x80000000 | ((~ch) << 4) | 1)
        if coll[ch]:
            f, l = rng[ch]
            return _as_int(0x80000000 | (int(f) << 4) | int(l - f + 1))
        return int(ch)

    nodes = np.zeros((n - 1, 4, 4), f32)
    far = (np.full(3, 1e30, f32), np.full(3, 1e30, f32))
    for p in range(n - 1):
        if p == 0 and coll[0]:
            c0, c1, r0, r1 = _as_int(0x80000000 | n), _as_int(0x80000000), (nlo[0], nhi[0]), far
        else:
            c0, c1 = code(child[p][0]), code(child[p][1])
            r0, r1 = rec(child[p][0])[:2], rec(child[p][1])[:2]
        nodes[p, 0] = (r0[0][0], r0[1][0], r0[0][1], r0[1][1])
        nodes[p, 1] = (r1[0][0], r1[1][0], r1[0][1], r1[1][1])
        nodes[p, 2] = (r0[0][2], r0[1][2], r1[0][2], r1[1][2])
        nodes[p, 3] = np.array([c0, c1, ipar[p], 0], np.int32).view(f32)
    v0, e1, e2 = (np.zeros((n, 4), f32) for _ in range(3))
    Pp = P[order]
    v0[:, :3] = Pp[:, 0]
    v0[:, 3] = order.astype(np.int32).view(f32)
    e1[:, :3] = Pp[:, 1] - Pp[:, 0]
    e2[:, :3] = Pp[:, 2] - Pp[:, 0]
    return nodes, v0, e1, e2
