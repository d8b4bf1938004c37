"""Host-side checks of two arguments the pair kernels' traversal rests on
(csrc/traverse.cuh, csrc/pair.cu), restated in numpy:

* the box prune: a staged atom is dropped when the FP32 distance² from its
  FP32 coordinates to the bounding box of the home atoms' FP32 coordinates is
  not below c²·(1 + 2⁻¹⁰).  No atom within the exact FP64 cutoff of a home
  atom may be dropped — checked on random home sets with candidates placed at
  c·(1 ± 1e-7 … 1e-3) from a home atom, the hardest cases;
* the flat drain: the lanes' lists (or a pass's per-home masks) form one owner-major sequence, lane l
  takes entries [l·R, (l+1)·R) with R = ceil(total/32), stores the partial of
  owner h in slot l + h, and owner h adds the slots of lanes off_h/R …
  (off_h + cnt_h − 1)/R.  Slots must be unique, and each owner must collect
  exactly its own entries — checked on random count vectors, zero counts
  included;
* the half-stencil pass walks each lane's share directly on the per-home
  candidate masks: every entry taken once, in home-major order, in range;
* the ACE site kernel's balanced adjoint sums every term once, in order;
* the snapshot fill compacts each lane's in-range candidates in place and
  writes the lanes' entries with the whole warp: every entry of every centre
  lands once, in visit order, inside the centre's CSR range;
* on minimum-image grids with the per-cell wrap (at least 4 bins of width
  >= c per periodic axis) the stencil entry's shift s equals the reference's
  image -rint((x_j - x_i)/L) for every in-range pair.
"""
import numpy as np

GUARD = np.float32(1.0 + 1.0 / 1024.0)


def box_keep(cand32, lo32, hi32, c2hi):
    """The kernel's FP32 box test: fmaf(ex, ex, fmaf(ey, ey, ez * ez)) < c2hi."""
    e = np.maximum(np.maximum(lo32 - cand32, cand32 - hi32), np.float32(0.0)).astype(np.float32)
    ez2 = (e[..., 2] * e[..., 2]).astype(np.float32)
    # fmaf: exact product and sum in float64, one rounding to float32
    t = (e[..., 1].astype(np.float64) * e[..., 1] + ez2).astype(np.float32)
    d2 = (e[..., 0].astype(np.float64) * e[..., 0] + t).astype(np.float32)
    return d2 < c2hi


def test_box_prune_never_drops_a_neighbour():
    rng = np.random.default_rng(20)
    for c in (2.0, 5.5, 8.5):
        c2 = c * c
        c2hi = np.float32(np.float32(c2) * GUARD)
        for trial in range(200):
            L = rng.uniform(0.5, 1.5) * c
            base = rng.uniform(-300.0, 300.0, 3)  # absolute coordinates far from 0
            home = base + rng.uniform(0.0, L, (rng.integers(1, 33), 3))
            ref = home[0]
            rel32 = (home - ref).astype(np.float32)
            lo32, hi32 = rel32.min(axis=0), rel32.max(axis=0)
            # candidates just inside the cutoff of a random home atom, in random directions
            k = rng.integers(0, len(home), 256)
            u = rng.normal(size=(256, 3))
            u /= np.linalg.norm(u, axis=1)[:, None]
            r = c * (1.0 - 10.0 ** rng.uniform(-7, -3, 256))
            cand = home[k] + u * r[:, None]
            d = cand - home[k]
            exact = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
            inside = exact < c2
            cand32 = (cand - ref).astype(np.float32)
            keep = box_keep(cand32, lo32, hi32, c2hi)
            assert np.all(keep[inside]), (c, trial)


def flat_partition(cnt, W=32):
    cnt = np.asarray(cnt)
    off = np.concatenate([[0], np.cumsum(cnt)])
    total = int(off[-1])
    R = (total + W - 1) // W
    slots = {}
    for lane in range(W):
        q0, q1 = lane * R, min(lane * R + R, total)
        for q in range(q0, q1):
            h = int(np.searchsorted(off[:W], q, side="right") - 1)  # last owner with off <= q
            assert off[h] <= q < off[h + 1]
            key = lane + h
            if key in slots:
                assert slots[key][0] == lane and slots[key][1] == h  # the same segment continues
                slots[key][2].append(q)
            else:
                slots[key] = [lane, h, [q]]
    # each owner's partials: lanes off_h / R .. (off_h + cnt_h - 1) / R
    for h in range(W):
        if cnt[h] == 0:
            continue
        la, lb = off[h] // R, (off[h] + cnt[h] - 1) // R
        got = []
        for lane in range(la, lb + 1):
            seg = slots[lane + h]
            assert seg[0] == lane and seg[1] == h
            got += seg[2]
        assert got == list(range(off[h], off[h + 1]))
    assert max(slots) <= 62 if slots else True


def test_flat_drain_slots_are_unique_and_complete():
    rng = np.random.default_rng(5)
    flat_partition([0] * 32)
    flat_partition([1] + [0] * 31)
    flat_partition([0] * 31 + [72])
    flat_partition([72] * 32)
    for _ in range(300):
        nh = int(rng.integers(1, 33))
        cnt = np.zeros(32, int)
        cnt[:nh] = rng.integers(0, 73, nh) * (rng.random(nh) > 0.2)
        flat_partition(cnt)


def popc(x):
    return bin(int(x)).count("1")


def mask_walk(mh, n):
    """The half-stencil pass's share walk (csrc/pair_half.cu), restated: home
    h's entries are the set bits of mh[0][h], mh[1][h], ... (candidate 32w +
    bit), listed home-major; lane l takes entries [l·R, l·R + R) with R =
    ceil(total/32) and walks them on the masks without a list.  Every entry
    must be taken exactly once, by the lane whose share holds its position,
    with t < n and h < 32."""
    W = len(mh)
    cnt = [sum(popc(mh[w][h]) for w in range(W)) for h in range(32)]
    off = np.concatenate([[0], np.cumsum(cnt)]).astype(int)
    total = int(off[32])
    R = (total + 31) // 32
    want = [(h, 32 * w + b) for h in range(32) for w in range(W) for b in range(32) if (mh[w][h] >> b) & 1]
    assert len(want) == total
    got = []
    for lane in range(32):
        q = lane * R
        nmine = max(0, min(q + R, total) - q)
        if nmine == 0:
            continue
        h = 0
        for stp in (16, 8, 4, 2, 1):
            if h + stp <= 32 and off[h + stp] <= q:
                h += stp
        h = min(h, 31)
        r = q - off[h]
        w = 0
        m = mh[0][h]
        while r >= popc(m) and w + 1 < W:
            r -= popc(m)
            w += 1
            m = mh[w][h]
        for _ in range(r):
            m &= m - 1
        left = nmine
        for _ in range(nmine):
            assert m != 0 and h < 32
            t = 32 * w + ((m & -m).bit_length() - 1)
            assert t < n
            got.append((h, t))
            m &= m - 1
            left -= 1
            if left > 0:
                while m == 0:
                    w += 1
                    if w == W:
                        w = 0
                        h += 1
                        if h == 32:
                            break
                    m = mh[w][h]
        assert got[-nmine:] == want[q:q + nmine], lane
    assert got == want


def test_half_pass_mask_walk_takes_every_entry_once():
    rng = np.random.default_rng(14)
    mask_walk([[0] * 32], 1)
    mask_walk([[1] + [0] * 31], 1)
    mask_walk([[0xFFFFFFFF] * 32] * 5, 160)
    for _ in range(300):
        n = int(rng.integers(1, 161))
        W = (n + 31) // 32
        nh = int(rng.integers(1, 33))
        dens = rng.uniform(0.0, 1.0)
        mh = []
        for w in range(W):
            valid = min(32, n - 32 * w)
            row = []
            for h in range(32):
                bits = (rng.random(32) < dens) & (np.arange(32) < valid) & (h < nh) & (rng.random() > 0.15)
                row.append(int(sum(1 << b for b in range(32) if bits[b])))
            mh.append(row)
        mask_walk(mh, n)


def balanced_adjoint(toff, G=64):
    """The ACE site kernel's balanced adjoint sums (csrc/ace_site.cuh,
    adjoint_terms), restated: thread lt sums terms [lt·T/G, (lt+1)·T/G) density
    by density; a density split between threads is finished by the thread
    holding its first term from the later threads' partials.  Returns, per
    density, the list of term indices in the order they were added."""
    toff = list(toff)
    D, T = len(toff) - 1, toff[-1]
    dA = [[] for _ in range(D)]
    plo, phi, alo, ahi = [None] * G, [None] * G, [-1] * G, [-1] * G
    for lt in range(G):
        q0, q1 = lt * T // G, (lt + 1) * T // G
        if q0 >= q1:
            alo[lt] = -2  # an empty share
            continue
        lo, hi = 0, D - 1
        while lo < hi:
            mid = (lo + hi + 1) >> 1
            if toff[mid] <= q0:
                lo = mid
            else:
                hi = mid - 1
        a, q = lo, q0
        while q < q1:
            assert a < D
            qe = min(toff[a + 1], q1)
            left = q == q0 and toff[a] < q0
            right = qe == q1 and q1 < toff[a + 1]
            acc = list(range(q, qe))
            q = qe
            if left:
                plo[lt], alo[lt] = acc, a
            elif right:
                phi[lt], ahi[lt] = acc, a
            else:
                dA[a] = acc
            a += 1
    for lt in range(G):
        if ahi[lt] >= 0:
            a, acc = ahi[lt], list(phi[lt])
            t = lt + 1
            while t < G and alo[t] in (a, -2):
                if alo[t] == a:
                    acc += plo[t]
                t += 1
            dA[a] = acc
    return dA


def test_balanced_adjoint_sums_every_term_once_in_order():
    rng = np.random.default_rng(3)
    cases = [[0, 0], [0, 5], [0, 0, 300, 300, 301], [0, 265] + [265 + 3 * k for k in range(1, 60)]]
    for _ in range(200):
        D = int(rng.integers(1, 220))
        counts = rng.integers(0, 30, D) * (rng.random(D) > 0.2)
        if rng.random() < 0.3:
            counts[rng.integers(0, D)] += int(rng.integers(100, 400))
        cases.append(np.concatenate([[0], np.cumsum(counts)]).tolist())
    for toff in cases:
        for G in (64, 128):
            dA = balanced_adjoint(toff, G)
            for a in range(len(toff) - 1):
                assert dA[a] == list(range(toff[a], toff[a + 1])), (a, toff[:5])


def list_slot(slot, lane):
    """The shared-memory list layout (csrc/traverse.cuh): slot·32 + (lane ^ (slot & 31))."""
    return slot * 32 + (lane ^ (slot & 31))


def snapshot_fill(chunks, K=64):
    """The snapshot fill (csrc/snapshot.cu, k_nb_fill), restated for one warp.

    chunks: per chunk of home atoms, a list of drains; a drain gives each of
    the 32 lanes (centre atom id, or None) a list of (candidate id, in range).
    Returns the offsets of the count pass and the output array of
    (centre, candidate) written by the warp-cooperative fill."""
    # count pass: in-range candidates per centre
    count = {}
    for drains in chunks:
        for drain in drains:
            for centre, cand in drain:
                if centre is not None:
                    count[centre] = count.get(centre, 0) + sum(1 for _, ok in cand if ok)
    centres = sorted(count)
    offsets, total = {}, 0
    for a in centres:
        offsets[a] = total
        total += count[a]
    out = [None] * total
    written = [0] * total
    cur, o = [None] * 32, [0] * 32
    for drains in chunks:
        for drain in drains:
            lists = [None] * (K * 32)
            np_ = [0] * 32
            for lane, (centre, cand) in enumerate(drain):
                assert len(cand) <= K
                for q, item in enumerate(cand):
                    lists[list_slot(q, lane)] = item
                if centre is None:
                    continue
                if centre != cur[lane]:
                    cur[lane], o[lane] = centre, offsets[centre]
                # compaction in place: slot np <= q has been read already
                for q in range(len(cand)):
                    item = lists[list_slot(q, lane)]
                    if item[1]:
                        assert np_[lane] <= q
                        lists[list_slot(np_[lane], lane)] = item
                        np_[lane] += 1
            for L in range(32):
                for t0 in range(0, np_[L], 32):
                    slots = [list_slot(t, L) for t in range(t0, min(t0 + 32, np_[L]))]
                    assert len({s % 32 for s in slots}) == len(slots)  # distinct banks
                    for t in range(t0, min(t0 + 32, np_[L])):
                        e = o[L] + t
                        assert 0 <= e < total
                        out[e] = (cur[L], lists[list_slot(t, L)][0])
                        written[e] += 1
            for lane in range(32):
                o[lane] += np_[lane]
    return offsets, count, out, written


def test_snapshot_fill_writes_every_entry_once_in_visit_order():
    rng = np.random.default_rng(11)
    for _ in range(60):
        chunks, expect, next_id = [], {}, 0
        for _c in range(int(rng.integers(1, 4))):
            nh = int(rng.integers(1, 33))
            homes = list(range(next_id, next_id + nh))
            next_id += nh
            drains = []
            for _d in range(int(rng.integers(1, 6))):
                drain = []
                for lane in range(32):
                    if lane >= nh:
                        drain.append((None, []))
                        continue
                    n = int(rng.integers(0, 65)) if rng.random() > 0.1 else 0
                    cand = [(int(rng.integers(0, 10 ** 6)), bool(rng.random() < 0.6)) for _ in range(n)]
                    drain.append((homes[lane], cand))
                    expect.setdefault(homes[lane], []).extend(j for j, ok in cand if ok)
                drains.append(drain)
            chunks.append(drains)
        offsets, count, out, written = snapshot_fill(chunks)
        assert all(w == 1 for w in written)
        for a, js in expect.items():
            assert count[a] == len(js)
            assert [out[offsets[a] + k] for k in range(count[a])] == [(a, j) for j in js]


def test_per_cell_wrap_shift_is_the_minimum_image_lattice():
    """csrc/traverse.cuh pair_image: with L >= 4c the image of an in-range
    pair found through stencil offset o (shift s when the neighbour cell index
    wraps) is -rint(fl(fl(x_j - x_i) / L)) = s; checked per axis on wrapped
    coordinates, pairs placed at distances up to c(1 - 1e-15) and at cell and
    box edges."""
    rng = np.random.default_rng(5)
    wrapped = checked = 0
    for _ in range(300):
        c = float(rng.uniform(0.5, 10.0))
        dims = int(rng.integers(4, 40))
        L = float(rng.uniform(dims * c, (dims + 1) * c))  # floor(L / c) = dims
        dims = int(np.floor(L / c))
        assert dims >= 4
        size = L / dims
        xi = np.concatenate([rng.uniform(0.0, L, 200), [0.0, np.nextafter(L, 0.0), size, np.nextafter(size, 0.0)]])
        dist = np.concatenate([rng.uniform(-c, c, 200), [c * (1 - 1e-15), -c * (1 - 1e-15), 0.5 * c, -0.5 * c]])
        xj = np.mod(xi + dist, L)
        xj = np.where(xj >= L, 0.0, xj)
        ci = np.minimum(np.floor(xi / size).astype(int), dims - 1)
        cj = np.minimum(np.floor(xj / size).astype(int), dims - 1)
        for a_i, a_j, k_i, k_j in zip(xi, xj, ci, cj):
            for o in (-1, 0, 1):
                v = k_i + o
                s = -1 if v < 0 else (1 if v >= dims else 0)
                if (v - s * dims) != k_j:
                    continue
                d = (a_j - a_i) + s * L  # the kernel's displacement through this entry
                if abs(d) >= c:
                    continue
                lattice = -int(np.rint((a_j - a_i) / L))
                assert lattice == s, (c, L, a_i, a_j, o)
                checked += 1
                wrapped += s != 0
    assert checked > 30000 and wrapped > 1000, (checked, wrapped)
