"""CPU check of the transposed network's layout algebra for multi-warp and
cluster tiles (cuda-sort_b200/csrc/cta_xpose.cuh), restated here in numpy:
the window layouts, per-thread bases, compile-time register offsets, the
mirrored reflection window, the chain of windows of each stage, and the
cross-CTA layers in window layout LT.  The simulated network must equal the
reflection network of cusort_v6.hpp:90-142 with the keep-own rule of
cusort.hpp:460-472 element for element (payloads carry the input position,
so the order of equal keys is checked too), every store of a layout change
must write W distinct addresses, and (model of the shared-memory banks) the
accesses of a quarter-warp (16-byte elements) or half-warp (8-byte) must hit
distinct bank groups.
"""
import numpy as np
import pytest


def xp_addr(i, lk):
    return i + (i >> lk)


def reference(keys, pay):
    keys, pay = keys.copy(), pay.copy()
    idx = np.arange(len(keys))

    def layer(mask):
        lo = idx[idx < (idx ^ mask)]
        hi = lo ^ mask
        sw = keys[hi] < keys[lo]
        a, b = lo[sw], hi[sw]
        keys[a], keys[b] = keys[b].copy(), keys[a].copy()
        pay[a], pay[b] = pay[b].copy(), pay[a].copy()

    for st in range(len(keys).bit_length() - 1):
        layer((2 << st) - 1)
        for j in range(st - 1, -1, -1):
            layer(1 << j)
    return keys, pay


class Tile:
    """2^lc CTAs of 2^lt threads holding 2^lk registers each."""

    def __init__(self, lk, lt, lc, keys, pay, elem_bytes):
        self.lk, self.lt, self.lc = lk, lt, lc
        self.k, self.t_n, self.c = 1 << lk, 1 << lt, 1 << lc
        self.w = self.k * self.t_n
        self.eb = elem_bytes
        self.t = np.arange(self.t_n)
        self.vk = np.zeros((self.c, self.k, self.t_n), dtype=keys.dtype)
        self.vp = np.zeros_like(self.vk)
        for c in range(self.c):
            for q in range(self.k):
                g = c * self.w + self.t * self.k + q          # blocked load
                self.vk[c, q], self.vp[c, q] = keys[g], pay[g]
        size = xp_addr(self.w - 1, lk) + 1
        self.sk = np.zeros((self.c, size), dtype=keys.dtype)
        self.sp = np.zeros_like(self.sk)
        self.conflicts = 0

    # addresses of register q in window a (mirrored: upper half complemented)
    def addr(self, a, mir, q):
        h = self.k >> 1
        low = (1 << a) - 1
        m = mir and (q & h)
        lo = (self.t & low) ^ low if m else (self.t & low)
        base = xp_addr(((self.t >> a) << (a + self.lk)) | lo, self.lk)
        qq = q ^ (h - 1) if m else q
        return base + xp_addr(qq << a, self.lk)

    def banks(self, a):
        groups = 16 if self.eb == 8 else 8
        for w0 in range(0, self.t_n, 32):
            lanes = a[w0:w0 + 32]
            for g0 in range(0, 32, groups):
                part = lanes[g0:g0 + groups]
                unit = (part * self.eb // 16) % 8 if self.eb == 16 else (part * self.eb // 8) % 16
                self.conflicts += len(part) - len(set(unit.tolist()))

    def put(self, a, mir):
        for c in range(self.c):
            seen = []
            for q in range(self.k):
                ad = self.addr(a, mir, q)
                self.sk[c, ad], self.sp[c, ad] = self.vk[c, q], self.vp[c, q]
                seen.append(ad)
                if c == 0:
                    self.banks(ad)
            allad = np.concatenate(seen)
            assert len(np.unique(allad)) == self.w

    def get(self, a, mir):
        for c in range(self.c):
            for q in range(self.k):
                ad = self.addr(a, mir, q)
                self.vk[c, q], self.vp[c, q] = self.sk[c, ad], self.sp[c, ad]
                if c == 0:
                    self.banks(ad)

    def move(self, af, mf, at, mt):
        self.put(af, mf)
        self.get(at, mt)

    def cex(self, lo, hi):
        sw = self.vk[:, hi] < self.vk[:, lo]
        for v in (self.vk, self.vp):
            a, b = v[:, lo].copy(), v[:, hi].copy()
            v[:, lo], v[:, hi] = np.where(sw, b, a), np.where(sw, a, b)

    def merges(self, r_hi):
        for r in range(r_hi, -1, -1):
            for q in range(self.k):
                if not q & (1 << r):
                    self.cex(q, q | (1 << r))

    def chain(self, acur, mcur, hi):
        if hi < 0:
            if acur or mcur:
                self.move(acur, mcur, 0, False)
            return
        an = max(hi - self.lk + 1, 0)
        if an != acur or mcur:
            self.move(acur, mcur, an, False)
        self.merges(hi - an)
        if an > 0:
            self.chain(an, False, an - 1)

    def stage(self, st):
        k, h = self.k, self.k >> 1
        if st < self.lk:
            m = (2 << st) - 1
            for q in range(k):
                if q < q ^ m:
                    self.cex(q, q ^ m)
            if st:
                self.merges(st - 1)
            return
        a1 = st - self.lk + 1
        self.move(0, False, a1, True)
        for q in range(h):
            self.cex(q, q + h)
        for r in range(self.lk - 2, -1, -1):
            for q in range(k):
                if not q & (1 << r):
                    if q & h:
                        self.cex(q | (1 << r), q)
                    else:
                        self.cex(q, q | (1 << r))
        self.chain(a1, True, a1 - 1)

    def cluster_layer(self, reflect, cm, upper):
        self.put(self.lt, False)
        nk, npay = self.vk.copy(), self.vp.copy()
        for c in range(self.c):
            pc = c ^ cm
            pt = self.t_n - 1 - self.t if reflect else self.t
            for q in range(self.k):
                ad = xp_addr(pt, self.lk) + xp_addr((self.k - 1 - q if reflect else q) << self.lt, self.lk)
                bk, bp = self.sk[pc, ad], self.sp[pc, ad]
                own = self.vk[c, q]
                take = own < bk if upper(c) else bk < own
                nk[c, q] = np.where(take, bk, own)
                npay[c, q] = np.where(take, bp, self.vp[c, q])
        self.vk, self.vp = nk, npay

    def network(self):
        local = self.lk + self.lt
        for st in range(local):
            self.stage(st)
        for st in range(local, local + self.lc):
            self.move(0, False, self.lt, False)
            self.cluster_layer(True, (2 << (st - local)) - 1, lambda c, s=st: (c >> (s - local)) & 1)
            for j in range(st - 1, local - 1, -1):
                self.cluster_layer(False, 1 << (j - local), lambda c, j=j: (c >> (j - local)) & 1)
            self.merges(self.lk - 1)
            self.chain(self.lt, False, self.lt - 1)

    def result(self):
        n = self.c * self.w
        keys = np.zeros(n, dtype=self.vk.dtype)
        pay = np.zeros(n, dtype=self.vp.dtype)
        for c in range(self.c):
            for q in range(self.k):
                g = c * self.w + self.t * self.k + q
                keys[g], pay[g] = self.vk[c, q], self.vp[c, q]
        return keys, pay


# (log2 registers, log2 threads, log2 CTAs, element bytes): the shapes of the
# compiled tiles, scaled down in threads where the algebra does not change
SHAPES = [(4, 5, 0, 8), (4, 6, 0, 16), (5, 6, 0, 8), (4, 7, 0, 8), (4, 5, 1, 16), (4, 6, 2, 8), (4, 5, 3, 16),
          (5, 5, 1, 8)]


@pytest.mark.parametrize("lk,lt,lc,eb", SHAPES)
@pytest.mark.parametrize("distinct", [3, 1 << 30])
def test_transposed_tile_equals_the_reference_network(lk, lt, lc, eb, distinct):
    rng = np.random.default_rng(lk * 100 + lt * 10 + lc)
    w = 1 << (lk + lt + lc)
    keys = rng.integers(0, distinct, w).astype(np.int64)
    pay = np.arange(w, dtype=np.int64)
    want_k, want_p = reference(keys, pay)
    tile = Tile(lk, lt, lc, keys, pay, eb)
    tile.network()
    got_k, got_p = tile.result()
    assert np.array_equal(got_k, want_k)
    assert np.array_equal(got_p, want_p)      # tie order of equal keys included
    assert tile.conflicts == 0
