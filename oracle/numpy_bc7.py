"""Second, independent restatement of the reference BC7 encoder -- TEST
INFRASTRUCTURE ONLY (the tests diff it against the C++ oracle; nothing else
imports it).

Written in numpy from the Rust of block_compression v0.3.0
(src/encode/bc7.rs, the coding helpers of src/encode/common.rs:520-613 and
the BC7 driver of src/encode.rs:609-660), separately from the C++ oracle:
every step runs on all blocks at once in float32 / integer arrays, with the
reference's operation order, and per-block decisions become masks. The
shared float primitives (block_quant, opt_endpoints, the PCA bound,
block_segment_core, ep_quant_dequant) are the ones of numpy_restatement.py;
the BPTC tables are the reference's own, extracted into
tests/golden/encoder_tables.json by tests/golden/make_golden.py.

Settings are the reference's BC7Settings as the u32 list of its #[repr(C)]
fields: refine_iterations[8], mode_selection[4], skip_mode2,
fast_skip_threshold_mode1, _mode3, _mode7, mode45_channel0,
refine_iterations_channel, channels.
"""
import json
import os

import numpy as np

from . import numpy_restatement as nr

F = np.float32
U32 = 0xFFFFFFFF
INF = F(np.inf)

_TABLES = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                       "encoder_tables.json")


def _tables():
    t = json.load(open(_TABLES))
    return (np.array(t["pattern"], np.int64), np.array(t["pattern_mask"], np.int64), np.array(t["skip"], np.int64))


PATTERN, PATTERN_MASK, SKIP = _tables()


def pattern_mask(part, j):
    """get_pattern_mask (common.rs:49-83) for arrays of partitions."""
    packed = PATTERN_MASK[part]
    m0, m1 = packed & 0xFFFF, packed >> 16
    if j == 0:
        return m0
    if j == 1:
        return m1
    return (~m0 & ~m1) & U32


def skips(part):
    """get_skips (common.rs:85-101): (n, 3)."""
    s = SKIP[part]
    return np.stack([np.zeros_like(s), s >> 4, s & 15], 1)


class Settings:
    def __init__(self, values):
        v = [int(x) for x in values]
        self.refine = v[0:8]
        self.mode_selection = v[8:12]
        self.skip_mode2 = v[12]
        self.t1, self.t3, self.t7 = v[13], v[14], v[15]
        self.channel0 = v[16]
        self.refine_channel = v[17]
        self.channels = v[18]


# ---- bit writer over n blocks (common.rs:103-124) ----------------------------------------


def put_bits(data, pos, bits, v):
    """put_bits at a position shared by every block; v (n,) non-negative."""
    v = np.asarray(v, np.int64) & ((1 << bits) - 1 if bits < 64 else -1)
    w, s = pos // 32, pos % 32
    data[:, w] |= (v << s) & U32
    if s + bits > 32:
        data[:, w + 1] |= (v >> (32 - s)) & U32
    return pos + bits


def data_shl_1bit_from(data, from_bits):
    """data_shl_1bit_from with a per-block from_bits (n,)."""
    fb = np.asarray(from_bits, np.int64)
    d = data.copy()
    lo = fb < 96
    hi = (fb >= 96) & (fb < 128)
    # from_bits < 96
    shifted = ((d[:, 2] >> 1) | (d[:, 3] << 31)) & U32
    mask = (((np.int64(1) << np.clip(fb - 64, 0, 31)) - 1) >> 1) & U32
    d2 = (mask & d[:, 2]) | (~mask & U32 & shifted)
    d3 = ((d[:, 3] >> 1) | (d[:, 4] << 31)) & U32
    d4 = d[:, 4] >> 1
    # 96 <= from_bits < 128
    shifted_h = ((d[:, 3] >> 1) | (d[:, 4] << 31)) & U32
    mask_h = (((np.int64(1) << np.clip(fb - 96, 0, 31)) - 1) >> 1) & U32
    d3h = (mask_h & d[:, 3]) | (~mask_h & U32 & shifted_h)
    data[:, 2] = np.where(lo, d2, data[:, 2])
    data[:, 3] = np.where(lo, d3, np.where(hi, d3h, data[:, 3]))
    data[:, 4] = np.where(lo | hi, d4, data[:, 4])


def code_qblock(data, pos, qblock, bits, flips):
    """bc7_code_qblock (common.rs:520-547)."""
    levels = 1 << bits
    for k in range(16):
        q = (qblock[:, k // 8] >> (4 * (k % 8))) & 15
        q = np.where((flips >> k) & 1 == 1, (levels - 1) - q, q)
        pos = put_bits(data, pos, bits - 1 if k == 0 else bits, q)
    return pos


def apply_swap_mode456(qep, channels, qblock, bits):
    """bc7_code_apply_swap_mode456 (common.rs:564-581), in place."""
    levels = 1 << bits
    sw = (qblock[:, 0] & 15) >= levels // 2
    for p in range(channels):
        a, b = qep[:, p].copy(), qep[:, channels + p].copy()
        qep[:, p] = np.where(sw, b, a)
        qep[:, channels + p] = np.where(sw, a, b)
    for i in range(2):
        qblock[:, i] = np.where(sw, ((0x11111111 * (levels - 1)) - qblock[:, i]) & U32, qblock[:, i])


def apply_swap_mode01237(qep, qblock, mode, part):
    """bc7_code_apply_swap_mode01237 (common.rs:583-613): swaps in place,
    returns the flip mask."""
    bits = 3 if mode in (0, 1) else 2
    pairs = 3 if mode in (0, 2) else 2
    levels = 1 << bits
    sk = skips(part)
    flips = np.zeros(qep.shape[0], np.int64)
    for j in range(pairs):
        k0 = sk[:, j]
        word = np.where(k0 >> 3 == 0, qblock[:, 0], qblock[:, 1])
        q = ((word << (28 - (k0 & 7) * 4)) & U32) >> 28
        sw = q >= levels // 2
        for p in range(4):
            a, b = qep[:, 8 * j + p].copy(), qep[:, 8 * j + 4 + p].copy()
            qep[:, 8 * j + p] = np.where(sw, b, a)
            qep[:, 8 * j + 4 + p] = np.where(sw, a, b)
        flips |= np.where(sw, pattern_mask(part, j), 0)
    return flips


def code_mode01237(qep, qblock, part, mode):
    """bc7_code_mode01237 (bc7.rs:381-440): (n, 4) words."""
    n = qep.shape[0]
    qep, qblock = qep.copy(), qblock.copy()
    bits = 3 if mode in (0, 1) else 2
    pairs = 3 if mode in (0, 2) else 2
    channels = 4 if mode == 7 else 3
    flips = apply_swap_mode01237(qep, qblock, mode, part)
    data = np.zeros((n, 5), np.int64)
    pos = put_bits(data, 0, mode + 1, np.full(n, 1 << mode))
    pos = put_bits(data, pos, 4, part & 15) if mode == 0 else put_bits(data, pos, 6, part & 63)
    width = {0: 4, 1: 6, 2: 5, 3: 7, 7: 5}[mode]
    for p in range(channels):
        for j in range(pairs * 2):
            v = qep[:, j * 4 + p]
            pos = put_bits(data, pos, width, v if mode == 2 else v >> 1)
    if mode == 1:
        for j in range(2):
            pos = put_bits(data, pos, 1, qep[:, j * 8] & 1)
    if mode in (0, 3, 7):
        for j in range(pairs * 2):
            pos = put_bits(data, pos, 1, qep[:, j * 4] & 1)
    pos = code_qblock(data, pos, qblock, bits, flips)
    # bc7_code_adjust_skip_mode01237 (common.rs:549-562)
    sk = skips(part)
    s1, s2 = sk[:, 1].copy(), sk[:, 2].copy()
    if pairs > 2:
        sw = s1 < s2
        s1, s2 = np.where(sw, s2, s1), np.where(sw, s1, s2)
    data_shl_1bit_from(data, 128 + (pairs - 1) - (15 - s1) * bits)
    if pairs > 2:
        data_shl_1bit_from(data, 128 + (pairs - 1) - (15 - s2) * bits)
    return data[:, :4]


def code_mode45(qep, qblock, aqep, aqblock, rotation, swap, mode):
    """bc7_code_mode45 (bc7.rs:442-492)."""
    n = qep.shape[0]
    qep, qblock, aqep, aqblock = qep.copy(), qblock.copy(), aqep.copy(), aqblock.copy()
    abits = 3 if mode == 4 else 2
    epbits = 5 if mode == 4 else 7
    aepbits = 6 if mode == 4 else 8
    s0 = swap == 0
    # swap == 0
    q0, a0, qb0, aqb0 = qep.copy(), aqep.copy(), qblock.copy(), aqblock.copy()
    apply_swap_mode456(q0, 4, qb0, 2)
    apply_swap_mode456(a0, 1, aqb0, abits)
    # swap == 1: the index sets exchange places
    q1, a1, qb1, aqb1 = qep.copy(), aqep.copy(), aqblock.copy(), qblock.copy()
    apply_swap_mode456(a1, 1, qb1, 2)
    apply_swap_mode456(q1, 4, aqb1, abits)
    qep = np.where(s0[:, None], q0, q1)
    aqep = np.where(s0[:, None], a0, a1)
    qblock = np.where(s0[:, None], qb0, qb1)
    aqblock = np.where(s0[:, None], aqb0, aqb1)
    data = np.zeros((n, 5), np.int64)
    pos = put_bits(data, 0, mode + 1, np.full(n, 1 << mode))
    pos = put_bits(data, pos, 2, (rotation + 1) & 3)
    if mode == 4:
        pos = put_bits(data, pos, 1, swap)
    for p in range(3):
        pos = put_bits(data, pos, epbits, qep[:, p])
        pos = put_bits(data, pos, epbits, qep[:, 4 + p])
    pos = put_bits(data, pos, aepbits, aqep[:, 0])
    pos = put_bits(data, pos, aepbits, aqep[:, 1])
    pos = code_qblock(data, pos, qblock, 2, np.zeros(n, np.int64))
    pos = code_qblock(data, pos, aqblock, abits, np.zeros(n, np.int64))
    return data[:, :4]


def code_mode6(qep, qblock):
    """bc7_code_mode6 (bc7.rs:494-515)."""
    n = qep.shape[0]
    qep, qblock = qep.copy(), qblock.copy()
    apply_swap_mode456(qep, 4, qblock, 4)
    data = np.zeros((n, 5), np.int64)
    pos = put_bits(data, 0, 7, np.full(n, 64))
    for p in range(4):
        pos = put_bits(data, pos, 7, qep[:, p] >> 1)
        pos = put_bits(data, pos, 7, qep[:, 4 + p] >> 1)
    pos = put_bits(data, pos, 1, qep[:, 0] & 1)
    pos = put_bits(data, pos, 1, qep[:, 4] & 1)
    pos = code_qblock(data, pos, qblock, 4, np.zeros(n, np.int64))
    return data[:, :4]


# ---- encoder (bc7.rs) ----------------------------------------------------------------------


def block_segment(block, mask, channels):
    """block_segment (bc7.rs:371-379): block_segment_core clamped to 0..255."""
    ep = nr.block_segment_core(block, mask, channels)
    for i in range(2):
        for p in range(channels):
            ep[:, 4 * i + p] = nr.clamp_f(ep[:, 4 * i + p], 0.0, 255.0)
    return ep


def qep24(qep, ep):
    out = np.zeros((ep.shape[0], 24), np.int64)
    out[:, :qep.shape[1]] = qep
    return out


class Encoder:
    """State of compress_block_bc7_core for n blocks."""

    def __init__(self, block, settings):
        self.block = np.asarray(block, F)
        self.s = Settings(settings)
        n = self.block.shape[0]
        self.n = n
        self.best_err = np.full(n, INF, F)
        self.data = np.zeros((n, 4), np.int64)
        # compute_opaque_err (bc7.rs:869-879)
        if self.s.channels == 3:
            self.opaque_err = np.zeros(n, F)
        else:
            e = F(0.0)
            for k in range(16):
                e = e + nr.sq(self.block[:, 48 + k] - F(255.0))
            self.opaque_err = np.asarray(e, F) * np.ones(n, F)

    def part_fast(self, part, mode):
        """bc7_enc_mode01237_part_fast (bc7.rs:517-538)."""
        bits = 3 if mode in (0, 1) else 2
        pairs = 3 if mode in (0, 2) else 2
        channels = 4 if mode == 7 else 3
        ep = np.zeros((self.n, 24), F)
        for j in range(pairs):
            ep[:, 8 * j:8 * j + 8] = block_segment(self.block, pattern_mask(part, j), channels)
        qep, ep = nr.ep_quant_dequant(ep, mode, channels)
        qblock, err = nr.block_quant(self.block, bits, ep, PATTERN[part], channels)
        return qep, qblock.astype(np.int64), err

    def enc_mode01237(self, mode, parts):
        """bc7_enc_mode01237 (bc7.rs:540-610); parts (n, count) partition ids."""
        count = parts.shape[1]
        if count == 0:
            return
        bits = 3 if mode in (0, 1) else 2
        pairs = 3 if mode in (0, 2) else 2
        channels = 4 if mode == 7 else 3
        best_qep = np.zeros((self.n, 24), np.int64)
        best_q = np.zeros((self.n, 2), np.int64)
        best_part = np.full(self.n, -1, np.int64)
        best = np.full(self.n, INF, F)
        for c in range(count):
            part = parts[:, c]
            qep, qblock, err = self.part_fast(part, mode)
            up = err < best
            best_qep[:, :8 * pairs] = np.where(up[:, None], qep[:, :8 * pairs], best_qep[:, :8 * pairs])
            best_q = np.where(up[:, None], qblock, best_q)
            best_part = np.where(up, part, best_part)
            best = np.where(up, err, best)
        found = best_part >= 0
        bp = np.where(found, best_part, 64 if pairs == 3 else 0)
        for _ in range(self.s.refine[mode]):
            ep = np.zeros((self.n, 24), F)
            for j in range(pairs):
                ep[:, 8 * j:8 * j + 8] = nr.opt_endpoints(ep[:, 8 * j:8 * j + 8], self.block, bits, best_q,
                                                          pattern_mask(bp, j), channels)
            qep, ep = nr.ep_quant_dequant(ep, mode, channels)
            qblock, err = nr.block_quant(self.block, bits, ep, PATTERN[bp], channels)
            qblock = qblock.astype(np.int64)
            up = (err < best) & found
            best_qep[:, :8 * pairs] = np.where(up[:, None], qep[:, :8 * pairs], best_qep[:, :8 * pairs])
            best_q = np.where(up[:, None], qblock, best_q)
            best = np.where(up, err, best)
        if mode != 7:
            best = best + self.opaque_err
        win = (best < self.best_err) & found
        if win.any():
            coded = code_mode01237(best_qep, best_q, bp, mode)
            self.data = np.where(win[:, None], coded, self.data)
            self.best_err = np.where(win, best, self.best_err)

    def bound_list(self, channels, k):
        """The 64 PCA split bounds and the first k entries of the ascending
        list (bc7.rs:628-640, 829-844; partial_sort_list, common.rs:126-140:
        the keys are unique, so its first k entries are the k smallest)."""
        keys = np.zeros((self.n, 64), np.int64)
        for part in range(64):
            mask = np.full(self.n, pattern_mask(np.array([part]), 0)[0], np.int64)
            b12 = nr.block_pca_bound_split(self.block, mask, channels)
            keys[:, part] = part + nr.as_int(b12) * 64
        return np.sort(keys, axis=1)[:, :k] & 63

    def opt_channel(self, cb, bits, epbits):
        """opt_channel (bc7.rs:239-266) with channel_quant_dequant,
        channel_opt_quant and channel_opt_endpoints (:268-369)."""
        n = self.n
        e0 = np.full(n, 255.0, F)
        e1 = np.zeros(n, F)
        for k in range(16):
            e0 = np.fmin(e0, cb[:, k])
            e1 = np.fmax(e1, cb[:, k])
        elevels = 1 << epbits

        def quant_dequant(a, b):
            qs, es = [], []
            for v in (a, b):
                q = np.clip(nr.as_int(v / F(255.0) * F(elevels - 1) + F(0.5)), 0, elevels - 1)
                vv = q << (8 - epbits)
                qs.append(q)
                es.append((vv + (vv >> epbits)).astype(F))
            return qs, es

        def opt_quant(a, b):
            levels = 1 << bits
            table = nr.UNQUANT[bits]
            qb = [np.zeros(n, np.int64), np.zeros(n, np.int64)]
            total = F(0.0)
            with np.errstate(divide="ignore", invalid="ignore"):
                for k in range(16):
                    proj = (cb[:, k] - a) / (b - a + F(0.001))
                    q1 = np.clip(nr.as_int(proj * F(levels) + F(0.5)), 1, levels - 1)
                    w0, w1 = table[q1 - 1], table[q1]
                    ia, ib = nr.as_int(a), nr.as_int(b)
                    v0 = nr.tdiv((64 - w0) * ia + w0 * ib + 32, 64).astype(F)
                    v1 = nr.tdiv((64 - w1) * ia + w1 * ib + 32, 64).astype(F)
                    err0 = F(0.0) + nr.sq(v0 - cb[:, k])
                    err1 = F(0.0) + nr.sq(v1 - cb[:, k])
                    t0 = err0 < err1
                    qb[k // 8] |= np.where(t0, q1 - 1, q1) << (4 * (k % 8))
                    total = total + np.where(t0, err0, err1)
            return np.stack(qb, 1), np.asarray(total, F)

        def opt_endpoints(qblock):
            l1 = F((1 << bits) - 1)
            atb1 = np.zeros(n, F)
            sum_q = np.zeros(n, F)
            sum_qq = np.zeros(n, F)
            s = np.zeros(n, F)
            for k in range(16):
                q = ((qblock[:, k // 8] >> (4 * (k % 8))) & 15).astype(F)
                x = l1 - q
                sum_q = sum_q + q
                sum_qq = sum_qq + q * q
                s = s + cb[:, k]
                atb1 = atb1 + x * cb[:, k]
            atb2 = l1 * s - atb1
            cxx = F(16.0) * nr.sq(l1) - F(2.0) * l1 * sum_q + sum_qq
            cyy = sum_qq
            cxy = l1 * sum_q - sum_qq
            det = cxx * cyy - cxy * cxy
            with np.errstate(divide="ignore", invalid="ignore"):
                scale = l1 / det
                a = nr.clamp_f((atb1 * cyy - atb2 * cxy) * scale, 0.0, 255.0)
                b = nr.clamp_f((atb2 * cxx - atb1 * cxy) * scale, 0.0, 255.0)
            flat = np.abs(det) < F(0.001)
            m = s / F(16.0)
            return np.where(flat, m, a).astype(F), np.where(flat, m, b).astype(F)

        (qa, qb_), (a, b) = quant_dequant(e0, e1)
        qblock, err = opt_quant(a, b)
        for _ in range(self.s.refine_channel):
            a, b = opt_endpoints(qblock)
            (qa, qb_), (a, b) = quant_dequant(a, b)
            qblock, err = opt_quant(a, b)
        return qblock, np.stack([qa, qb_], 1), err

    def mode45_candidate(self, cand, mode, rotation, swap):
        """bc7_enc_mode45_candidate (bc7.rs:657-733); updates `cand` where the
        candidate beats cand['err']."""
        bits, abits, aepbits = 2, 2, 8
        if mode == 4:
            abits, aepbits = 3, 6
        if swap == 1:
            bits, abits = 3, 2
        cb = np.zeros((self.n, 64), F)
        cb[:, :48] = self.block[:, :48]
        if rotation < 3:
            if self.s.channels == 4:
                cb[:, rotation * 16:rotation * 16 + 16] = self.block[:, 48:64]
            if self.s.channels == 3:
                cb[:, rotation * 16:rotation * 16 + 16] = F(255.0)
        full = np.full(self.n, 0xFFFFFFFF, np.int64)
        ep = np.zeros((self.n, 24), F)
        ep[:, :8] = block_segment(cb, full, 3)
        qep, ep = nr.ep_quant_dequant(ep, mode, 3)
        qblock, err = nr.block_quant(cb, bits, ep, np.zeros(self.n, np.int64), 3)
        for _ in range(self.s.refine[mode]):
            ep[:, :8] = nr.opt_endpoints(ep[:, :8], cb, bits, qblock, full, 3)
            qep, ep = nr.ep_quant_dequant(ep, mode, 3)
            qblock, err = nr.block_quant(cb, bits, ep, np.zeros(self.n, np.int64), 3)
        aqblock, aqep, aerr = self.opt_channel(self.block[:, rotation * 16:rotation * 16 + 16], abits, aepbits)
        err = err + aerr
        up = err < cand["err"]
        cand["qep"] = np.where(up[:, None], qep[:, :8], cand["qep"])
        cand["qblock"] = np.where(up[:, None], qblock.astype(np.int64), cand["qblock"])
        cand["aqblock"] = np.where(up[:, None], aqblock, cand["aqblock"])
        cand["aqep"] = np.where(up[:, None], aqep, cand["aqep"])
        cand["rotation"] = np.where(up, rotation, cand["rotation"])
        cand["swap"] = np.where(up, swap, cand["swap"])
        cand["err"] = np.where(up, err, cand["err"])

    def enc_mode45(self):
        """bc7_enc_mode45 (bc7.rs:735-760)."""
        n = self.n
        cand = {"qep": np.zeros((n, 8), np.int64), "qblock": np.zeros((n, 2), np.int64),
                "aqep": np.zeros((n, 2), np.int64), "aqblock": np.zeros((n, 2), np.int64),
                "rotation": np.zeros(n, np.int64), "swap": np.zeros(n, np.int64), "err": self.best_err.copy()}
        for p in range(self.s.channel0, self.s.channels):
            self.mode45_candidate(cand, 4, p, 0)
            self.mode45_candidate(cand, 4, p, 1)
        for mode in (4, 5):
            if mode == 5:
                for p in range(self.s.channel0, self.s.channels):
                    self.mode45_candidate(cand, 5, p, 0)
            win = cand["err"] < self.best_err
            if win.any():
                coded = code_mode45(cand["qep"], cand["qblock"], cand["aqep"], cand["aqblock"], cand["rotation"],
                                    cand["swap"], mode)
                self.data = np.where(win[:, None], coded, self.data)
                self.best_err = np.where(win, cand["err"], self.best_err)

    def enc_mode6(self):
        """bc7_enc_mode6 (bc7.rs:762-817)."""
        ch = self.s.channels
        full = np.full(self.n, 0xFFFFFFFF, np.int64)
        ep = np.zeros((self.n, 24), F)
        ep[:, :8] = block_segment(self.block, full, ch)
        if ch == 3:
            ep[:, 3] = F(255.0)
            ep[:, 7] = F(255.0)
        qep, ep = nr.ep_quant_dequant(ep, 6, ch)
        qblock, err = nr.block_quant(self.block, 4, ep, np.zeros(self.n, np.int64), ch)
        for _ in range(self.s.refine[6]):
            ep[:, :8] = nr.opt_endpoints(ep[:, :8], self.block, 4, qblock, full, ch)
            qep, ep = nr.ep_quant_dequant(ep, 6, ch)
            qblock, err = nr.block_quant(self.block, 4, ep, np.zeros(self.n, np.int64), ch)
        win = err < self.best_err
        if win.any():
            coded = code_mode6(qep[:, :8], qblock.astype(np.int64))
            self.data = np.where(win[:, None], coded, self.data)
            self.best_err = np.where(win, err, self.best_err)

    def encode(self):
        """compress_block_bc7_core (bc7.rs:853-867): (n, 4) uint32 words."""
        s = self.s
        if s.mode_selection[0]:
            self.enc_mode01237(0, np.tile(np.arange(16) + 64, (self.n, 1)))
            if s.skip_mode2 == 0:
                self.enc_mode01237(2, np.tile(np.arange(64) + 64, (self.n, 1)))
        if s.mode_selection[1]:
            if s.t1 or s.t3:
                lst = self.bound_list(3, max(s.t1, s.t3))
                self.enc_mode01237(1, lst[:, :s.t1])
                self.enc_mode01237(3, lst[:, :s.t3])
            if s.t7:
                self.enc_mode01237(7, self.bound_list(s.channels, s.t7))
        if s.mode_selection[2]:
            self.enc_mode45()
        if s.mode_selection[3]:
            self.enc_mode6()
        return (self.data & U32).astype(np.uint32)


def compress_bc7(img, settings):
    """compress_bc7 (src/encode.rs:609-660) of an (h, w, 4) uint8 image ->
    the packed little-endian 16-byte blocks, row-major."""
    words = Encoder(nr.planar_blocks(img), settings).encode()
    return np.ascontiguousarray(words.astype("<u4")).view(np.uint8).reshape(-1)
